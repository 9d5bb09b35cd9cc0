"""Test helper: the arrays of a deck, for Project.from_arrays (fx_model_from_arrays).

The deck is parsed by the oracle's restatement of the reference parser
(src/solver/parser.rs:111-482) and its Project is written out as the arrays the
binary mesh entry point takes, so a test can build the same model both ways.
"""
from __future__ import annotations

import numpy as np

from oracle import inp

_SOLVERS = {"DEFAULT": 0, "DIRECT": 1, "ITERATIVE": 2}


def arrays_from_deck(text: str, default_temperature: float = 0.0) -> dict:
    o = inp.parse_inp_text(text)
    node_ids = np.fromiter(o.nodes.keys(), dtype=np.int64, count=len(o.nodes))
    xyz = np.array([o.nodes[i] for i in node_ids], dtype=np.float64).reshape(-1, 3)
    groups = {}
    for npe, name in ((4, "C3D4"), (20, "C3D20")):
        ids = [eid for eid, (t, _) in o.elements.items() if t == name]
        conn = np.array([o.elements[e][1] for e in ids], dtype=np.int64).reshape(-1, npe)
        mat = np.array([o.element_materials.get(e, -1) for e in ids], dtype=np.int32)
        groups[npe] = (np.array(ids, dtype=np.int64), conn, mat) if ids else None

    def pairs(lut):
        return [] if lut is None else list(lut.data)

    materials = [{"name": m.name, "E": pairs(m.youngs_modulus), "nu": pairs(m.poisson_ratio),
                  "alpha": pairs(m.thermal_expansion), "tref": m.reference_temperature} for m in o.materials]
    amps, index = [], {}

    def amp_index(a):
        if a is None or a.times is None:
            return -1
        if id(a) not in index:
            index[id(a)] = len(amps)
            amps.append({"time": list(a.times), "value": list(a.values), "total_time": a.total_time,
                         "shift_x": a.shift_x, "shift_y": a.shift_y})
        return index[id(a)]

    steps = []
    for st in o.steps:
        inc = st.increment
        steps.append({
            "nlgeom": st.nlgeom, "solver": _SOLVERS[st.solver],
            "increment": (inc.initial_time_increment, inc.time_period, inc.min_time_increment,
                          inc.max_time_increment),
            "max_increments": inc.max_iterations,
            "loads": [(r.node_id, r.dof, r.value, amp_index(r.amplitude), r.origin_step) for r in st.loads],
            "bcs": [(r.node_id, r.dof, r.value, amp_index(r.amplitude), r.origin_step) for r in st.bcs],
        })
    return {"node_ids": node_ids, "xyz": xyz, "c3d4": groups[4], "c3d20": groups[20], "materials": materials,
            "amplitudes": amps, "steps": steps, "default_temperature": default_temperature,
            "initial_temperatures": dict(o.initial_temperatures)}
