"""Result fields on the GPU against the oracle: nodal-averaged stress / strain
(StaticStep::calculate_stress_strain, static_step.rs:271-379) and the VTK
writer (io/vtk.rs:72-319).

Tolerances: stress and strain 1e-10 of the largest entry (FP64 throughout, only
summation orders differ); VTK values read back 1e-12 relative (shortest
round-trip number formatting)."""
import numpy as np
import pytest

import ferrix_b200 as fx
from ferrix_b200 import decks
from oracle import inp, stress

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = fx.Context(0)
    yield c
    c.close()


CASES = {
    "c3d4_box": lambda: decks.c3d4_cantilever(3, 4, 5),
    "c3d20_jittered": lambda: decks.c3d20_box(2, 3, 4),
    "tdep_thermal_beam": lambda: decks.c3d4_nlgeom_beam(6, 2, 2),
}


def _setup(ctx, text, rng):
    p = fx.Project.from_inp_text(text, ctx)
    p.default_initial_temperature = 20.0
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    st.initialize(p)
    o = inp.parse_inp_text(text)
    o.default_initial_temperature = 20.0
    t0 = inp.initial_temperatures(o)
    t1 = t0 + rng.uniform(0.0, 150.0, size=t0.shape)  # T_cur != T_init exercises the thermal strain change
    st.set_temperatures(t0, t1)
    u = rng.normal(scale=1e-2, size=p.num_dofs)
    st.displacements = u
    return p, st, o, u, t0, t1


@pytest.mark.parametrize("case", list(CASES))
def test_nodal_stress_strain_matches_oracle(ctx, case):
    rng = np.random.default_rng(7)
    p, st, o, u, t0, t1 = _setup(ctx, CASES[case](), rng)
    S, E = p.nodal_stress_strain()
    S_or, E_or = stress.nodal_stress_strain(o, u, t0, t1)
    assert np.abs(S - S_or).max() <= 1e-10 * np.abs(S_or).max()
    assert np.abs(E - E_or).max() <= 1e-10 * np.abs(E_or).max()


def test_stress_after_a_solve(ctx):
    text = decks.c3d20_box(2, 2, 6)
    p = fx.Project.from_inp_text(text, ctx)
    p.default_initial_temperature = 20.0
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    st.initialize(p)
    p.steps[0].solve(1, p, st)
    u = st.displacements
    S, E = p.nodal_stress_strain()
    o = inp.parse_inp_text(text)
    o.default_initial_temperature = 20.0
    t = inp.initial_temperatures(o)
    S_or, E_or = stress.nodal_stress_strain(o, u, t, t)
    assert np.abs(S - S_or).max() <= 1e-10 * np.abs(S_or).max()
    assert np.abs(E - E_or).max() <= 1e-10 * np.abs(E_or).max()


def _read_vtk(path):
    lines = open(path).read().split("\n")
    out, k = {}, 0
    while k < len(lines):
        w = lines[k].split()
        if not w:
            k += 1
            continue
        if w[0] == "POINTS":
            n = int(w[1])
            out["POINTS"] = np.array([[float(v) for v in l.split()] for l in lines[k + 1:k + 1 + n]])
            k += 1 + n
        elif w[0] == "CELLS":
            n = int(w[1])
            out["CELLS"] = [[int(v) for v in l.split()] for l in lines[k + 1:k + 1 + n]]
            out["CELLS_SIZE"] = int(w[2])
            k += 1 + n
        elif w[0] == "CELL_TYPES":
            n = int(w[1])
            out["CELL_TYPES"] = [int(l) for l in lines[k + 1:k + 1 + n]]
            k += 1 + n
        elif w[0] == "POINT_DATA":
            out["N"] = int(w[1])
            k += 1
        elif w[0] == "VECTORS":
            n = out["N"]
            out[w[1]] = np.array([[float(v) for v in l.split()] for l in lines[k + 1:k + 1 + n]])
            k += 1 + n
        elif w[0] == "SCALARS":
            n = out["N"]
            out[w[1]] = np.array([[float(v) for v in l.split()] for l in lines[k + 2:k + 2 + n]])
            k += 2 + n
        else:
            k += 1
    return out


def test_vtk_file_matches_oracle(ctx, tmp_path):
    rng = np.random.default_rng(9)
    text = decks.c3d20_box(2, 2, 3)
    p, st, o, u, t0, t1 = _setup(ctx, text, rng)
    path = str(tmp_path / "step_1_1.vtk")
    p.write_vtk(path)
    v = _read_vtk(path)
    S_or, E_or = stress.nodal_stress_strain(o, u, t0, t1)
    xyz = np.asarray([o.nodes[i] for i in o.index_to_node_id])
    assert np.array_equal(v["POINTS"], xyz)
    n_el = len(o.elements)
    assert len(v["CELLS"]) == n_el and v["CELLS_SIZE"] == 21 * n_el and set(v["CELL_TYPES"]) == {25}
    conn = {tuple(c[1:]) for c in v["CELLS"]}
    want = {tuple(o.node_id_to_index[n] for n in nodes) for _, nodes in o.elements.values()}
    assert conn == want
    assert np.array_equal(v["U"], u.reshape(-1, 3))
    assert np.abs(v["S"] - S_or).max() <= 1e-10 * np.abs(S_or).max()
    assert np.abs(v["E"] - E_or).max() <= 1e-10 * np.abs(E_or).max()
    assert np.array_equal(v["NT"][:, 0], t1)
    assert np.abs(v["MISES"][:, 0] - stress.mises(S_or)).max() <= 1e-9 * stress.mises(S_or).max()
    assert np.abs(v["TRESCA"][:, 0] - stress.tresca(S_or)).max() <= 1e-9 * stress.tresca(S_or).max()
