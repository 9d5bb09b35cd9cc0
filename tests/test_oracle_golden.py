"""The oracle against the CalculiX displacement goldens of tests/calculix_parity.rs."""
import gzip
import json
import os

import numpy as np
import pytest

from oracle import inp, static_step

CASES = ["C3D4_staticstep", "C3D4_2staticstep", "C3D20", "NLGEOM_test"]


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_calculix(golden_dir, name):
    gold = json.load(open(os.path.join(golden_dir, "calculix.json")))[name]
    with gzip.open(os.path.join(golden_dir, "decks", name + ".inp.gz"), "rt") as fh:
        p = inp.parse_inp_text(fh.read())
    p.default_initial_temperature = 20.0  # tests/calculix_parity.rs:29
    runner = static_step.Runner(p)
    state = static_step.new_state(p)
    timer = inp.SolverTime()
    idx = p.index_of(gold["node"])
    fix = np.load(os.path.join(golden_dir, f"oracle_{name}.npz"))
    for k, want in enumerate(gold["steps"]):
        runner.solve_step(k, state, timer)
        u = state.displacements[3 * idx:3 * idx + 3]
        assert np.all(np.abs(u - np.array(want)) < gold["tol"]), (name, k, u, want)
        ref = fix[f"step{k + 1}"]
        assert np.linalg.norm(state.displacements - ref) <= 1e-9 * np.linalg.norm(ref)
