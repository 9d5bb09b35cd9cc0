"""GPU parity at full size for the NLGEOM path: the C3D4 beam the benchmark times
(240,000 C3D4, 133,623 DOF; E(T) table, initial temperature gradient 20 -> 220 C,
tip load ramped by *AMPLITUDE over 10 increments, NLGEOM) against the oracle's FP64
Cholesky Newton run committed in tests/golden/oracle_c3d4_nlgeom_beam.npz
(tests/golden/make_fixtures.py beam).

Tolerance: relative displacement error in the 2-norm, 1e-8 (each increment's Newton
iterations follow the oracle's; the last update carries the linear-solve error), and
the same number of increments as the oracle.
"""
import os

import numpy as np
import pytest

import ferrix_b200 as fx
from ferrix_b200 import decks
from tests.golden.make_fixtures import BEAM_FIXTURE, deck_digest

pytestmark = pytest.mark.gpu

TOL_NLGEOM = 1e-8

ARMS = [
    ("mixed_amg (default)", fx.PREC_MIXED, fx.PRECOND_AMG),
    ("fp64_amg", fx.PREC_FP64, fx.PRECOND_AMG),
    ("fp64_block_jacobi", fx.PREC_FP64, fx.PRECOND_BLOCK_JACOBI),
]


@pytest.fixture(scope="module")
def beam(golden_dir):
    fix = np.load(os.path.join(golden_dir, BEAM_FIXTURE))
    text = decks.c3d4_nlgeom_beam()
    assert str(fix["deck_sha256"]) == deck_digest(text), "deck generator changed: regenerate the fixture"
    ctx = fx.Context(0)
    p = fx.Project.from_inp_text(text, ctx)
    p.default_initial_temperature = 20.0
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    yield p, st, fix
    p.close()
    ctx.close()


@pytest.mark.parametrize("name,prec,pc", ARMS, ids=[a[0] for a in ARMS])
def test_nlgeom_beam_133k_dof_matches_oracle(beam, name, prec, pc):
    p, st, fix = beam
    assert p.num_dofs == 133623
    st.initialize(p)
    stats = p.steps[0].solve(1, p, st, opts=fx.solve_opts(precision=prec, preconditioner=pc))
    assert stats["increments"] == int(fix["increments"]), (name, stats)
    ref = fix["u"]
    err = float(np.linalg.norm(st.displacements - ref) / np.linalg.norm(ref))
    assert err <= TOL_NLGEOM, (name, err, stats)
