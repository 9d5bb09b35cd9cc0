"""GPU parity at full size: the 417,123-DOF C3D20 box the benchmark solves
(20x20x80 bricks, interior nodes jittered, clamped z=0, 5000 N on z=80),
every solver arm against the oracle's FP64 multifrontal-Cholesky solution
committed in tests/golden/oracle_c3d20_box.npz (tests/golden/make_fixtures.py box).

Tolerance: relative displacement error in the 2-norm, 1e-10 for the FP64
solvers and 1e-8 for the mixed ones, at the default rtol = 1e-8.
"""
import os

import numpy as np
import pytest

import ferrix_b200 as fx
from ferrix_b200 import decks
from tests.golden.make_fixtures import BOX_FIXTURE, deck_digest

pytestmark = pytest.mark.gpu

ARMS = [
    ("mixed_amg (default)", fx.PREC_MIXED, fx.PRECOND_AMG, 1e-8),
    ("fp64_amg", fx.PREC_FP64, fx.PRECOND_AMG, 1e-10),
    ("mixed_block_jacobi", fx.PREC_MIXED, fx.PRECOND_BLOCK_JACOBI, 1e-8),
    ("fp64_block_jacobi", fx.PREC_FP64, fx.PRECOND_BLOCK_JACOBI, 1e-10),
    ("plain_fp64_csr_jacobi", fx.PREC_FP64_CSR, fx.PRECOND_BLOCK_JACOBI, 1e-10),
]


@pytest.fixture(scope="module")
def box(golden_dir):
    fix = np.load(os.path.join(golden_dir, BOX_FIXTURE))
    text = decks.c3d20_box()
    assert str(fix["deck_sha256"]) == deck_digest(text), "deck generator changed: regenerate the fixture"
    ctx = fx.Context(0)
    p = fx.Project.from_inp_text(text, ctx)
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    yield p, st, fix["u"]
    p.close()
    ctx.close()


@pytest.mark.parametrize("name,prec,pc,tol", ARMS, ids=[a[0] for a in ARMS])
def test_c3d20_box_417k_dof_matches_oracle(box, name, prec, pc, tol):
    p, st, ref = box
    assert p.num_dofs == 417123
    st.initialize(p)
    stats = p.steps[0].solve(1, p, st, opts=fx.solve_opts(precision=prec, preconditioner=pc))
    err = float(np.linalg.norm(st.displacements - ref) / np.linalg.norm(ref))
    assert err <= tol, (name, err, stats["pcg_iterations"])
