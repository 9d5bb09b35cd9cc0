"""fx_model_from_arrays on the GPU: a deck solved from its text and from its
arrays gives the same displacements bit for bit (the two entry points build the
same model), and both match the oracle's FP64 direct solution (1e-8, the
default mixed solver)."""
import gzip
import os

import numpy as np
import pytest

import ferrix_b200 as fx
from ferrix_b200 import decks
from oracle import inp, static_step
from tests.deck_arrays import arrays_from_deck

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = fx.Context(0)
    yield c
    c.close()


def _solve_all(p):
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    st.initialize(p)
    out = []
    for k, step in enumerate(p.steps):
        step.solve(k + 1, p, st)
        out.append(st.displacements)
    return out


def _deck(golden_dir, name):
    with gzip.open(os.path.join(golden_dir, "decks", name + ".inp.gz"), "rt") as fh:
        return fh.read()


@pytest.mark.parametrize("name", ["C3D4_2staticstep", "C3D20", "NLGEOM_test"])
def test_reference_deck_from_arrays_solves_bitwise_like_its_text(ctx, golden_dir, name):
    text = _deck(golden_dir, name)
    a = fx.Project.from_inp_text(text, ctx)
    a.default_initial_temperature = 20.0
    b = fx.Project.from_arrays(**arrays_from_deck(text, default_temperature=20.0), ctx=ctx)
    for ua, ub in zip(_solve_all(a), _solve_all(b)):
        assert np.array_equal(ua, ub)
    fix = np.load(os.path.join(golden_dir, f"oracle_{name}.npz"))
    ref = fix[f"step{len(a.steps)}"]
    tol = 1e-8
    assert np.linalg.norm(ub - ref) <= tol * np.linalg.norm(ref)


@pytest.mark.parametrize("spec", [lambda: decks.c3d4_nlgeom_beam_spec(12, 3, 3, tip_load=2.0e3, increments=4),
                                  lambda: decks.c3d20_box_spec(3, 3, 8)])
def test_generated_model_from_arrays_solves_bitwise_like_its_text(ctx, spec):
    s = spec()
    text = decks.write_deck(s)
    a = fx.Project.from_inp_text(text, ctx)
    a.default_initial_temperature = 20.0
    b = fx.Project.from_arrays(**dict(decks.deck_arrays(s), default_temperature=20.0), ctx=ctx)
    ua, ub = _solve_all(a)[-1], _solve_all(b)[-1]
    assert np.array_equal(ua, ub)
    o = inp.parse_inp_text(text)
    o.default_initial_temperature = 20.0
    ref = static_step.Runner(o).run().displacements
    assert np.linalg.norm(ub - ref) <= 1e-8 * np.linalg.norm(ref)


def test_arrays_model_served_by_the_request_loop(ctx):
    """A host-only model from arrays goes through fx_server_* like a parsed deck."""
    kw, _ = decks.random_box(np.random.default_rng(4), 8000.0, 4, arrays=True)
    srv = fx.Server(0, slots=2)
    try:
        p = fx.Project.from_arrays(**dict(kw, default_temperature=20.0))
        u, r = srv.wait(srv.submit(p), timeout=600.0)
    finally:
        srv.close()
    assert r["status"] == 0
    q = fx.Project.from_arrays(**dict(kw, default_temperature=20.0), ctx=ctx)
    assert np.array_equal(u, _solve_all(q)[0])
