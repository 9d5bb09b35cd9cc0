"""Request loop (fx_server_*): results alone vs in the mix, admission by HBM
footprint, and agreement with the oracle's direct solve.

Tolerance: displacement 1e-8 relative (2-norm) against the oracle; results of
the same deck alone and in the mix are compared bit for bit (each request runs
the same launch sequence on its own stream)."""
import numpy as np
import pytest

import ferrix_b200 as fx
from ferrix_b200 import decks
from oracle import inp, static_step

pytestmark = pytest.mark.gpu


def _pool():
    # mixed C3D4 / C3D20 boxes of uneven size (1.5k - 40k DOF)
    return [text for text, _ in decks.batch_population(8, seed=5, dof_lo=1500, dof_hi=40000, c3d20_fraction=0.4)]


def _host_project(text):
    p = fx.Project.from_inp_text(text)
    p.default_initial_temperature = 20.0
    return p


def _serve(texts, slots, budget=0.0, opts=None):
    srv = fx.Server(0, slots=slots, hbm_budget_bytes=budget, opts=opts)
    try:
        projs = [_host_project(t) for t in texts]
        tickets = [srv.submit(p) for p in projs]
        out = [srv.wait(t, timeout=600.0) for t in tickets]
    finally:
        srv.close()
    for p in projs:
        p.close()
    return out


@pytest.mark.parametrize("preconditioner", [fx.PRECOND_BLOCK_JACOBI, fx.PRECOND_AMG])
def test_results_same_alone_and_in_the_mix(preconditioner):
    texts = _pool()
    opts = fx.solve_opts(precision=fx.PREC_MIXED, preconditioner=preconditioner)
    alone = [_serve([t], 1, opts=opts)[0] for t in texts]
    mixed = _serve(texts, 4, opts=opts)
    for (ua, ra), (um, rm) in zip(alone, mixed):
        assert ra["status"] == 0 and rm["status"] == 0, (ra["error"], rm["error"])
        assert np.array_equal(ua, um)
    # the mix overlapped on the device: some admission happened before an earlier request finished
    spans = sorted((r["admit_at_ms"], r["done_at_ms"]) for _, r in mixed)
    assert any(spans[i + 1][0] < spans[i][1] for i in range(len(spans) - 1))
    for text, (u, _) in list(zip(texts, mixed))[:3]:
        o = inp.parse_inp_text(text)
        o.default_initial_temperature = 20.0
        ref = static_step.Runner(o).run().displacements
        assert np.linalg.norm(u - ref) <= 1e-8 * np.linalg.norm(ref)


def test_admission_by_footprint_serialises_when_budget_is_small():
    texts = _pool()[:4]
    out = _serve(texts, 4, budget=1.0)  # every request exceeds the budget: each runs alone
    spans = sorted((r["admit_at_ms"], r["done_at_ms"]) for _, r in out)
    for i in range(len(spans) - 1):
        assert spans[i + 1][0] >= spans[i][1]
    assert all(r["status"] == 0 for _, r in out)
    assert all(r["footprint_bytes"] > 1.0 for _, r in out)


def test_failed_request_reports_its_error_and_the_loop_continues():
    # parses, but its elements have no section (no material): fails at solve time
    bad = decks.c3d4_cantilever(2, 2, 2).replace("*Solid section, Elset=Vol, Material=Mat", "**", 1)
    good = decks.c3d4_cantilever(2, 2, 4)
    srv = fx.Server(0, slots=2)
    try:
        pb = _host_project(bad)
        pg = _host_project(good)
        tb = srv.submit(pb)
        tg = srv.submit(pg)
        u, r = srv.wait(tb, timeout=120.0)
        assert u is None and r["status"] == 13 and "material" in r["error"].lower()
        u, r = srv.wait(tg, timeout=120.0)
        assert r["status"] == 0 and np.all(np.isfinite(u))
    finally:
        srv.close()


def test_wait_with_a_short_limit_reports_not_finished():
    """Failure detection on the host: a wait that runs out returns FX_TIMEOUT and the ticket stays valid."""
    srv = fx.Server(0, slots=1)
    try:
        big = _host_project(decks.c3d20_box(10, 10, 40))
        t = srv.submit(big)
        with pytest.raises(fx.FerrixError) as e:
            srv.wait(t, timeout=0.0)
        assert e.value.kind == "Timeout"
        u, r = srv.wait(t, timeout=600.0)
        assert r["status"] == 0 and np.all(np.isfinite(u))
    finally:
        srv.close()
    big.close()


def test_closing_the_server_cancels_queued_requests_and_models_stay_usable():
    texts = _pool()[:6]
    projs = [_host_project(t) for t in texts]
    srv = fx.Server(0, slots=1)
    for p in projs:
        srv.submit(p)
    srv.close()  # finishes the running request, cancels the rest
    # every model is unbound again and can be served by a new loop
    out = _serve_projects(projs, 2)
    assert all(r["status"] == 0 for _, r in out)
    for p in projs:
        p.close()


def _serve_projects(projs, slots):
    srv = fx.Server(0, slots=slots)
    try:
        tickets = [srv.submit(p) for p in projs]
        return [srv.wait(t, timeout=600.0) for t in tickets]
    finally:
        srv.close()


def test_server_reports_its_setup():
    """fx_server_get_info: every slot found all kernels loaded, and the HBM budget is held in the
    device's memory pool (so that no request grows the pool while other requests' kernels run)."""
    srv = fx.Server(0, slots=3, hbm_budget_bytes=2e9)
    try:
        info = srv.info()
    finally:
        srv.close()
    assert info["slots"] == 3
    assert info["preloaded_kernels"] >= 50, info
    assert info["reservation"] in (0, 1), info
    assert info["budget_bytes"] == 2e9 and info["pool_reserved_bytes"] >= 2e9, info
