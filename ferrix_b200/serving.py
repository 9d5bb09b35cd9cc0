"""Serving-loop measurement: a seeded Poisson stream of deck requests through
`Server` (fx_server_*), with latency percentiles and throughput.

Pool: mixed C3D4 (60 %) / C3D20 (40 %) boxes, DOF log-uniform in
[dof_lo, dof_hi], E log-uniform [70, 210] GPa, nu uniform [0.25, 0.35], one face
clamped, a random-direction load of 100-5000 N on the opposite face. Each
request draws a pool deck; its model is parsed on the host before the timed
stream starts (a request carries an already parsed deck), so latency counts
from submission: queueing for a slot and HBM budget, upload, symbolic pattern,
assembly, solve to 1e-8 and the download of the displacements. The result
splits each request's latency into queueing, set-up / upload, the solve (host
wall time and device time) and download / release, as p50 / p99.
"""
from __future__ import annotations

import ctypes as C
import time
from typing import Dict, List, Optional

import numpy as np

from . import Project, Server, decks, _lib


def make_pool(n: int = 16, seed: int = 2027, dof_lo: float = 5e3, dof_hi: float = 5e5,
              c3d20_fraction: float = 0.4, arrays: bool = False) -> List[object]:
    """The seeded deck pool: deck texts, or with arrays=True the same models as
    Project.from_arrays arguments (the binary mesh path, no text)."""
    return [d for d, _ in decks.batch_population(n, seed=seed, dof_lo=dof_lo, dof_hi=dof_hi,
                                                  c3d20_fraction=c3d20_fraction, arrays=arrays)]


def _host_model(entry) -> Project:
    if isinstance(entry, dict):
        p = Project.from_arrays(**dict(entry, default_temperature=20.0))
    else:
        p = Project.from_inp_text(entry)
        p.default_initial_temperature = 20.0
    n4 = C.c_int64()
    n20 = C.c_int64()
    # builds the dense arrays now (counts only), so that submission is cheap
    p.lib.fx_model_export(p.handle, None, C.byref(n4), None, None, C.byref(n20), None, None)
    return p


def run_stream(pool: List[str], rate: float, n_requests: int, opts, device: int = 0, slots: int = 4,
               seed: int = 0, hbm_budget_bytes: float = 0.0, keep: Optional[List[int]] = None,
               each_once: bool = False) -> Dict:
    """Submits n_requests at Poisson arrival times (rate per second) and waits for all.

    The decks are drawn from `pool` at random (with replacement), or with each_once
    every deck of the pool once in a random order (n_requests = len(pool)). Returns
    latency percentiles (ms), throughput (solves/s, first submission to last
    completion) and per-request records; `keep` lists pool indices whose
    displacements are returned (for accuracy checks)."""
    rng = np.random.default_rng(seed)
    if each_once:
        if n_requests != len(pool):
            raise ValueError("each_once needs n_requests == len(pool)")
        order = rng.permutation(len(pool))
    else:
        order = rng.integers(0, len(pool), size=n_requests)
    gaps = rng.exponential(1.0 / rate, size=n_requests)
    arrivals = np.cumsum(gaps) - gaps[0]
    models = [_host_model(pool[i]) for i in order]
    srv = Server(device, slots=slots, hbm_budget_bytes=hbm_budget_bytes, opts=opts)
    try:
        # the smallest deck of each element type once per slot: loads the kernels of both
        # element types and builds every slot's workspaces before the timed stream
        def is20(e):
            return e["c3d20"] is not None if isinstance(e, dict) else "C3D20" in e

        def size(e):
            return len(e["node_ids"]) if isinstance(e, dict) else len(e)
        kinds = [[t for t in pool if is20(t) == want] for want in (False, True)]
        smalls = [min(k, key=size) for k in kinds if k]
        warm = [_host_model(t) for t in smalls for _ in range(slots)]
        for t in [srv.submit(w) for w in warm]:
            srv.wait(t, timeout=600.0)
        for w in warm:
            w.close()
        t0 = time.perf_counter()
        tickets = []
        for k in range(n_requests):
            now = time.perf_counter() - t0
            if arrivals[k] > now:
                time.sleep(arrivals[k] - now)
            tickets.append(srv.submit(models[k]))
        outs = [srv.wait(t, timeout=3600.0) for t in tickets]
        t_end = time.perf_counter()
        info = srv.info()
    finally:
        srv.close()
    kept = {}
    recs = []
    for k, (u, r) in enumerate(outs):
        recs.append({"pool": int(order[k]), "status": r["status"], "latency_ms": r["latency_ms"],
                     "queue_ms": r["queue_ms"], "service_ms": r["service_ms"], "device_ms": r["stats"]["t_total_ms"],
                     "setup_ms": r["setup_ms"], "solve_ms": r["solve_ms"], "finish_ms": r["finish_ms"],
                     "dofs": models[k].num_dofs, "pcg_iterations": r["stats"]["pcg_iterations"],
                     "error": r["error"]})
        if keep is not None and int(order[k]) in keep and int(order[k]) not in kept and u is not None:
            kept[int(order[k])] = u
    for m in models:
        m.close()
    lat = np.array([r["latency_ms"] for r in recs if r["status"] == 0])
    ok = int(sum(1 for r in recs if r["status"] == 0))
    span = max(t_end - t0, 1e-9)
    # where the latency goes: p50 / p99 of each part over the completed requests
    parts = {}
    for key in ("queue_ms", "service_ms", "setup_ms", "solve_ms", "device_ms", "finish_ms"):
        v = np.array([r[key] for r in recs if r["status"] == 0])
        if len(v):
            parts[key] = [round(float(np.percentile(v, 50)), 2), round(float(np.percentile(v, 99)), 2)]
    return {"rate_per_s": rate, "requests": n_requests, "completed": ok, "slots": slots,
            "p50_p99_parts_ms": parts, "server": info,
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "mean_ms": float(lat.mean()) if len(lat) else None,
            "solves_per_s": ok / span, "span_s": span,
            "mean_dofs": float(np.mean([r["dofs"] for r in recs])), "records": recs, "kept": kept}
