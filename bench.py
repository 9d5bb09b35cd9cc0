#!/usr/bin/env python
"""Benchmark of the linear-static C3D20 solve (the headline workload); further modes
time batched decks, the serving loop and the NLGEOM beam.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision mixed|fp64|fp64_csr]
                    [--preconditioner amg|bj]

Workload: C3D20 box 20x20x80 mm, 20x20x80 serendipity bricks (32,000 elements,
139,041 nodes, 417,123 DOF), interior nodes jittered U(+-10% h) with a fixed
seed, E=70000 MPa, nu=0.33, z=0 face clamped (*BOUNDARY 1..6), 5000 N in -x
spread over the z=80 face nodes; written as `.inp` text and parsed like any deck.

One step = one StaticStep::solve of that deck to a displacement accurate to
1e-8 against the FP64 direct solution: residual, symbolic pattern (rebuilt every
step), element stiffness + BSR3 assembly, penalty BCs, PCG to the stated
tolerance, update, convergence re-check. The default solver is the FP64 CG with
the aggregation-multigrid preconditioner whose fine-level smoother reads FP32
matrix values (`--precision mixed --preconditioner amg`); the comparison arms
time the other solvers on the same deck, among them the plain FP64 GPU PCG
(scalar CSR + Jacobi, the reference IterativeSolver's algorithm). `value` is solves/s over all ranks with
the model already resident on the device; `e2e` is the same through the public
API from host text and host buffers (parse, upload, solve, download).
With N GPUs each rank solves its own replica (no collective: a single deck is
not sharded); value = N*K / max-over-ranks time.

The oracle (FP64 multifrontal Cholesky restatement of the reference's CPU path)
runs in a separate process on the host cores during the GPU timing; it supplies
the rel. error of the GPU solution and the `cpu_baseline` entry.
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "C3D20 time-to-1e-8 (mixed vs FP64 GPU PCG); solves/s; serving p50/p99 latency"
WORKLOAD = "C3D20 box 20x20x80 cells, 417,123 DOF, linear *STATIC, clamped z=0, 5000 N on z=80, tol 1e-8 vs FP64 direct"


def _deck():
    from ferrix_b200 import decks
    return decks.c3d20_box()


# CUDA-core peaks of a B200 at its maximum SM clock (148 SMs x 1.965 GHz x 2 flop per FMA):
# 128 FP32 lanes and 64 FP64 lanes per SM. Nominal figures (no measured copy in this repo).
CUDA_CORE_TFLOPS = {"fp32": 148 * 128 * 2 * 1.965e9 / 1e12, "fp64": 148 * 64 * 2 * 1.965e9 / 1e12}


def _secondary(bj_ms, bj_bytes, asm, peak_gbs):
    """Roofline entries beside the dominant kernel: the block-Jacobi PCG SpMV and the
    assembly kernels (element stiffness against the nominal CUDA-core peak, the gather
    against the measured copy bandwidth), each timed standalone with CUDA events."""
    out = [{"kernel": "k_pcg_spmv<float> (block-Jacobi PCG SpMV)", "bound": "hbm", "unit": "GB/s",
            "achieved": bj_bytes / (bj_ms * 1e-3) / 1e9, "peak": peak_gbs,
            "frac": bj_bytes / (bj_ms * 1e-3) / 1e9 / peak_gbs, "ms_per_launch": bj_ms,
            "bytes_per_launch": bj_bytes}]
    for prec, (st_ms, flops, ga_ms, ga_bytes) in asm.items():
        t = "double" if prec == "fp64" else "float"
        tf = flops / (st_ms * 1e-3) / 1e12
        out.append({"kernel": f"k_stiff20<{t}> (C3D20 element stiffness, 354,780 declared flop per element)",
                    "bound": prec + " CUDA cores", "unit": "TFLOP/s", "achieved": tf,
                    "peak": CUDA_CORE_TFLOPS[prec], "peak_source": "nominal 148 SM x lanes x 2 x 1.965 GHz",
                    "frac": tf / CUDA_CORE_TFLOPS[prec], "ms_per_launch": st_ms, "flops_per_launch": flops})
        gb = ga_bytes / (ga_ms * 1e-3) / 1e9
        out.append({"kernel": f"k_bsr_gather<{t}> (element-pair blocks into BSR3)", "bound": "hbm",
                    "unit": "GB/s", "achieved": gb, "peak": peak_gbs, "frac": gb / peak_gbs,
                    "ms_per_launch": ga_ms, "bytes_per_launch": ga_bytes})
    return out


def _config(world: int) -> dict:
    """The workload as both arms print it (the solver used is reported beside it)."""
    return {"workload": WORKLOAD, "accuracy": "1e-8 relative displacement error vs the FP64 direct solution",
            "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"}


def _oracle_job(out_path: str, q, go=None) -> None:
    """CPU reference path (oracle restatement): parse, serial assembly, CSR, FP64 Cholesky, Newton check.
    With `go`, it starts when `go` is set (after the GPU measurements, so that neither perturbs the other)."""
    import numpy as np
    from oracle import inp, static_step
    text = _deck()
    if go is not None:
        go.wait()
    t0 = time.perf_counter()
    p = inp.parse_inp_text(text)
    r = static_step.Runner(p)
    st = r.run()
    dt = time.perf_counter() - t0
    np.save(out_path, st.displacements)
    threads = os.environ.get("OPENBLAS_NUM_THREADS")
    q.put({"seconds": dt, "phases": {k: round(v, 3) for k, v in vars(r.t).items()},
           "cores": int(threads) if threads else os.cpu_count(), "host_cores": os.cpu_count(),
           "blas_threads": threads or "all"})


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms. The sampler starts before
    the warm-up steps and stops after all GPU measurements: starting and stopping nvidia-smi
    (NVML initialisation and teardown) stalled the CUDA work beside it by up to ~0.5 s on
    these hosts, which must not fall inside a timed region. mark() delimits the samples
    that the summary covers (those taken during the timed region)."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None
        self.span = None

    def mark(self):
        """Row count now: call at the start and at the end of the timed region."""
        return len(self.rows)

    def summary(self, i0: int, i1: int):
        """Median SM clock and throttle reasons of the samples taken between two marks (the
        neighbouring sample on each side when none fell inside a short region)."""
        self.span = (max(0, i0 - 1), i1 + 1) if i1 <= i0 else (i0, i1)
        return self._summarise(self.rows[self.span[0]:self.span[1]])

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([s.strip() for s in line.split(",")])

    def stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()

    def _summarise(self, rows):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx = float(r[1])
                for k, name in enumerate(names):
                    if r[4 + k].lower().startswith("active"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


BATCH_DECKS = 64


def _batch_figure(ctx, stream):
    """64 C3D4 box decks of the batched workload's population (DOF log-uniform [2k, 60k],
    E log-uniform, random load), built from arrays (fx_model_from_arrays, no text) and
    solved by one fx_batch_solve with the default options: each deck's first step
    (pattern, assembly, multigrid setup, CG to 1e-8, Newton re-check), the decks spread
    over the context's four worker streams. Device time, mean of two timed batches after
    one untimed. Beside it, the same 64 decks submitted at once to the request loop
    (fx_server, 4 slots): its span from the first submission to the last completion."""
    import numpy as np
    import torch
    import ferrix_b200 as fx
    from ferrix_b200 import decks
    pop = decks.batch_population(BATCH_DECKS, seed=7, dof_lo=2e3, dof_hi=6e4, c3d20_fraction=0.0, arrays=True)
    opts = fx.solve_opts()
    times, first = [], None
    for rep in range(3):
        ps = [fx.Project.from_arrays(**dict(kw, default_temperature=20.0), ctx=ctx) for kw, _ in pop]
        for p in ps:
            fx.SolutionState(p.num_dofs, p.num_nodes).initialize(p)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        status, stats = fx.batch_solve(ctx, ps, opts)
        e1.record(stream)
        torch.cuda.synchronize()
        if rep > 0:
            times.append(e0.elapsed_time(e1))
        if first is None:
            first = []
            for p in ps[:2]:
                st = fx.SolutionState(p.num_dofs, p.num_nodes)
                st.project = p
                first.append(st.displacements)
        for p in ps:
            p.close()
    ms = float(np.mean(times))
    from ferrix_b200 import serving
    loop = serving.run_stream([kw for kw, _ in pop], 1e6, BATCH_DECKS, opts, device=torch.cuda.current_device(),
                              slots=4, seed=1, each_once=True)
    return {"decks": BATCH_DECKS, "total_dofs": int(sum(d for _, d in pop)), "device_ms": ms,
            "solves_per_s": BATCH_DECKS / (ms * 1e-3), "failed": int(np.sum(status != 0)),
            "pcg_iterations_max": int(max(s["pcg_iterations"] for s in stats)),
            "solver": "default (mixed multigrid CG, multi-launch per system; four worker streams)",
            "input": "fx_model_from_arrays",
            "request_loop_same_decks": {"slots": 4, "completed": loop["completed"], "span_s": loop["span_s"],
                                        "solves_per_s": loop["completed"] / loop["span_s"]}}, first


def _batch_oracle_errors(first):
    """Relative errors of the first two batch decks against the oracle's FP64 direct solve."""
    import numpy as np
    from ferrix_b200 import decks
    from oracle import inp, static_step
    errs = []
    for (text, _), u in zip(decks.batch_population(2, seed=7, dof_lo=2e3, dof_hi=6e4, c3d20_fraction=0.0), first):
        o = inp.parse_inp_text(text)
        o.default_initial_temperature = 20.0
        ref = static_step.Runner(o).run().displacements
        errs.append(float(np.linalg.norm(u - ref) / np.linalg.norm(ref)))
    return errs


def run_reference(args, rank: int, world: int) -> None:
    """--impl reference: the reference's CPU path (oracle port) on this host's cores, rank 0 only."""
    if rank != 0:
        return
    if args.threads > 0:  # before NumPy loads its BLAS (the oracle's only parallel part)
        for k in ("OPENBLAS_NUM_THREADS", "OMP_NUM_THREADS", "MKL_NUM_THREADS"):
            os.environ[k] = str(args.threads)
    q = mp.get_context("spawn").Queue()
    t0 = time.perf_counter()
    _oracle_job(os.path.join("/tmp", f"u_oracle_ref_{os.getpid()}.npy"), q)
    res = q.get()
    sec = res["seconds"]
    line = {
        "metric": METRIC, "impl": "reference", "value": 1.0 / sec, "unit": "solves/s", "n_gpus": world,
        "steps": 1, "warmup": 0, "requested_steps": args.steps, "requested_warmup": args.warmup,
        "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded deck generator)",
        "config": _config(world),
        "solver": {"name": "FP64 multifrontal Cholesky (oracle port of the reference DirectSolver path)",
                   "precision": "fp64"},
        "cpu_baseline": {"value": 1.0 / sec, "unit": "solves/s", "cores": res["cores"], "kind": "port",
                         "host_cores": res["host_cores"],
                         "sample": "one full-size solve (the step is ~minutes on the CPU, so 1 step regardless of K)",
                         "phases_s": res["phases"]},
        "e2e": {"value": 1.0 / sec, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_once(args, rank: int, local: int) -> None:
    """--mode once: parse the C3D20 box (--cells) and run one step with the default solver options
    and --precision / --preconditioner; prints the step statistics (for profiler runs)."""
    import ferrix_b200 as fx
    from ferrix_b200 import decks
    nx, ny, nz = (int(v) for v in args.cells.split(","))
    prec = {"fp64": fx.PREC_FP64, "mixed": fx.PREC_MIXED, "fp64_csr": fx.PREC_FP64_CSR}[args.precision]
    pc = {"amg": fx.PRECOND_AMG, "bj": fx.PRECOND_BLOCK_JACOBI}[args.preconditioner]
    ctx = fx.Context(local)
    p = fx.Project.from_inp_text(decks.c3d20_box(nx, ny, nz), ctx)
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    st.initialize(p)
    s = p.steps[0].solve(1, p, st, opts=fx.solve_opts(precision=prec, preconditioner=pc))
    print(json.dumps({"mode": "once", "dofs": p.num_dofs, **{k: s[k] for k in (
        "pcg_iterations", "amg_levels", "amg_setup_ms", "t_assembly_ms", "t_pcg_ms", "t_total_ms", "bsr_blocks")}}),
          flush=True)
    p.close()
    ctx.close()


def _serve_summary(res):
    return {k: res[k] for k in ("rate_per_s", "requests", "completed", "slots", "p50_ms", "p99_ms", "mean_ms",
                                "solves_per_s", "mean_dofs", "p50_p99_parts_ms", "server")}


def run_serve(args, rank: int, local: int) -> None:
    """--mode serve: Poisson request streams through the request loop, mixed multigrid vs plain FP64 PCG."""
    if rank != 0:
        return
    import ferrix_b200 as fx
    from ferrix_b200 import serving
    pool = serving.make_pool()
    rates = [float(r) for r in args.rates.split(",")]
    out = {"mode": "serve", "metric": "serving p50/p99 latency (ms) and solves/s at 1e-8",
           "pool": "16 seeded boxes, 60% C3D4 / 40% C3D20, DOF log-uniform [5k, 500k]", "arms": {}}
    arms = (("mixed_amg", fx.solve_opts(precision=fx.PREC_MIXED, preconditioner=fx.PRECOND_AMG), rates),
            ("plain_fp64_csr_jacobi", fx.solve_opts(precision=fx.PREC_FP64_CSR), rates[:2]))
    import numpy as np
    from oracle import inp, static_step
    smallest = [int(i) for i in np.argsort([len(t) for t in pool])[:3]]
    refs = {}
    for name, o, rs in arms:
        out["arms"][name] = []
        for r in rs:
            res = serving.run_stream(pool, r, args.requests, o, device=local, slots=args.slots, seed=int(r),
                                     keep=smallest)
            line = _serve_summary(res)
            # accuracy of served results (the smallest pool decks that were drawn) against the oracle
            errs = {}
            for i, u in res["kept"].items():
                if i not in refs:
                    q = inp.parse_inp_text(pool[i])
                    q.default_initial_temperature = 20.0
                    refs[i] = static_step.Runner(q).run().displacements
                errs[i] = float(np.linalg.norm(u - refs[i]) / np.linalg.norm(refs[i]))
            line["rel_err_vs_oracle"] = errs
            out["arms"][name].append(line)
    print(json.dumps(out), flush=True)


NLGEOM_FULL = (100, 20, 20)  # 240,000 C3D4, 133,623 DOF
NLGEOM_MID = (50, 10, 10)    # 30,000 C3D4, 16,833 DOF: same beam, coarser, for the oracle


def _oracle_nlgeom_job(out_path: str, q, go=None) -> None:
    """The oracle's NLGEOM run of the mid-size beam; with `go`, it starts when `go` is set."""
    import numpy as np
    from ferrix_b200 import decks
    from oracle import inp, static_step
    text = decks.c3d4_nlgeom_beam(*NLGEOM_MID)
    if go is not None:
        go.wait()
    t0 = time.perf_counter()
    p = inp.parse_inp_text(text)
    p.default_initial_temperature = 20.0
    r = static_step.Runner(p)
    st = r.run()
    dt = time.perf_counter() - t0
    np.save(out_path, st.displacements)
    q.put({"seconds": dt, "increments": len(r.log), "newton_iterations": sum(len(l.residuals) - 1 for l in r.log),
           "cores": os.cpu_count(), "phases": {k: round(v, 3) for k, v in vars(r.t).items()}})


def run_nlgeom(args, rank: int, local: int) -> None:
    """--mode nlgeom: the C3D4 NLGEOM beam (E(T), initial temperature gradient, amplitude
    ramp over 10 increments) at full size (240,000 C3D4, 133,623 DOF): whole-step device time
    for three solvers, their agreement with each other; the same beam at 30,000 C3D4 against
    the oracle's FP64 Cholesky Newton run (spawned on the host cores; a full-size oracle run
    takes most of an hour)."""
    if rank != 0:
        return
    import numpy as np
    ctxmp = mp.get_context("spawn")
    q = ctxmp.Queue()
    out_path = os.path.join("/tmp", f"u_oracle_nl_{os.getpid()}.npy")
    proc = None
    go = ctxmp.Event()  # the oracle starts after the GPU timings, so that neither perturbs the other
    if not args.no_oracle:
        proc = ctxmp.Process(target=_oracle_nlgeom_job, args=(out_path, q, go), daemon=True)
        proc.start()
    import torch
    import ferrix_b200 as fx
    from ferrix_b200 import decks
    ctx = fx.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    solvers = (("mixed_amg", fx.solve_opts()),
               ("mixed_blockjacobi", fx.solve_opts(preconditioner=fx.PRECOND_BLOCK_JACOBI)),
               ("fp64_blockjacobi", fx.solve_opts(precision=fx.PREC_FP64, preconditioner=fx.PRECOND_BLOCK_JACOBI)))
    out = {"mode": "nlgeom", "metric": "C3D4 NLGEOM step: device time (ms) and accuracy vs FP64 oracle",
           "full": {}, "mid": {}}
    for size, key, reps in ((NLGEOM_FULL, "full", 2), (NLGEOM_MID, "mid", 1)):
        p = fx.Project.from_inp_text(decks.c3d4_nlgeom_beam(*size), ctx)
        p.default_initial_temperature = 20.0
        st = fx.SolutionState(p.num_dofs, p.num_nodes)
        out[key]["dofs"] = p.num_dofs
        for name, o in solvers:
            best = None
            for _ in range(reps):
                st.initialize(p)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                s = p.steps[0].solve(1, p, st, opts=o)
                e1.record(stream)
                torch.cuda.synchronize()
                ms = e0.elapsed_time(e1)
                best = ms if best is None else min(best, ms)
            out[key][name] = {"ms": best, "increments": s["increments"], "newton_iterations": s["newton_iterations"],
                              "linear_solves": s["linear_solves"], "pcg_iterations": s["pcg_iterations"],
                              "u": st.displacements}
        u64 = out[key]["fp64_blockjacobi"]["u"]
        for name, _ in solvers:
            a = out[key][name]
            a["rel_diff_vs_fp64_blockjacobi"] = float(np.linalg.norm(a["u"] - u64) / np.linalg.norm(u64))
        p.close()
    if proc is not None:
        go.set()
        res = q.get(timeout=7200)
        proc.join(timeout=60)
        u_ref = np.load(out_path)
        for name, _ in solvers:
            a = out["mid"][name]
            a["rel_err_vs_oracle"] = float(np.linalg.norm(a["u"] - u_ref) / np.linalg.norm(u_ref))
        out["mid"]["cpu_oracle"] = {"seconds": res["seconds"], "increments": res["increments"],
                                    "newton_iterations": res["newton_iterations"], "cores": res["cores"],
                                    "phases_s": res["phases"]}
        os.remove(out_path)
    for key in ("full", "mid"):
        for name, _ in solvers:
            out[key][name].pop("u")
    ctx.close()
    print(json.dumps(out), flush=True)


def run_batch(args, rank: int, local: int) -> None:
    """--mode batch: many independent C3D4 decks (DOF log-uniform [2k, 60k]) solved to 1e-8, solves/s.

    Arms: one fx_batch_solve over all decks (mixed block-Jacobi PCG, all systems in
    one launch sequence per iteration block), the same decks one after another, and
    the request loop (4 slots, multigrid) fed with all decks at once. Under torchrun
    the decks are partitioned across the ranks by DOF count (footprint), no
    collective on the data path; solves/s = all decks / max-over-ranks time."""
    import numpy as np
    import torch
    import ferrix_b200 as fx
    from ferrix_b200 import decks, multi
    from oracle import inp, static_step
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    t0 = time.perf_counter()
    pop = decks.batch_population(args.decks, seed=7, dof_lo=2e3, dof_hi=6e4, c3d20_fraction=0.0)
    gen_s = time.perf_counter() - t0
    all_dofs = [d for _, d in pop]
    mine = multi.partition_by_footprint(all_dofs, world)[rank]
    texts = [pop[i][0] for i in mine]
    dofs = np.array([pop[i][1] for i in mine])
    ctx = fx.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    out = {"mode": "batch", "metric": "batched linear static solves/s (C3D4 decks, mixed precision, 1e-8)",
           "decks": len(pop), "n_gpus": world, "total_dofs": int(np.sum(all_dofs)),
           "mean_dofs": float(np.mean(all_dofs)), "deck_generation_s": gen_s, "arms": {}}

    def projects():
        ps = [fx.Project.from_inp_text(t, ctx) for t in texts]
        for p in ps:
            p.default_initial_temperature = 20.0
            fx.SolutionState(p.num_dofs, p.num_nodes).initialize(p)
        return ps

    def timed(fn):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        w0 = time.perf_counter()
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1) / 1e3, time.perf_counter() - w0

    o_bj = fx.solve_opts(precision=fx.PREC_MIXED, rtol=1e-8, preconditioner=fx.PRECOND_BLOCK_JACOBI)
    for rep in range(2):  # the first pass also loads kernels and builds graphs
        ps = projects()
        (st, stats), dev_s, wall_s = timed(lambda: fx.batch_solve(ctx, ps, o_bj))
        us = [fx.SolutionState(p.num_dofs, p.num_nodes) for p in ps]
        u_batch = []
        for p, s in zip(ps, us):
            s.project = p
            u_batch.append(s.displacements)
        for p in ps:
            p.close()
    dev_max = multi.max_over_ranks(dev_s, device="cuda")
    out["arms"]["fx_batch_solve_mixed_bj"] = {"solves_per_s": len(pop) / dev_max, "device_s": dev_max,
                                              "wall_s": wall_s,
                                              "failed": int(multi.sum_over_ranks(float(np.sum(st != 0)), "cuda")),
                                              "pcg_iterations_max": int(max(s["pcg_iterations"] for s in stats))}
    o_amg = fx.solve_opts(rtol=1e-8)  # default: mixed multigrid, the decks spread over four worker streams
    for rep in range(2):
        ps = projects()
        (st_a, _), dev_s, wall_s = timed(lambda: fx.batch_solve(ctx, ps, o_amg))
        for p in ps:
            p.close()
    dev_max = multi.max_over_ranks(dev_s, device="cuda")
    out["arms"]["fx_batch_solve_mixed_amg"] = {"solves_per_s": len(pop) / dev_max, "device_s": dev_max,
                                               "wall_s": wall_s,
                                               "failed": int(multi.sum_over_ranks(float(np.sum(st_a != 0)), "cuda"))}
    ps = projects()

    def seq():
        bad = 0
        for p in ps:
            try:
                p.steps[0].solve(1, p, fx.SolutionState(p.num_dofs, p.num_nodes), opts=o_bj)
            except fx.FerrixError:
                bad += 1
        return bad
    bad, dev_s, wall_s = timed(seq)
    for p in ps:
        p.close()
    dev_max = multi.max_over_ranks(dev_s, device="cuda")
    out["arms"]["sequential_mixed_bj"] = {"solves_per_s": len(pop) / dev_max, "device_s": dev_max, "wall_s": wall_s,
                                          "failed": int(multi.sum_over_ranks(float(bad), "cuda"))}
    ctx.close()
    from ferrix_b200 import serving
    res = serving.run_stream(texts, 1e6, len(texts), fx.solve_opts(precision=fx.PREC_MIXED,
                                                                  preconditioner=fx.PRECOND_AMG, rtol=1e-8),
                             device=local, slots=4, seed=1, each_once=True)
    span = multi.max_over_ranks(res["span_s"], device="cuda")
    out["arms"]["request_loop_mixed_amg_4_slots"] = {"solves_per_s": len(pop) / span, "wall_s": span,
                                                     "failed": int(multi.sum_over_ranks(
                                                         float(len(texts) - res["completed"]), "cuda"))}
    # accuracy of the batched result on the first decks against the oracle's direct solve
    errs = []
    for k in range(min(4, len(texts))):
        o = inp.parse_inp_text(texts[k])
        o.default_initial_temperature = 20.0
        ref = static_step.Runner(o).run().displacements
        errs.append(float(np.linalg.norm(u_batch[k] - ref) / np.linalg.norm(ref)))
    out["rel_err_vs_oracle_first4"] = errs
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "fp64_csr"])
    ap.add_argument("--preconditioner", default="amg", choices=["amg", "bj"])
    ap.add_argument("--no-oracle", action="store_true", help="skip the CPU oracle (accuracy / cpu_baseline)")
    ap.add_argument("--no-arms", action="store_true", help="skip the comparison arms")
    ap.add_argument("--rates", default="10,25,50,100,500", help="serve mode: arrival rates (requests/s)")
    ap.add_argument("--requests", type=int, default=48, help="serve mode: requests per rate")
    ap.add_argument("--slots", type=int, default=4, help="serve mode: concurrent requests on the GPU")
    ap.add_argument("--decks", type=int, default=256, help="batch mode: number of decks")
    ap.add_argument("--cells", default="20,20,80", help="once mode: C3D20 box cells nx,ny,nz")
    ap.add_argument("--mode", default="solve", choices=["solve", "spmv", "serve", "batch", "nlgeom", "once"],
                    help="spmv: only assemble and time REPS standalone SpMV launches (profiling case)")
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--threads", type=int, default=0,
                    help="reference arm: BLAS threads of the CPU path (0 = all host cores; FerriX's default pool is 4)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.mode == "once":
        return run_once(args, rank, local)
    if args.mode == "serve":
        return run_serve(args, rank, local)
    if args.mode == "batch":
        return run_batch(args, rank, local)
    if args.mode == "nlgeom":
        return run_nlgeom(args, rank, local)
    if args.mode == "spmv":
        import ferrix_b200 as fx
        ctx = fx.Context(local)
        p = fx.Project.from_inp_text(_deck(), ctx)
        st = fx.SolutionState(p.num_dofs, p.num_nodes)
        st.initialize(p)
        prec = {"fp64": fx.PREC_FP64, "mixed": fx.PREC_MIXED, "fp64_csr": fx.PREC_FP64}[args.precision]
        ms, by = p.profile_spmv(prec, args.reps)
        print(json.dumps({"mode": "spmv", "precision": args.precision, "ms_per_launch": ms, "bytes": by,
                          "GBps": by / ms / 1e6}), flush=True)
        p.close()
        ctx.close()
        return

    # the oracle process starts before any CUDA initialisation (spawn)
    oracle_q = oracle_p = None
    oracle_out = os.path.join("/tmp", f"u_oracle_{os.getpid()}.npy")
    if rank == 0 and not args.no_oracle:
        ctxmp = mp.get_context("spawn")
        oracle_q = ctxmp.Queue()
        oracle_go = ctxmp.Event()
        oracle_p = ctxmp.Process(target=_oracle_job, args=(oracle_out, oracle_q, oracle_go), daemon=True)
        oracle_p.start()

    import numpy as np
    import torch
    import ferrix_b200 as fx

    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    prec = {"fp64": fx.PREC_FP64, "mixed": fx.PREC_MIXED, "fp64_csr": fx.PREC_FP64_CSR}[args.precision]
    pc = {"amg": fx.PRECOND_AMG, "bj": fx.PRECOND_BLOCK_JACOBI}[args.preconditioner]
    use_amg = pc == fx.PRECOND_AMG and prec != fx.PREC_FP64_CSR
    opts = fx.solve_opts(precision=prec, rtol=1e-8, preconditioner=pc)
    text = _deck()
    ctx = fx.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream)
    project = fx.Project.from_inp_text(text, ctx)
    state = fx.SolutionState(project.num_dofs, project.num_nodes)

    def one_step():
        state.initialize(project)
        project.drop_cache()
        return project.steps[0].solve(1, project, state, opts=opts)

    clocks = ClockSampler(local)
    clocks.start()  # before the warm-up: nvidia-smi's start-up stall lands there
    for _ in range(max(3, args.warmup)):
        one_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = ctx.kernel_launches
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    mark0 = clocks.mark()
    ev0.record(stream)
    stats = []
    for _ in range(args.steps):
        stats.append(one_step())
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.summary(mark0, clocks.mark())
    elapsed = ev0.elapsed_time(ev1) / 1e3
    launches = ctx.kernel_launches - launches0
    u_gpu = state.displacements
    if dist:
        from ferrix_b200 import multi
        elapsed = multi.max_over_ranks(elapsed, device="cuda")
        dist.barrier()

    # dominant kernel, timed standalone with CUDA events on the context stream:
    # the fused fine-level smoothing step (multigrid) or the fused PCG SpMV
    if use_amg:  # with mixed precision the default smoother reads FP16 values of the scaled matrix
        spmv_ms, spmv_bytes = project.profile_smoother(prec, 30, fp16=prec == fx.PREC_MIXED)
    else:
        spmv_ms, spmv_bytes = project.profile_spmv(prec if prec != fx.PREC_FP64_CSR else fx.PREC_FP64, 30)
    bj_ms, bj_bytes = project.profile_spmv(fx.PREC_MIXED, 30)
    asm = {name: project.profile_assembly(pr, 10) for name, pr in (("fp64", fx.PREC_FP64), ("fp32", fx.PREC_MIXED))}

    arms = {}
    if rank == 0 and not args.no_arms:
        arm_list = (("plain_fp64_csr_jacobi", fx.PREC_FP64_CSR, fx.PRECOND_BLOCK_JACOBI),
                    ("fp64_bsr_blockjacobi", fx.PREC_FP64, fx.PRECOND_BLOCK_JACOBI),
                    ("mixed_bsr_blockjacobi", fx.PREC_MIXED, fx.PRECOND_BLOCK_JACOBI),
                    ("fp64_amg", fx.PREC_FP64, fx.PRECOND_AMG),
                    ("mixed_amg", fx.PREC_MIXED, fx.PRECOND_AMG))
        for name, pr, pcn in arm_list:
            if pr == prec and (pcn == pc or pr == fx.PREC_FP64_CSR):
                arms[name] = {"ms": elapsed / args.steps * 1e3, "pcg_iterations": stats[-1]["pcg_iterations"],
                              "u": u_gpu, "headline": True}
                continue
            o2 = fx.solve_opts(precision=pr, rtol=1e-8, preconditioner=pcn)
            try:
                best = None
                for _ in range(2):  # the first run also instantiates this solver's graphs
                    state.initialize(project)
                    project.drop_cache()
                    torch.cuda.synchronize()
                    a0 = torch.cuda.Event(enable_timing=True)
                    a1 = torch.cuda.Event(enable_timing=True)
                    a0.record(stream)
                    st = project.steps[0].solve(1, project, state, opts=o2)
                    a1.record(stream)
                    torch.cuda.synchronize()
                    ms = a0.elapsed_time(a1)
                    best = ms if best is None else min(best, ms)
                arms[name] = {"ms": best, "pcg_iterations": st["pcg_iterations"],
                              "fp64_fallbacks": st["fp64_fallbacks"], "u": state.displacements}
            except fx.FerrixError as e:
                arms[name] = {"error": str(e)}

    # e2e through the public API from the deck's bytes in host memory (what a caller of
    # fx_model_from_inp passes; a file read by Project.from_jobname arrives the same way)
    # to displacements in host memory (the oracle has not started yet)
    h2d = d2h = 0
    e2e_elapsed = None
    deck_bytes = text.encode()
    if rank == 0 or True:
        def e2e_step():
            p = fx.Project.from_inp_text(deck_bytes, ctx)
            s = fx.SolutionState(p.num_dofs, p.num_nodes)
            s.initialize(p)
            p.steps[0].solve(1, p, s, opts=opts)
            u = s.displacements
            p.close()
            return u
        e2e_step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ke = max(1, args.steps)  # as many steps as the device-resident timing
        e2e_steps = []  # host wall time of each step (each ends with the D2H read of u)
        for _ in range(ke):
            h0 = time.perf_counter()
            e2e_step()
            e2e_steps.append((time.perf_counter() - h0) * 1e3)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_elapsed = e0.elapsed_time(e1) / 1e3 / ke
        xyz, groups = project.export()
        n_el = sum(len(g[1]) for g in groups.values())
        h2d = (xyz.size * 8 + sum(g[0].size * 4 + g[1].size * 4 for g in groups.values())
               + 2 * project.num_nodes * 8)
        d2h = project.num_dofs * 8

    batch_line = batch_first = None
    if rank == 0 and not args.no_arms:
        batch_line, batch_first = _batch_figure(ctx, stream)

    serving_line = None
    if rank == 0 and not args.no_arms:
        from ferrix_b200 import serving
        pool = serving.make_pool(arrays=True)  # the same 16 models as the deck pool, built from arrays
        res = serving.run_stream(pool, 25.0, 32, fx.solve_opts(precision=fx.PREC_MIXED, preconditioner=fx.PRECOND_AMG),
                                 device=local, slots=4, seed=25)
        serving_line = _serve_summary(res)
        serving_line["solver"] = "mixed multigrid CG"
        serving_line["pool"] = "16 seeded boxes, 60% C3D4 / 40% C3D20, DOF log-uniform [5k, 500k]"
        serving_line["input"] = "fx_model_from_arrays"
    clocks.stop()  # after every GPU measurement (its teardown must not overlap one)

    cpu = None
    rel_err = None
    if oracle_p is not None:  # the CPU oracle runs now, after every GPU measurement
        oracle_go.set()
        res = oracle_q.get(timeout=3600)
        oracle_p.join(timeout=60)
        u_ref = np.load(oracle_out)
        rel_err = float(np.linalg.norm(u_gpu - u_ref) / np.linalg.norm(u_ref))
        for a in arms.values():
            if "u" in a:
                a["rel_err_vs_oracle"] = float(np.linalg.norm(a["u"] - u_ref) / np.linalg.norm(u_ref))
        cpu = {"value": 1.0 / res["seconds"], "unit": "solves/s", "cores": res["cores"], "kind": "port",
               "sample": "one full-size solve of the same deck (parse, serial assembly, CSR, FP64 multifrontal "
                         "Cholesky, Newton re-check), in a spawned process after the GPU measurements",
               "phases_s": res["phases"]}
        try:
            os.remove(oracle_out)
        except OSError:
            pass
    for a in arms.values():
        a.pop("u", None)
    if batch_line is not None and oracle_p is not None:
        batch_line["rel_err_vs_oracle_first2"] = _batch_oracle_errors(batch_first)

    if rank == 0:
        import json as _j
        peaks = {}
        try:
            peaks = _j.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        peak = peaks.get("hbm_gbs", 6650.0)
        achieved = spmv_bytes / (spmv_ms * 1e-3) / 1e9
        traffic = None  # DRAM read+write per launch from the committed ncu capture of the same kernel / workload
        prof_name = "k_l0_op_c3d20_box.md" if use_amg else "k_pcg_spmv_c3d20_box.md"
        try:
            import re
            prof = open(os.path.join(ROOT, "profiles", prof_name)).read()
            if use_amg:  # one row per smoother variant: traffic_bytes_per_launch_<fp16|fp64> | N
                variant = "fp16" if prec == fx.PREC_MIXED else args.precision
                m = re.search(r"traffic_bytes_per_launch_%s[^|]*\|\s*([\d,]+)" % variant, prof)
                if m:
                    traffic = int(m.group(1).replace(",", ""))
            else:
                m = re.search(r"traffic_bytes_per_launch[^|]*\|\s*([\d,]+)\s*\|\s*([\d,]+)", prof)
                if m:
                    traffic = int((m.group(2) if prec == fx.PREC_MIXED else m.group(1)).replace(",", ""))
        except OSError:
            pass
        plain = arms.get("plain_fp64_csr_jacobi", {}).get("ms")
        fp64_same = arms.get("fp64_amg" if use_amg else "fp64_bsr_blockjacobi", {}).get("ms")
        s0 = stats[-1]
        line = {
            "metric": METRIC, "value": world * args.steps / elapsed, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(3, args.warmup), "ms_per_step": elapsed / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "mixed": ("f64 CG, f16 scaled smoother matrix" if use_amg else
                                               "f32 matrix / f64 residual"), "fp64_csr": "f64"}[args.precision],
            "data": "synthetic (seeded .inp deck generator; inputs exceed L2: BSR3 FP64 matrix ~600 MB)",
            "config": _config(world),
            "solver": {"name": ("CG + aggregation multigrid V-cycle (Chebyshev-2 smoothing), BSR3" if use_amg else
                                "PCG + 3x3 block-Jacobi, BSR3"), "precision": args.precision, "rtol_M": 1e-8},
            "time_to_1e8_ms": elapsed / args.steps * 1e3,
            "speedup_vs_plain_fp64_gpu_pcg": (plain / (elapsed / args.steps * 1e3)) if plain else None,
            "speedup_vs_fp64_same_preconditioner": (fp64_same / (elapsed / args.steps * 1e3)) if fp64_same else None,
            "rel_err_vs_oracle": rel_err,
            "pcg_iterations": s0["pcg_iterations"],
            "phase_ms": {k: round(s0[k], 3) for k in ("t_assembly_ms", "t_pcg_ms", "t_total_ms")},
            "arms": arms,
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": ("k_l0_op<__half, ChebK> (fused fine-level SpMV + Chebyshev update, "
                                                    "FP16 values of the scaled matrix)" if use_amg and
                                                    prec == fx.PREC_MIXED else
                                                    "k_l0_op<double, ChebK> (fused fine-level SpMV + Chebyshev update)"
                                                    if use_amg else
                                                    "k_pcg_spmv (fused BSR3 SpMV + direction update + p.q)"),
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else
                         "fallback 6650 GB/s", "bytes_per_launch": spmv_bytes, "ms_per_launch": spmv_ms,
                         "traffic": traffic, "traffic_source": f"profiles/{prof_name} (ncu)",
                         "secondary": _secondary(bj_ms, bj_bytes, asm, peak)},
            "clocks": clk,
            "e2e": {"value": 1.0 / e2e_elapsed if e2e_elapsed else None, "unit": "solves/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "ms_per_step": e2e_elapsed * 1e3 if e2e_elapsed else None,
                    # the spread shows a stall of the shared host (one slow step) apart from a slow path
                    "step_ms": {"median": round(statistics.median(e2e_steps), 2),
                                "min": round(min(e2e_steps), 2), "max": round(max(e2e_steps), 2)}
                    if e2e_elapsed else None},
            "cpu_baseline": cpu,
            "batch": batch_line,
            "serving": serving_line,
        }
        print(json.dumps(line), flush=True)
    project.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
