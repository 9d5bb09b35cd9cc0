"""GPU parity: every result of libferrix_b200.so (through the C ABI) against the
oracle's FP64 restatement of the FerriX path on the same inputs.

Tolerances (relative, stated per check):
  * FP64 stiffness entries / maxdiag: 1e-12 of the largest entry
  * FP32 stiffness entries: 2e-6 of the largest entry (FP32 element kernels)
  * FP64 internal / thermal force: 1e-11 of the largest entry
  * displacement, 2-norm, against the oracle's FP64 direct solution: 1e-10 for
    the FP64 solvers (FX_PREC_FP64, FX_PREC_FP64_CSR), 1e-8 for the mixed ones
    (FX_PREC_MIXED), at the default rtol = 1e-8
  * NLGEOM displacement: 1e-8 in the 2-norm (each increment's Newton iterations
    follow the oracle's, the last one's update carries the linear-solve error)
"""
import ctypes as C
import gzip
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

import ferrix_b200 as fx
from ferrix_b200 import decks
from oracle import elem, inp, static_step

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = fx.Context(0)
    yield c
    c.close()


def _deck(golden_dir, name):
    with gzip.open(os.path.join(golden_dir, "decks", name + ".inp.gz"), "rt") as fh:
        return fh.read()


def _project(ctx, text, t_default=20.0):
    p = fx.Project.from_inp_text(text, ctx)
    p.default_initial_temperature = t_default
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    st.initialize(p)
    return p, st


def _oracle(text, t_default=20.0):
    o = inp.parse_inp_text(text)
    o.default_initial_temperature = t_default
    return o, inp.model_arrays(o)


def _csr(p, u, prec):
    ip, ind, dat, md = p.assemble_csr(u, prec)
    return sp.csr_matrix((dat, ind, ip), shape=(p.num_dofs, p.num_dofs)), md


TOL_FP64 = 1e-10   # plain / block FP64 PCG and FP64 multigrid CG
TOL_MIXED = 1e-8   # FP32 SpMV / smoother inside FP64 refinement
TOL_NLGEOM = 1e-8


def _tol(prec):
    return TOL_MIXED if prec == fx.PREC_MIXED else TOL_FP64


def _err(u, ref):
    return float(np.linalg.norm(u - ref) / np.linalg.norm(ref))


SMALL = {
    "one_c3d4": lambda: decks.c3d4_cantilever(1, 1, 1),
    "one_c3d20": lambda: decks.c3d20_box(1, 1, 1),
    "c3d4_box": lambda: decks.c3d4_cantilever(3, 4, 5),
    "c3d20_box": lambda: decks.c3d20_box(2, 3, 4),
    "tdep_beam": lambda: decks.c3d4_nlgeom_beam(6, 2, 2),
}


@pytest.mark.parametrize("case", list(SMALL))
@pytest.mark.parametrize("with_u", [False, True])
def test_stiffness_matches_oracle(ctx, case, with_u):
    text = SMALL[case]()
    p, st = _project(ctx, text)
    o, m = _oracle(text)
    t = inp.initial_temperatures(o)
    u = np.random.default_rng(1).normal(scale=1e-2, size=p.num_dofs) if with_u else None
    K_or, md_or = elem.assemble(m, u, t)
    scale = abs(K_or).max()
    for prec, tol in ((fx.PREC_FP64, 1e-12), (fx.PREC_MIXED, 2e-6)):
        K, md = _csr(p, u, prec)
        assert abs(K - K_or).max() <= tol * scale, (case, prec)
        assert abs(md - md_or) <= tol * md_or


@pytest.mark.parametrize("case", list(SMALL))
def test_internal_and_thermal_force_match_oracle(ctx, case):
    text = SMALL[case]()
    p, st = _project(ctx, text)
    o, m = _oracle(text)
    rng = np.random.default_rng(2)
    t0 = inp.initial_temperatures(o)
    t1 = t0 + rng.uniform(0, 150, size=t0.shape)   # T_cur != T_init exercises eps_th
    st.set_temperatures(t0, t1)
    u = rng.normal(scale=1e-2, size=p.num_dofs)
    for uconf in (None, u):
        f = p.internal_force(u, uconf)
        f_or = elem.internal_force(m, u, uconf, t0, t1)
        assert np.abs(f - f_or).max() <= 1e-11 * np.abs(f_or).max()
    fth = p.thermal_force()
    fth_or = elem.thermal_force(m, t0, t1)
    if np.abs(fth_or).max() > 0:
        assert np.abs(fth - fth_or).max() <= 1e-11 * np.abs(fth_or).max()
    else:
        assert np.abs(fth).max() == 0.0


@pytest.mark.parametrize("name", ["C3D4_staticstep", "C3D4_2staticstep", "C3D20", "NLGEOM_test"])
@pytest.mark.parametrize("prec", [fx.PREC_MIXED, fx.PREC_FP64])
@pytest.mark.parametrize("pc", [fx.PRECOND_BLOCK_JACOBI, fx.PRECOND_AMG])
def test_reference_decks(ctx, golden_dir, name, prec, pc):
    gold = json.load(open(os.path.join(golden_dir, "calculix.json")))[name]
    fix = np.load(os.path.join(golden_dir, f"oracle_{name}.npz"))
    p, st = _project(ctx, _deck(golden_dir, name))
    idx = p.mesh.get_index_for_node_id(gold["node"])
    tol = TOL_NLGEOM if name.startswith("NLGEOM") else _tol(prec)
    for k, want in enumerate(gold["steps"]):
        stats = p.steps[k].solve(k + 1, p, st, opts=fx.solve_opts(precision=prec, preconditioner=pc))
        u = st.displacements
        ref = fix[f"step{k + 1}"]
        err = np.linalg.norm(u - ref) / np.linalg.norm(ref)
        assert err <= tol, (name, k, err, stats)
        assert np.all(np.abs(u[3 * idx:3 * idx + 3] - np.array(want)) < gold["tol"])


def _oracle_run(text, t_default=20.0):
    o = inp.parse_inp_text(text)
    o.default_initial_temperature = t_default
    r = static_step.Runner(o)
    s = r.run()
    return s.displacements, r


@pytest.mark.parametrize("prec", [fx.PREC_MIXED, fx.PREC_FP64])
@pytest.mark.parametrize("pc", [fx.PRECOND_BLOCK_JACOBI, fx.PRECOND_AMG])
def test_c3d4_cantilever_full_size(ctx, prec, pc):
    text = decks.c3d4_cantilever()   # 24,000 C3D4, 14,883 DOF
    ref, _ = _oracle_run(text)
    p, st = _project(ctx, text)
    stats = p.steps[0].solve(1, p, st, opts=fx.solve_opts(precision=prec, preconditioner=pc))
    err = _err(st.displacements, ref)
    assert err <= _tol(prec), (err, stats)


@pytest.mark.parametrize("prec", [fx.PREC_MIXED, fx.PREC_FP64])
@pytest.mark.parametrize("pc", [fx.PRECOND_BLOCK_JACOBI, fx.PRECOND_AMG])
def test_c3d20_jittered_box(ctx, prec, pc):
    text = decks.c3d20_box(4, 4, 16, lengths=(20.0, 20.0, 80.0))
    ref, _ = _oracle_run(text)
    p, st = _project(ctx, text)
    stats = p.steps[0].solve(1, p, st, opts=fx.solve_opts(precision=prec, preconditioner=pc))
    err = _err(st.displacements, ref)
    assert err <= _tol(prec), (err, stats)


def test_nlgeom_thermal_beam(ctx):
    # E(T) table, initial temperature gradient, *AMPLITUDE ramp, 4 increments, NLGEOM
    text = decks.c3d4_nlgeom_beam(12, 3, 3, tip_load=2.0e3, increments=4)
    ref, r = _oracle_run(text)
    p, st = _project(ctx, text)
    for pc in (fx.PRECOND_BLOCK_JACOBI, fx.PRECOND_AMG):
        st.initialize(p)
        stats = p.steps[0].solve(1, p, st, opts=fx.solve_opts(precision=fx.PREC_MIXED, preconditioner=pc))
        assert stats["increments"] == sum(1 for l in r.log)
        err = _err(st.displacements, ref)
        assert err <= TOL_NLGEOM, (pc, err, stats)


@pytest.mark.parametrize("pc", [fx.PRECOND_BLOCK_JACOBI, fx.PRECOND_AMG])
def test_batch_matches_single(ctx, pc):
    """A system's arithmetic does not depend on the others in its batch: alone and batched on
    the same path (multigrid: the persistent cluster launch, threshold set for both) it gives
    the same bits. (With the default options a multigrid system above 2,000 DOF takes the
    multi-launch path alone and batched; test_batch_default_options checks that case.)"""
    pop = decks.batch_population(6, seed=11, dof_lo=500, dof_hi=6000, c3d20_fraction=0.3)
    o = fx.solve_opts(preconditioner=pc, precision=fx.PREC_MIXED,
                      amg_persistent_max_dof=100000 if pc == fx.PRECOND_AMG else 0)
    singles = []
    for text, _ in pop:
        p, st = _project(ctx, text)
        p.steps[0].solve(1, p, st, opts=o)
        singles.append(st.displacements)
    projs = [_project(ctx, text)[0] for text, _ in pop]
    status, stats = fx.batch_solve(ctx, projs, o)
    assert np.all(status == 0)
    for p, u1, (text, _) in zip(projs, singles, pop):
        st = fx.SolutionState(p.num_dofs, p.num_nodes)
        st.project = p
        u = st.displacements
        assert np.array_equal(u, u1)  # same per-system arithmetic alone and in the batch
        ref, _ = _oracle_run(text)
        err = _err(u, ref)
        assert err <= TOL_MIXED, err


def test_batch_default_options(ctx):
    """Default options: the batch's multigrid systems (3k-20k DOF) take the multi-launch path on
    the context's worker streams, as each does alone, so batched and alone give the same bits;
    both meet the mixed bound against the oracle."""
    pop = decks.batch_population(4, seed=13, dof_lo=3000, dof_hi=20000, c3d20_fraction=0.5)
    projs = [_project(ctx, text)[0] for text, _ in pop]
    status, stats = fx.batch_solve(ctx, projs, fx.solve_opts())
    assert np.all(status == 0)
    for p, (text, _) in zip(projs, pop):
        st = fx.SolutionState(p.num_dofs, p.num_nodes)
        st.project = p
        ub = st.displacements
        q, sq = _project(ctx, text)
        q.steps[0].solve(1, q, sq)
        assert np.array_equal(ub, sq.displacements)
        ref, _ = _oracle_run(text)
        for u in (ub, sq.displacements):
            err = _err(u, ref)
            assert err <= TOL_MIXED, err


def test_solve_csr_seam(ctx):
    text = decks.c3d4_cantilever(4, 4, 12)
    o = inp.parse_inp_text(text)
    r = static_step.Runner(o)
    r.run()
    K, R, du = r.last_K.tocsr(), r.last_R, r.last_du
    K.sort_indices()
    ip = K.indptr.astype(np.int64)
    ind = K.indices.astype(np.int64)
    lib = fx._lib.load()
    # DirectSolver stand-ins (relative stop at the library's rtol): block-Jacobi in both precisions and
    # the scalar-CSR FP64 PCG; IterativeSolver (reference_iterative: absolute sqrt(r.z) < tol, max_iter)
    for prec, ref_it, tol in ((fx.PREC_MIXED, 0, TOL_MIXED), (fx.PREC_FP64, 0, TOL_FP64),
                              (fx.PREC_FP64_CSR, 0, TOL_FP64)):
        x = np.empty_like(R)
        st = fx.StepStats()
        o_ = fx.solve_opts(precision=prec, reference_iterative=bool(ref_it))
        rc = lib.fx_solve_csr(ctx.handle, K.shape[0], fx._p(ip), fx._p(ind), fx._p(K.data), fx._p(R), fx._p(x),
                              C.byref(o_), C.byref(st))
        assert rc == 0, lib.fx_ctx_last_error(ctx.handle)
        err = _err(x, du)
        assert err <= tol, (prec, err)
    # the reference IterativeSolver's own semantics against the oracle's restatement of it
    x_or = static_step.jacobi_pcg(K, R, tol=1e-8, max_iter=1000)
    x = np.empty_like(R)
    o_ = fx.solve_opts(precision=fx.PREC_FP64_CSR, reference_iterative=True, rtol=1e-8, max_iter=1000)
    rc = lib.fx_solve_csr(ctx.handle, K.shape[0], fx._p(ip), fx._p(ind), fx._p(K.data), fx._p(R), fx._p(x),
                          C.byref(o_), None)
    assert rc == 0, lib.fx_ctx_last_error(ctx.handle)
    err = _err(x, x_or)
    assert err <= TOL_FP64, err
    # and its iteration cap: ConvergenceError with the reference's message
    o_ = fx.solve_opts(precision=fx.PREC_FP64_CSR, reference_iterative=True, rtol=1e-30, max_iter=5)
    rc = lib.fx_solve_csr(ctx.handle, K.shape[0], fx._p(ip), fx._p(ind), fx._p(K.data), fx._p(R), fx._p(x),
                          C.byref(o_), None)
    assert rc == 12 and b"did not converge after 5 iterations" in lib.fx_ctx_last_error(ctx.handle)


@pytest.mark.parametrize("prec", [fx.PREC_FP64_CSR])
def test_plain_fp64_csr_jacobi(ctx, prec):
    text = decks.c3d20_box(2, 2, 6)
    ref, _ = _oracle_run(text)
    p, st = _project(ctx, text)
    stats = p.steps[0].solve(1, p, st, opts=fx.solve_opts(precision=prec))
    err = _err(st.displacements, ref)
    assert err <= TOL_FP64, (err, stats)


def test_iterative_solver_reference_semantics(ctx, golden_dir):
    # *STATIC, SOLVER=ITERATIVE SCALING: Jacobi PCG with absolute sqrt(r.z) < 1e-8 and 1000 iterations
    text = decks.c3d4_cantilever(2, 2, 3).replace("*Static, Solver=Spooles", "*Static, Solver=Iterative scaling")
    ref, r = _oracle_run(text)
    p, st = _project(ctx, text)
    assert p.steps[0].info.solver == "ITERATIVE"
    p.steps[0].solve(1, p, st, opts=fx.solve_opts(reference_iterative=True))
    # the oracle runs the same Jacobi PCG with the same absolute stop (iterative.rs:26-136), in FP64
    err = _err(st.displacements, ref)
    assert err <= TOL_FP64, err
    # the reference's 1000-iteration cap surfaces as ConvergenceError (the oracle raises it too on this deck)
    hard = _deck(golden_dir, "C3D20").replace("*Static, Solver=Spooles", "*Static, Solver=Iterative scaling")
    p, st = _project(ctx, hard)
    with pytest.raises(fx.FerrixError) as e:
        p.steps[0].solve(1, p, st, opts=fx.solve_opts(reference_iterative=True))
    assert e.value.kind == "ConvergenceError"


@pytest.mark.parametrize("case", ["one_c3d4", "one_c3d20", "c3d4_box"])
@pytest.mark.parametrize("pc", [fx.PRECOND_BLOCK_JACOBI, fx.PRECOND_AMG])
def test_tiny_decks_solve(ctx, case, pc):
    """Single-element and few-element decks through the default solver and block-Jacobi (the
    multigrid hierarchy degenerates to one aggregate, i.e. a direct solve on the rigid-body modes)."""
    text = SMALL[case]()
    ref, _ = _oracle_run(text)
    p, st = _project(ctx, text)
    p.steps[0].solve(1, p, st, opts=fx.solve_opts(preconditioner=pc, precision=fx.PREC_FP64))
    err = _err(st.displacements, ref)
    assert err <= TOL_FP64, err


AMG_CASES = {
    "c3d4_cantilever": lambda: decks.c3d4_cantilever(),
    "c3d20_box": lambda: decks.c3d20_box(4, 4, 16, lengths=(20.0, 20.0, 80.0)),
    "small_c3d20": lambda: decks.c3d20_box(2, 2, 3),
    "c3d20_box_3_levels": lambda: decks.c3d20_box(8, 8, 32),
}


@pytest.mark.parametrize("case", list(AMG_CASES))
@pytest.mark.parametrize("prec", [fx.PREC_FP64, fx.PREC_MIXED])
def test_amg_preconditioned_solve(ctx, case, prec):
    """Multigrid-preconditioned CG (FP64 outer iteration; with PREC_MIXED the
    fine-level smoother reads FP32 values) against the oracle's direct solve."""
    text = AMG_CASES[case]()
    ref, _ = _oracle_run(text)
    p, st = _project(ctx, text)
    stats = p.steps[0].solve(1, p, st, opts=fx.solve_opts(preconditioner=fx.PRECOND_AMG, precision=prec))
    assert stats["amg_levels"] >= (3 if case.endswith("3_levels") else 2)
    err = _err(st.displacements, ref)
    assert err <= _tol(prec), (err, stats)


@pytest.mark.parametrize("degree,cycle,kind", [(1, 0, 0), (3, 0, 0), (2, 1, 0), (1, 1, 0), (2, 0, 1), (3, 1, 1)])
def test_amg_smoother_degree_and_cycle(ctx, degree, cycle, kind):
    """Chebyshev degree and kind, V- / K-cycle (flexible outer CG) variants against the oracle."""
    text = AMG_CASES["c3d20_box_3_levels"]()
    ref, _ = _oracle_run(text)
    p, st = _project(ctx, text)
    opts = fx.solve_opts(preconditioner=fx.PRECOND_AMG, amg_smoother_degree=degree, amg_aggregate_nodes=60,
                         amg_cycle=cycle, amg_smoother=kind)
    stats = p.steps[0].solve(1, p, st, opts=opts)
    err = _err(st.displacements, ref)
    assert err <= TOL_MIXED, (err, stats)


@pytest.mark.parametrize("overcorrect,ratio", [(1.0, 30.0), (1.7, 12.0), (1.95, 8.0), (1.3, 50.0)])
def test_amg_coarse_correction_scale_and_interval(ctx, overcorrect, ratio):
    """Coarse-correction scale in (0, 2) and Chebyshev interval [lmax/ratio, lmax] against the oracle
    (1.0 / 30 is the unscaled cycle; 1.7 / 12 the default)."""
    text = AMG_CASES["c3d20_box_3_levels"]()
    ref, _ = _oracle_run(text)
    p, st = _project(ctx, text)
    opts = fx.solve_opts(preconditioner=fx.PRECOND_AMG, amg_overcorrect=overcorrect, amg_cheb_ratio=ratio)
    stats = p.steps[0].solve(1, p, st, opts=opts)
    err = _err(st.displacements, ref)
    assert err <= TOL_MIXED, (err, stats)
    if (overcorrect, ratio) == (1.7, 12.0):  # the defaults
        st.initialize(p)
        d = p.steps[0].solve(1, p, st, opts=fx.solve_opts(preconditioner=fx.PRECOND_AMG))
        assert d["pcg_iterations"] == stats["pcg_iterations"]


@pytest.mark.parametrize("name", ["C3D4_staticstep", "C3D20", "NLGEOM_test"])
def test_amg_reference_decks(ctx, golden_dir, name):
    gold = json.load(open(os.path.join(golden_dir, "calculix.json")))[name]
    fix = np.load(os.path.join(golden_dir, f"oracle_{name}.npz"))
    p, st = _project(ctx, _deck(golden_dir, name))
    tol = TOL_NLGEOM if name.startswith("NLGEOM") else TOL_MIXED
    for k, want in enumerate(gold["steps"]):
        stats = p.steps[k].solve(k + 1, p, st, opts=fx.solve_opts(preconditioner=fx.PRECOND_AMG))
        ref = fix[f"step{k + 1}"]
        err = np.linalg.norm(st.displacements - ref) / np.linalg.norm(ref)
        assert err <= tol, (name, k, err, stats)


def test_nlgeom_repeatable(ctx):
    """An NLGEOM step solved twice on the same model gives the same bits: each increment's first
    Newton iteration rebuilds the multigrid hierarchy, the later ones refresh it, in the same order."""
    text = decks.c3d4_nlgeom_beam(12, 3, 3, tip_load=2.0e3, increments=4)
    p, st = _project(ctx, text)
    runs = []
    for _ in range(2):
        st.initialize(p)
        stats = p.steps[0].solve(1, p, st)
        runs.append((st.displacements.copy(), stats["pcg_iterations"], stats["newton_iterations"]))
    assert np.array_equal(runs[0][0], runs[1][0]) and runs[0][1:] == runs[1][1:]


def test_step_without_loads(ctx):
    """No *CLOAD: R = 0 passes the convergence test (absolute norm, static_step.rs:145-171)
    before any linear solve, so u stays exactly 0, as in the oracle."""
    text = decks.c3d4_cantilever(2, 2, 4)
    head, tail = text.split("*Cload, op=New", 1)
    text = head + "*End step" + tail.split("*End step", 1)[1]
    ref, r = _oracle_run(text)
    p, st = _project(ctx, text)
    stats = p.steps[0].solve(1, p, st)
    assert stats["linear_solves"] == 0 and np.array_equal(st.displacements, ref) and not ref.any()


def test_determinism(ctx):
    text = decks.c3d20_box(2, 2, 6)
    outs = []
    for _ in range(2):
        p, st = _project(ctx, text)
        p.steps[0].solve(1, p, st)
        outs.append(st.displacements)
    assert np.array_equal(outs[0], outs[1])


def test_errors_are_reported(ctx):
    # element without material: SolutionState::initialize panics in the reference
    bad = decks.c3d4_cantilever(1, 1, 1).replace("*Solid section, Elset=Vol, Material=Mat\n", "")
    p = fx.Project.from_inp_text(bad, ctx)
    with pytest.raises(fx.FerrixError) as e:
        fx.SolutionState().initialize(p)
    assert e.value.kind == "InvalidModelState"
    # degenerate (flat) tet: singular Jacobian
    flat = ("*NODE\n1,0,0,0\n2,1,0,0\n3,0,1,0\n4,1,1,0\n*ELEMENT, TYPE=C3D4, ELSET=E\n1,1,2,3,4\n"
            "*MATERIAL, NAME=M\n*ELASTIC\n1000,0.3\n*SOLID SECTION, ELSET=E, MATERIAL=M\n"
            "*STEP\n*STATIC\n*BOUNDARY\n1,1,3\n*CLOAD\n4,3,1.0\n*END STEP\n")
    p, st = _project(ctx, flat)
    with pytest.raises(fx.FerrixError) as e:
        p.steps[0].solve(1, p, st)
    assert e.value.kind == "NumericalError"
    # PCG iteration cap
    p, st = _project(ctx, decks.c3d4_cantilever(2, 2, 6))
    with pytest.raises(fx.FerrixError) as e:
        p.steps[0].solve(1, p, st, opts=fx.solve_opts(max_iter=2, poll_interval=2,
                                                      preconditioner=fx.PRECOND_BLOCK_JACOBI))
    assert e.value.kind == "ConvergenceError"
    # insufficient constraints (rigid-body modes): the reference's Cholesky fails with NumericalError
    # ("... Check for rigid body modes!"); the multigrid coarse solve finds the singular coarse operator
    # (the default solver), block-Jacobi PCG breaks down on the free deck (p.Kp <= 0)
    text = decks.c3d4_cantilever(3, 3, 6)
    lines, keep, skip = text.split("\n"), [], False
    for line in lines:  # the same deck without its *BOUNDARY blocks
        if line.upper().startswith("*BOUNDARY"):
            skip = True
            continue
        if skip and not line.startswith("*"):
            continue
        skip = False
        keep.append(line)
    free = "\n".join(keep)
    one_node = free.replace("*Cload", "*Boundary\n1, 1, 3\n*Cload", 1)  # one node fixed: rotations remain
    for deck, pcs in ((free, (fx.PRECOND_AMG, fx.PRECOND_BLOCK_JACOBI)), (one_node, (fx.PRECOND_AMG,))):
        for pc in pcs:
            p, st = _project(ctx, deck)
            with pytest.raises(fx.FerrixError) as e:
                p.steps[0].solve(1, p, st, opts=fx.solve_opts(preconditioner=pc))
            assert e.value.kind == "NumericalError" and "rigid body modes" in str(e.value), (pc, str(e.value))
    # unknown node in an element: NodeNotFound at the first element loop
    orphan = decks.c3d4_cantilever(1, 1, 1).replace("*Element, Type=C3D4, Elset=Solid\n",
                                                    "*Element, Type=C3D4, Elset=Solid\n99, 1, 2, 3, 12345\n")
    p, st = _project(ctx, orphan)
    with pytest.raises(fx.FerrixError) as e:
        p.steps[0].solve(1, p, st)
    assert e.value.kind == "NodeNotFound" and e.value.id == 12345 and e.value.line is None


def test_context_preloads_every_kernel(ctx):
    """fx_ctx_create loads all of the library's kernels on the device (a kernel loaded
    lazily at its first launch waits for the work of every other stream)."""
    n = ctx.preloaded_kernels
    assert n >= 50, n
    c2 = fx.Context(0)  # the second context on the device finds the same count
    try:
        assert c2.preloaded_kernels == n
    finally:
        c2.close()


@pytest.mark.parametrize("case", ["c3d4_cantilever", "c3d20_box_3_levels"])
def test_amg_fp16_smoother(ctx, case):
    """Fine-level smoothing with FP16 values of the scaled matrix D^-1/2 K D^-1/2 (the CG
    itself stays FP64): mixed-precision bound against the oracle, and about the iteration
    count of the FP32 smoother (multi-launch path, which is where the option applies)."""
    text = AMG_CASES[case]()
    ref, _ = _oracle_run(text)
    p, st = _project(ctx, text)
    s16 = p.steps[0].solve(1, p, st, opts=fx.solve_opts(amg_fp16_smoother=1, amg_persistent_max_dof=-1))
    err = _err(st.displacements, ref)
    st.initialize(p)
    s32 = p.steps[0].solve(1, p, st, opts=fx.solve_opts(amg_fp16_smoother=-1, amg_persistent_max_dof=-1))
    assert err <= TOL_MIXED, (err, s16)
    assert s16["pcg_iterations"] <= 1.25 * s32["pcg_iterations"] + 4, (s16["pcg_iterations"], s32["pcg_iterations"])
