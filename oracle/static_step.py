"""ORACLE — test infrastructure only (never imported by the product path).

Restatement of FerriX's static step driver:
  StaticStep::solve            src/solver/step/static_step.rs:47-267
  Step::solve (timer.new_step) src/solver/step/steps.rs:28-42
  IterativeSolver::solve       src/solver/solvers/iterative.rs:26-136
  DiagonalPreconditioner       src/solver/preconditioner.rs:36-58

Kept quirks: penalty = 1e6 x the largest single-element diagonal entry, added
once per BC record (static_step.rs:184-195); convergence on the BC-masked
||R||/||F_ext|| < 1e-3 with at most 15 Newton iterations (:99-171); NLGEOM
evaluates K and f_int on X+u with small-strain B (:121-181); the timer is
advanced at the start of every attempt, failed ones included (:84), and the
increment is only ever halved (:251-259).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np
import scipy.sparse as sp

from . import elem
from .inp import FerrixError, ModelArrays, Project, SolverTime, initial_temperatures, model_arrays
from .sparse_direct import MultifrontalCholesky


@dataclass
class SolutionState:
    displacements: np.ndarray
    initial_temperatures: np.ndarray
    temperatures: np.ndarray


def new_state(p: Project) -> SolutionState:
    n = len(p.index_to_node_id)
    t = initial_temperatures(p)
    return SolutionState(np.zeros(3 * n), t.copy(), t.copy())


@dataclass
class IncrementLog:
    step: int
    increment: int
    dt: float
    converged: bool
    residuals: List[float] = field(default_factory=list)


@dataclass
class Timings:
    assembly: float = 0.0
    csr: float = 0.0
    factor: float = 0.0
    solve: float = 0.0
    forces: float = 0.0
    analyse: float = 0.0


def jacobi_pcg(K: sp.csr_matrix, b: np.ndarray, tol: float = 1e-8, max_iter: int = 1000) -> np.ndarray:
    """IterativeSolver::solve (iterative.rs:26-136) with DiagonalPreconditioner."""
    d = K.diagonal()
    inv = np.ones_like(d)
    big = np.abs(d) > 1e-9
    inv[big] = 1.0 / d[big]
    x = np.zeros_like(b)
    r = b.copy()
    z = r * inv
    p = z.copy()
    rs = float(r @ z)
    for _ in range(max_iter):
        if np.sqrt(rs) < tol:
            return x
        ap = K @ p
        alpha = rs / float(p @ ap)
        x += alpha * p
        r -= alpha * ap
        z = r * inv
        rs_new = float(r @ z)
        p = z + (rs_new / rs) * p
        rs = rs_new
    raise FerrixError("ConvergenceError", f"PCG did not converge after {max_iter} iterations")


class Runner:
    """Holds the dense model view, the ordering and timings across steps."""

    def __init__(self, project: Project, verbose: bool = False, on_increment=None):
        self.p = project
        # on_increment(step_id, inc_id, global_time, displacements): called after every
        # converged increment, where static_step.rs:219-248 hands the result to the writer
        self.on_increment = on_increment
        self.m: ModelArrays = model_arrays(project)
        self.mf: Optional[MultifrontalCholesky] = None
        self.verbose = verbose
        self.log: List[IncrementLog] = []
        self.t = Timings()
        self.last_K = None
        self.last_R = None
        self.last_du = None

    def _direct(self, K, R):
        if self.mf is None:
            t0 = time.perf_counter()
            self.mf = MultifrontalCholesky(self.m.xyz, [g[1] for _, g in sorted(self.m.groups.items())])
            self.t.analyse += time.perf_counter() - t0
        t0 = time.perf_counter()
        self.mf.factor(K)
        t1 = time.perf_counter()
        x = self.mf.solve(R)
        self.t.factor += t1 - t0
        self.t.solve += time.perf_counter() - t1
        return x

    def solve_step(self, step_index: int, state: SolutionState, timer: SolverTime) -> None:
        """Step::solve + StaticStep::solve for project.steps[step_index] (step_id = index + 1)."""
        p, m = self.p, self.m
        step = p.steps[step_index]
        step_id = step_index + 1
        timer.new_step(step.increment.time_period)
        inc = step.increment
        ndof = state.displacements.shape[0]
        cur = 0.0
        n_inc = 0
        dt = inc.initial_time_increment
        u_start = state.displacements.copy()
        bc_idx = []
        for bc in step.bcs:
            i = p.index_of(bc.node_id)
            bc_idx.append(None if i is None else 3 * i + bc.dof)
        while cur < inc.time_period:
            n_inc += 1
            if n_inc > inc.max_iterations:
                raise FerrixError("ConvergenceError", f"Maximum increment count of {inc.max_iterations} exceeded.")
            if cur + dt > inc.time_period:
                dt = inc.time_period - cur
            timer.new_increment(dt)
            rec = IncrementLog(step_id, n_inc, dt, False)
            converged = False
            u = u_start.copy()
            for _ in range(15):
                t0 = time.perf_counter()
                f_ext = np.zeros(ndof)
                for ld in step.loads:
                    i = p.index_of(ld.node_id)
                    if i is not None:
                        f_ext[3 * i + ld.dof] += ld.eval(timer, step_id)
                f_ext += elem.thermal_force(m, state.initial_temperatures, state.temperatures)
                f_int = elem.internal_force(m, u, u if step.nlgeom else None, state.initial_temperatures,
                                            state.temperatures)
                R = f_ext - f_int
                rc = R.copy()
                fc = f_ext.copy()
                for gd in bc_idx:
                    if gd is not None and gd < ndof:
                        rc[gd] = 0.0
                        fc[gd] = 0.0
                rn = float(np.sqrt(np.sum(rc * rc)))
                fn = float(np.sqrt(np.sum(fc * fc)))
                rel = rn / fn if fn > 1e-6 else rn
                rec.residuals.append(rel)
                self.t.forces += time.perf_counter() - t0
                if self.verbose:
                    print(f"  step {step_id} inc {n_inc} |R|={rn:.3e} rel={rel:.3e}")
                if rel < 1e-3:
                    converged = True
                    break
                t0 = time.perf_counter()
                K, maxdiag = elem.assemble(m, u if step.nlgeom else None, state.temperatures)
                self.t.assembly += time.perf_counter() - t0
                t0 = time.perf_counter()
                if maxdiag > 0.0:
                    pen = maxdiag * 1.0e6
                    padd = np.zeros(ndof)
                    for bc, gd in zip(step.bcs, bc_idx):
                        if gd is None:
                            continue
                        padd[gd] += pen
                        R[gd] += pen * (bc.eval(timer, step_id) - u[gd])
                    K = (K + sp.diags(padd, format="csr")).tocsr()
                self.t.csr += time.perf_counter() - t0
                self.last_K, self.last_R = K, R
                if step.solver == "ITERATIVE":
                    t0 = time.perf_counter()
                    du = jacobi_pcg(K, R, 1e-8, 1000)
                    self.t.solve += time.perf_counter() - t0
                else:
                    du = self._direct(K, R)
                self.last_du = du
                u += du
            rec.converged = converged
            self.log.append(rec)
            if converged:
                cur += dt
                u_start = u.copy()
                if self.on_increment is not None:
                    self.on_increment(step_id, n_inc, timer.global_, u_start.copy())
            else:
                dt /= 2.0
                if dt < inc.min_time_increment:
                    raise FerrixError("ConvergenceError", "Minimum time increment reached. Convergence failed.")
        state.displacements = u_start

    def run(self, state: Optional[SolutionState] = None, steps: Optional[List[int]] = None) -> SolutionState:
        state = state or new_state(self.p)
        timer = SolverTime()
        for k in (steps if steps is not None else range(len(self.p.steps))):
            self.solve_step(k, state, timer)
        return state
