"""ferrix_b200 — B200 (sm_100a) solver for FerriX's linear-static and NLGEOM
*STATIC path (C3D4 / C3D20), behind the C ABI of include/ferrix_b200.h.

The Python layer mirrors the reference's host interface so a FerriX test
reads the same:

    ctx = Context(0)
    project = Project.from_jobname("tests/data/C3D4_staticstep", ctx)   # src/solver/project.rs:93-127
    project.default_initial_temperature = 20.0                          # tests/calculix_parity.rs:29
    state = SolutionState(project.num_dofs, project.num_nodes)          # src/solver/state.rs:32-42
    state.initialize(project)                                           # src/solver/state.rs:47-79
    timer = SolverTime()
    for i, step in enumerate(project.steps):
        step.solve(i + 1, project, state, writer, timer)                # src/solver/step/steps.rs:28-42
    idx = project.mesh.get_index_for_node_id(17)
    ux = state.displacements[idx * 3]

Errors raise FerrixError with the reference's variant name in `.kind`.
Everything numeric runs in libferrix_b200.so on the GPU; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import PRECOND_AMG, PRECOND_BLOCK_JACOBI, PREC_FP64, PREC_FP64_CSR, PREC_MIXED, SolveOpts, StepStats

__all__ = ["Context", "Project", "SolutionState", "SolverTime", "FerrixError", "SolveOptions", "solve_opts",
           "batch_solve", "Server", "StepStats", "PREC_MIXED", "PREC_FP64", "PREC_FP64_CSR", "PRECOND_AMG",
           "PRECOND_BLOCK_JACOBI"]


class FerrixError(Exception):
    """A FerrixError variant (src/solver/error.rs:12-72): `kind` is the variant's name,
    `line` the deck line of ParseError / UnsupportedKeyword, `id` the id of
    NodeNotFound / ElementNotFound (None where the variant has none), `text` the
    variant's string field (message, keyword, material / set / solver name)."""

    def __init__(self, status: int, message: str, line: Optional[int] = None, id: Optional[int] = None,
                 text: Optional[str] = None):
        self.status = status
        self.kind = _lib.STATUS_NAMES.get(status, str(status))
        self.message = message
        self.line = line
        self.id = id
        self.text = message if text is None else text
        super().__init__(f"{self.kind}: {message}")


def _check(rc: int, ctx=None, what: str = ""):
    if rc != 0:
        d = _lib.ErrorDetail()
        h = ctx.handle if ctx is not None and ctx.handle else None
        _lib.load().fx_last_error_detail(h, C.byref(d))
        if d.status == rc:
            msg = d.message.decode(errors="replace")
            raise FerrixError(rc, msg or what, None if d.line < 0 else int(d.line), None if d.id < 0 else int(d.id),
                              d.text.decode(errors="replace"))
        raise FerrixError(rc, what)


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class Context:
    """One GPU and one CUDA stream (fx_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        _check(self.lib.fx_ctx_create(device, C.byref(h)), None, f"fx_ctx_create({device})")
        self.handle = h
        # raw handles of the live models bound to this context: models must be
        # destroyed before their context, also when the garbage collector
        # finalizes a context and its projects in arbitrary order
        self._models = {}

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.fx_ctx_kernel_launches(self.handle))

    @property
    def preloaded_kernels(self) -> int:
        """Kernels of the library found loaded on the device at creation (-1: loaded at first use)."""
        return int(self.lib.fx_ctx_preloaded_kernels(self.handle))

    @property
    def stream(self) -> int:
        """cudaStream_t of the context (for CUDA events recorded by the caller)."""
        return int(self.lib.fx_ctx_stream(self.handle) or 0)

    def close(self):
        if self.handle:
            for h in list(self._models.values()):
                self.lib.fx_model_destroy(h)
            self._models.clear()
            self.lib.fx_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_opts(precision: int = PREC_MIXED, rtol: float = 1e-8, max_iter: int = 50000, poll_interval: int = 32,
               reliable_delta: float = 1e-2, use_graphs: bool = True, verbose: bool = False,
               reference_iterative: bool = False, preconditioner: int = PRECOND_AMG,
               amg_aggregate_nodes: int = 40, amg_smoother_degree: int = 2, amg_cycle: int = 0,
               amg_smoother: int = 0, amg_overcorrect: float = 0.0, amg_cheb_ratio: float = 0.0,
               amg_persistent_max_dof: int = 0, amg_fused_coarse: int = 0,
               amg_fp16_smoother: int = 0) -> SolveOpts:
    o = SolveOpts()
    _lib.load().fx_default_solve_opts(C.byref(o))
    o.precision = precision
    o.rtol = rtol
    o.max_iter = max_iter
    o.poll_interval = poll_interval
    o.reliable_delta = reliable_delta
    o.use_graphs = int(use_graphs)
    o.verbose = int(verbose)
    o.reference_iterative = int(reference_iterative)
    o.preconditioner = int(preconditioner)
    o.amg_aggregate_nodes = int(amg_aggregate_nodes)
    o.amg_smoother_degree = int(amg_smoother_degree)
    o.amg_cycle = int(amg_cycle)
    o.amg_smoother = int(amg_smoother)
    o.amg_overcorrect = float(amg_overcorrect)
    o.amg_cheb_ratio = float(amg_cheb_ratio)
    o.amg_persistent_max_dof = int(amg_persistent_max_dof)
    o.amg_fused_coarse = int(amg_fused_coarse)
    o.amg_fp16_smoother = int(amg_fp16_smoother)
    return o


SolveOptions = solve_opts


class SolverTime:
    """Marker mirroring src/solver/time.rs; the running time lives in the model."""


@dataclass
class IncResult:
    """A converged increment as Step.solve hands it to a writer's write_increment
    (IncResult, src/solver/results.rs; handed over at src/solver/step/static_step.rs:219-248):
    1-based step id, the step's increment counter (failed attempts included) and the global
    time. While write_increment runs, `project` holds that increment's displacements."""
    step_id: int
    inc_id: int
    time: float
    project: "Project"


class VtkWriter:
    """VtkWriter (src/solver/io/vtk.rs:19-334) as a Step.solve writer: init() creates
    `directory` and its results.vtk.series, write_increment() writes the increment's
    step_<step_id>_<inc_id>.vtk (displacements, temperatures, nodal stress / strain, Mises,
    Tresca) and its series entry, finish() closes the series."""

    def __init__(self, project: "Project", directory: str):
        self.project = project
        self.directory = directory

    def init(self) -> None:
        _check(_lib.load().fx_vtk_series_init(os.fsencode(self.directory)))

    def write_increment(self, inc: IncResult, timer: Optional[SolverTime] = None) -> None:
        name = f"step_{inc.step_id}_{inc.inc_id}.vtk"
        self.project.write_vtk(os.path.join(self.directory, name))
        _check(_lib.load().fx_vtk_series_add(os.fsencode(self.directory), name.encode(), float(inc.time)))

    def finish(self) -> None:
        _check(_lib.load().fx_vtk_series_finish(os.fsencode(self.directory)))


class _Mesh:
    def __init__(self, project: "Project"):
        self._p = project

    def get_index_for_node_id(self, node_id: int) -> Optional[int]:
        i = int(self._p.lib.fx_model_node_index(self._p.handle, int(node_id)))
        return None if i < 0 else i

    @property
    def index_to_node_id(self) -> np.ndarray:
        ids = np.empty(self._p.num_nodes, dtype=np.int64)
        _check(self._p.lib.fx_model_node_ids(self._p.handle, _p(ids)), self._p.ctx)
        return ids


@dataclass
class StepInfo:
    nlgeom: bool
    solver: str
    increment: tuple
    n_loads: int
    n_bcs: int


class Step:
    def __init__(self, project: "Project", index: int):
        self.project = project
        self.index = index
        nl = C.c_int()
        sv = C.c_int()
        inc = (C.c_double * 4)()
        a = C.c_int64()
        b = C.c_int64()
        _check(project.lib.fx_model_step_info(project.handle, index, C.byref(nl), C.byref(sv), inc, C.byref(a),
                                              C.byref(b)), project.ctx)
        self.info = StepInfo(bool(nl.value), ["DEFAULT", "DIRECT", "ITERATIVE"][sv.value], tuple(inc), a.value,
                             b.value)
        self.last_stats: Optional[dict] = None

    def solve(self, step_id: int, project: "Project", solution_state: "SolutionState", writer=None,
              timer: Optional[SolverTime] = None, opts: Optional[SolveOpts] = None) -> dict:
        """Step::solve (src/solver/step/steps.rs:28-42) for this step; step_id must be index + 1."""
        if step_id != self.index + 1:
            raise ValueError("step_id must be the 1-based position of the step")
        st = StepStats()
        o = opts if opts is not None else solve_opts()
        if writer is not None and hasattr(writer, "write_increment"):
            # the writer sees every converged increment, as ResultWriter::write_increment does
            errors = []

            def on_increment(user, model, step, inc, t):
                try:
                    writer.write_increment(IncResult(step, inc, t, project), timer)
                    return 0
                except Exception as e:  # ends the step (FX_GENERIC_IO); re-raised below
                    errors.append(e)
                    return 1
            cb = _lib.IncrementCallback(on_increment)
            rc = project.lib.fx_step_solve_cb(project.handle, self.index, C.byref(o), C.byref(st), cb, None)
            if errors:
                raise errors[0]
            _check(rc, project.ctx)
        else:
            _check(project.lib.fx_step_solve(project.handle, self.index, C.byref(o), C.byref(st)), project.ctx)
        self.last_stats = st.as_dict()
        return self.last_stats

    def records(self, bcs: bool = False):
        n = self.info.n_bcs if bcs else self.info.n_loads
        ids = np.empty(n, dtype=np.int64)
        dofs = np.empty(n, dtype=np.int32)
        vals = np.empty(n, dtype=np.float64)
        org = np.empty(n, dtype=np.int64)
        tab = np.empty(n, dtype=np.int32)
        _check(self.project.lib.fx_model_step_records(self.project.handle, self.index, int(bcs), _p(ids), _p(dofs),
                                                      _p(vals), _p(org), _p(tab)), self.project.ctx)
        return ids, dofs, vals, org, tab


class Project:
    """fx_model: the parsed deck plus its device-resident solution state."""

    def __init__(self, handle, ctx: Optional[Context]):
        self.lib = _lib.load()
        self.handle = handle
        self.ctx = ctx
        nn = C.c_int64()
        ne = C.c_int64()
        ns = C.c_int()
        nm = C.c_int()
        _check(self.lib.fx_model_sizes(handle, C.byref(nn), C.byref(ne), C.byref(ns), C.byref(nm)), ctx)
        self.num_nodes = nn.value
        self.num_elements = ne.value
        self.num_dofs = 3 * nn.value
        self.num_materials = nm.value
        self.mesh = _Mesh(self)
        self.steps: List[Step] = [Step(self, k) for k in range(ns.value)]
        self._default_t = 0.0
        if ctx is not None:
            ctx._models[id(self)] = handle

    @classmethod
    def from_inp_text(cls, text: str, ctx: Optional[Context] = None) -> "Project":
        lib = _lib.load()
        raw = bytes(text) if isinstance(text, (bytes, bytearray, memoryview)) else text.encode()
        h = C.c_void_p()
        _check(lib.fx_model_from_inp(ctx.handle if ctx else None, raw, len(raw), C.byref(h)), ctx)
        return cls(h, ctx)

    @classmethod
    def from_arrays(cls, node_ids, xyz, c3d4=None, c3d20=None, materials=(), amplitudes=(), steps=(),
                    default_temperature: float = 0.0, initial_temperatures=None,
                    ctx: Optional[Context] = None) -> "Project":
        """fx_model_from_arrays: the model a parsed deck gives, from arrays.

        node_ids (N,), xyz (N, 3); c3d4 / c3d20 = (element ids, node ids per element
        (E, 4 | 20), material index per element or None); materials = dicts with
        "name", "E", "nu", "alpha" ((T, value) pairs; alpha may be empty) and "tref";
        amplitudes = dicts with "time", "value", "total_time", "shift_x", "shift_y";
        steps = dicts with "nlgeom", "solver" (0 default, 1 direct, 2 iterative),
        "increment" (initial, period, min, max), "max_increments" and "loads" / "bcs":
        sequences of (node id, dof 0..2, value, amplitude index or -1, origin step);
        initial_temperatures = {node id: T}."""
        lib = _lib.load()
        keep = []  # every array the descriptor points into stays alive until the call returns

        def arr(a, dtype):
            a = np.ascontiguousarray(np.asarray(a, dtype=dtype))
            keep.append(a)
            return a

        def ptr(a):
            return a.ctypes.data_as(C.c_void_p) if a.size else None

        d = _lib.MeshDesc()
        ids = arr(node_ids, np.int64)
        xs = arr(xyz, np.float64).reshape(-1)
        d.n_nodes = ids.size
        d.node_ids, d.xyz = ptr(ids), ptr(xs)
        for npe, grp in ((4, c3d4), (20, c3d20)):
            if grp is None:
                continue
            eids = arr(grp[0], np.int64)
            conn = arr(grp[1], np.int64).reshape(-1)
            mat = None if len(grp) < 3 or grp[2] is None else arr(grp[2], np.int32)
            setattr(d, f"n_c3d{npe}", eids.size)
            setattr(d, f"c3d{npe}_ids", ptr(eids))
            setattr(d, f"c3d{npe}_nodes", ptr(conn))
            setattr(d, f"c3d{npe}_material", None if mat is None else ptr(mat))

        def lut(pairs):
            a = arr(pairs, np.float64).reshape(-1, 2) if len(pairs) else np.zeros((0, 2))
            t, v = arr(a[:, 0], np.float64), arr(a[:, 1], np.float64)
            return _lib.LutDesc(len(a), ptr(t), ptr(v))

        mats = (_lib.MaterialDesc * max(1, len(materials)))()
        for k, m in enumerate(materials):
            name = (m.get("name") or "").encode()
            keep.append(name)
            mats[k] = _lib.MaterialDesc(name, lut(m.get("E", ())), lut(m.get("nu", ())),
                                        lut(m.get("alpha", ())), float(m.get("tref", 0.0)))
        d.n_materials, d.materials = len(materials), C.cast(mats, C.c_void_p)
        amps = (_lib.AmplitudeDesc * max(1, len(amplitudes)))()
        for k, a in enumerate(amplitudes):
            t, v = arr(a["time"], np.float64), arr(a["value"], np.float64)
            amps[k] = _lib.AmplitudeDesc(t.size, ptr(t), ptr(v), int(bool(a.get("total_time", False))),
                                         float(a.get("shift_x", 0.0)), float(a.get("shift_y", 0.0)))
        d.n_amplitudes, d.amplitudes = len(amplitudes), C.cast(amps, C.c_void_p)

        rec_dtype = np.dtype({"names": ["node_id", "dof", "amplitude", "value", "origin_step"],
                              "formats": [np.int64, np.int32, np.int32, np.float64, np.int64],
                              "offsets": [0, 8, 12, 16, 24], "itemsize": C.sizeof(_lib.RecordDesc)})

        def records(recs):
            if isinstance(recs, np.ndarray) and recs.dtype == rec_dtype:
                r = np.ascontiguousarray(recs)
            else:
                r = np.zeros(len(recs), dtype=rec_dtype)
                if len(recs):
                    cols = list(zip(*recs))
                    r["node_id"], r["dof"], r["value"] = cols[0], cols[1], cols[2]
                    r["amplitude"], r["origin_step"] = cols[3], cols[4]
            keep.append(r)
            return r.size, (r.ctypes.data_as(C.c_void_p) if r.size else None)

        sts = (_lib.StepDesc * max(1, len(steps)))()
        for k, st in enumerate(steps):
            nl, lp = records(st.get("loads", ()))
            nb, bp = records(st.get("bcs", ()))
            sts[k] = _lib.StepDesc(int(bool(st.get("nlgeom", False))), int(st.get("solver", 0)),
                                   (C.c_double * 4)(*st.get("increment", (1.0, 1.0, 1e-5, 1.0))),
                                   int(st.get("max_increments", 10000)), nl, lp, nb, bp)
        d.n_steps, d.steps = len(steps), C.cast(sts, C.c_void_p)
        d.default_temperature = float(default_temperature)
        if initial_temperatures:
            ti = arr(list(initial_temperatures.keys()), np.int64)
            tv = arr(list(initial_temperatures.values()), np.float64)
            d.n_initial_temperatures, d.initial_temperature_ids, d.initial_temperatures = ti.size, ptr(ti), ptr(tv)
        h = C.c_void_p()
        _check(lib.fx_model_from_arrays(ctx.handle if ctx else None, C.byref(d), C.byref(h)), ctx)
        p = cls(h, ctx)
        p._default_t = float(default_temperature)
        return p

    @classmethod
    def from_jobname(cls, jobname: str, ctx: Optional[Context] = None) -> "Project":
        path = jobname if jobname.lower().endswith(".inp") else jobname + ".inp"
        try:
            with open(path, "rb") as fh:  # the bytes go to the parser as they are
                raw = fh.read()
        except OSError as e:
            raise FerrixError(1, f"IO error at {path}: {e}")
        return cls.from_inp_text(raw, ctx)

    @property
    def default_initial_temperature(self) -> float:
        return self._default_t

    @default_initial_temperature.setter
    def default_initial_temperature(self, t: float) -> None:
        self._default_t = float(t)
        _check(self.lib.fx_model_set_default_temperature(self.handle, float(t)), self.ctx)

    def export(self):
        """Dense arrays: xyz (N,3), {4: (conn, mat), 20: (conn, mat)}."""
        xyz = np.empty(3 * self.num_nodes)
        n4 = C.c_int64()
        n20 = C.c_int64()
        _check(self.lib.fx_model_export(self.handle, None, C.byref(n4), None, None, C.byref(n20), None, None), self.ctx)
        c4 = np.empty(4 * n4.value, dtype=np.int32)
        m4 = np.empty(n4.value, dtype=np.int32)
        c20 = np.empty(20 * n20.value, dtype=np.int32)
        m20 = np.empty(n20.value, dtype=np.int32)
        _check(self.lib.fx_model_export(self.handle, _p(xyz), C.byref(n4), _p(c4), _p(m4), C.byref(n20), _p(c20),
                                        _p(m20)), self.ctx)
        return xyz.reshape(-1, 3), {4: (c4.reshape(-1, 4), m4), 20: (c20.reshape(-1, 20), m20)}

    def assemble_csr(self, u: Optional[np.ndarray] = None, precision: int = PREC_FP64):
        """Assembler::assemble + to_csr on the GPU: (indptr, indices, data, maxdiag)."""
        nnz = C.c_int64()
        uu = None if u is None else np.ascontiguousarray(u, dtype=np.float64)
        _check(self.lib.fx_assemble_csr(self.handle, _p(uu), precision, C.byref(nnz), None, None, None, None),
               self.ctx)
        ip = np.empty(self.num_dofs + 1, dtype=np.int64)
        ind = np.empty(nnz.value, dtype=np.int64)
        dat = np.empty(nnz.value, dtype=np.float64)
        md = C.c_double()
        _check(self.lib.fx_assemble_csr(self.handle, _p(uu), precision, C.byref(nnz), _p(ip), _p(ind), _p(dat),
                                        C.byref(md)), self.ctx)
        return ip, ind, dat, md.value

    def internal_force(self, u: np.ndarray, uconf: Optional[np.ndarray] = None) -> np.ndarray:
        f = np.empty(self.num_dofs)
        uu = np.ascontiguousarray(u, dtype=np.float64)
        uc = None if uconf is None else np.ascontiguousarray(uconf, dtype=np.float64)
        _check(self.lib.fx_internal_force(self.handle, _p(uu), _p(uc), _p(f)), self.ctx)
        return f

    def drop_cache(self) -> None:
        _check(self.lib.fx_model_drop_cache(self.handle), self.ctx)

    def profile_spmv(self, precision: int = PREC_FP64, reps: int = 20):
        """(mean ms of one standalone SpMV launch, algorithmic bytes per launch)."""
        ms = C.c_double()
        by = C.c_double()
        _check(self.lib.fx_profile_spmv(self.handle, precision, reps, C.byref(ms), C.byref(by)), self.ctx)
        return ms.value, by.value

    def nodal_stress_strain(self):
        """(S, E): nodal-averaged stress and mechanical strain, (N, 6) each, Voigt xx yy zz xy yz zx
        (StaticStep::calculate_stress_strain, src/solver/step/static_step.rs:271-379)."""
        S = np.empty((self.num_nodes, 6))
        E = np.empty((self.num_nodes, 6))
        _check(self.lib.fx_nodal_stress_strain(self.handle, _p(S), _p(E)), self.ctx)
        return S, E

    def write_vtk(self, path: str) -> None:
        """Legacy ASCII VTK of the current state (VtkWriter::write_increment, src/solver/io/vtk.rs:72-319)."""
        _check(self.lib.fx_write_vtk(self.handle, os.fsencode(path)), self.ctx)

    def profile_assembly(self, precision: int = PREC_FP64, reps: int = 10):
        """fx_profile_assembly: (stiffness ms, declared FLOPs, gather ms, gather bytes) per launch."""
        a, b, c, d = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        _check(self.lib.fx_profile_assembly(self.handle, precision, reps, C.byref(a), C.byref(b), C.byref(c),
                                            C.byref(d)), self.ctx)
        return a.value, b.value, c.value, d.value

    def profile_smoother(self, precision: int = PREC_MIXED, reps: int = 20, fp16: bool = False):
        """(mean ms, compulsory bytes) of one fused fine-level multigrid smoothing step."""
        ms = C.c_double()
        by = C.c_double()
        _check(self.lib.fx_profile_smoother(self.handle, precision, int(fp16), reps, C.byref(ms), C.byref(by)),
               self.ctx)
        return ms.value, by.value

    def thermal_force(self) -> np.ndarray:
        f = np.empty(self.num_dofs)
        _check(self.lib.fx_thermal_force(self.handle, _p(f)), self.ctx)
        return f

    def close(self):
        if self.handle:
            if self.ctx is None:
                self.lib.fx_model_destroy(self.handle)
            elif self.ctx._models.pop(id(self), None) is not None:
                self.lib.fx_model_destroy(self.handle)
            # else: the context was closed first and destroyed this model with it
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolutionState:
    """SolutionState (src/solver/state.rs:16-79); the vectors stay on the GPU."""

    def __init__(self, num_dofs: int = 0, num_nodes: int = 0):
        self.num_dofs = num_dofs
        self.num_nodes = num_nodes
        self.project: Optional[Project] = None

    def initialize(self, project: Project) -> None:
        self.project = project
        _check(project.lib.fx_state_initialize(project.handle), project.ctx)

    @property
    def displacements(self) -> np.ndarray:
        u = np.empty(self.project.num_dofs)
        _check(self.project.lib.fx_state_get_displacements(self.project.handle, _p(u)), self.project.ctx)
        return u

    @displacements.setter
    def displacements(self, u: np.ndarray) -> None:
        uu = np.ascontiguousarray(u, dtype=np.float64)
        _check(self.project.lib.fx_state_set_displacements(self.project.handle, _p(uu)), self.project.ctx)

    @property
    def temperatures(self):
        ti = np.empty(self.project.num_nodes)
        tc = np.empty(self.project.num_nodes)
        _check(self.project.lib.fx_state_get_temperatures(self.project.handle, _p(ti), _p(tc)), self.project.ctx)
        return ti, tc

    def set_temperatures(self, t_init: Optional[np.ndarray] = None, t_cur: Optional[np.ndarray] = None) -> None:
        a = None if t_init is None else np.ascontiguousarray(t_init, dtype=np.float64)
        b = None if t_cur is None else np.ascontiguousarray(t_cur, dtype=np.float64)
        _check(self.project.lib.fx_state_set_temperatures(self.project.handle, _p(a), _p(b)), self.project.ctx)


def batch_solve(ctx: Context, projects: Sequence[Project], opts: Optional[SolveOpts] = None):
    """First step of every (initialized) project with the linear solves batched; returns (status, stats)."""
    lib = _lib.load()
    n = len(projects)
    arr = (C.c_void_p * n)(*[p.handle for p in projects])
    st = np.zeros(n, dtype=np.int32)
    stats = (StepStats * n)()
    o = opts if opts is not None else solve_opts()
    rc = lib.fx_batch_solve(ctx.handle, C.cast(arr, C.c_void_p), n, C.byref(o), _p(st), C.cast(stats, C.c_void_p))
    if rc != 0 and not np.any(st != 0):
        _check(rc, ctx)
    return st, [s.as_dict() for s in stats]


class Server:
    """Request loop with continuous batching on one GPU (fx_server_*).

    Projects are parsed on the host (`Project.from_inp_text(text)` without a
    context) and submitted; `slots` worker threads admit them by HBM footprint
    and solve their first step concurrently, each on its own stream. `wait`
    returns the displacements and the request's timing."""

    def __init__(self, device: int = 0, slots: int = 4, hbm_budget_bytes: float = 0.0,
                 opts: Optional[SolveOpts] = None):
        self.lib = _lib.load()
        so = _lib.ServerOpts()
        self.lib.fx_default_server_opts(C.byref(so))
        so.device = device
        so.slots = slots
        so.hbm_budget_bytes = float(hbm_budget_bytes)
        if opts is not None:
            so.opts = opts
        h = C.c_void_p()
        _check(self.lib.fx_server_create(C.byref(so), C.byref(h)), None, "fx_server_create")
        self.handle = h
        self._pending = {}  # ticket -> project (kept alive while the server uses it)

    def info(self) -> dict:
        """fx_server_get_info: slots, kernels the slot contexts found loaded, admission budget,
        device pool bytes held after the budget's reservation and its outcome (1 grew, 0 held
        enough already, -1 could not grow in one piece)."""
        i = _lib.ServerInfo()
        _check(self.lib.fx_server_get_info(self.handle, C.byref(i)), None, "fx_server_get_info")
        return {k: getattr(i, k) for k, _ in i._fields_}

    def submit(self, project: "Project") -> int:
        if project.ctx is not None:
            raise ValueError("submit a host-only project (Project.from_inp_text(text) without a context)")
        t = C.c_int64()
        _check(self.lib.fx_server_submit(self.handle, project.handle, C.byref(t)), None, "fx_server_submit")
        self._pending[t.value] = project
        return t.value

    def wait(self, ticket: int, timeout: float = -1.0):
        """(displacements or None, result dict); raises FerrixError(FX_TIMEOUT) when not done in time."""
        p = self._pending[ticket]
        u = np.empty(p.num_dofs)
        res = _lib.RequestResult()
        res.status = -1  # filled only once the request is done
        rc = self.lib.fx_server_wait(self.handle, ticket, float(timeout), _p(u), C.byref(res))
        if res.status == -1:
            raise FerrixError(rc, "request not finished" if rc == 16 else "fx_server_wait failed")
        self._pending.pop(ticket, None)
        out = {"status": res.status, "slot": res.slot, "queue_ms": res.queue_ms, "service_ms": res.service_ms,
               "latency_ms": res.latency_ms, "footprint_bytes": res.footprint_bytes,
               "admit_at_ms": res.admit_at_ms, "done_at_ms": res.done_at_ms,
               "stats": res.stats.as_dict(), "error": res.error.decode(errors="replace"),
               "setup_ms": res.setup_ms, "solve_ms": res.solve_ms, "finish_ms": res.finish_ms}
        return (u if res.status == 0 else None), out

    def close(self):
        if self.handle:
            self.lib.fx_server_destroy(self.handle)
            self.handle = None
            self._pending.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
