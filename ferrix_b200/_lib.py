"""ctypes binding of libferrix_b200.so (declarations in include/ferrix_b200.h).

The shared library is built in-tree by ferrix_b200/build.py. There is no
fallback: if the library cannot be loaded, importing the solver API raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libferrix_b200.so")

STATUS_NAMES = {
    0: "Ok", 1: "Io", 2: "GenericIo", 3: "ParseError", 4: "UnsupportedKeyword", 5: "UnknownSolver",
    6: "NodeNotFound", 7: "ElementNotFound", 8: "MaterialNotFound", 9: "ElsetNotFound", 10: "NsetNotFound",
    11: "NumericalError", 12: "ConvergenceError", 13: "InvalidModelState", 14: "Generic", 15: "Cancelled",
    16: "Timeout", 17: "Cuda", 18: "InvalidArgument",
}

PREC_MIXED = 0
PREC_FP64 = 1
PREC_FP64_CSR = 2
PRECOND_BLOCK_JACOBI = 0
PRECOND_AMG = 1


class SolveOpts(C.Structure):
    _fields_ = [("precision", C.c_int), ("rtol", C.c_double), ("max_iter", C.c_int), ("poll_interval", C.c_int),
                ("reliable_delta", C.c_double), ("use_graphs", C.c_int), ("verbose", C.c_int),
                ("reference_iterative", C.c_int), ("preconditioner", C.c_int),
                ("amg_aggregate_nodes", C.c_int), ("amg_smoother_degree", C.c_int), ("amg_cycle", C.c_int),
                ("amg_smoother", C.c_int), ("amg_overcorrect", C.c_double), ("amg_cheb_ratio", C.c_double),
                ("amg_persistent_max_dof", C.c_int), ("amg_fused_coarse", C.c_int),
                ("amg_fp16_smoother", C.c_int)]


class StepStats(C.Structure):
    _fields_ = [("increments", C.c_int), ("newton_iterations", C.c_int), ("linear_solves", C.c_int),
                ("pcg_iterations", C.c_longlong), ("reliable_updates", C.c_int),
                ("last_rel_residual", C.c_double), ("last_linear_relres", C.c_double),
                ("t_symbolic_ms", C.c_double), ("t_assembly_ms", C.c_double), ("t_forces_ms", C.c_double),
                ("t_pcg_ms", C.c_double), ("t_total_ms", C.c_double), ("bsr_blocks", C.c_int64),
                ("fp64_fallbacks", C.c_int), ("amg_levels", C.c_int), ("amg_setup_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("slots", C.c_int), ("hbm_budget_bytes", C.c_double), ("opts", SolveOpts)]


class RequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("slot", C.c_int), ("queue_ms", C.c_double), ("service_ms", C.c_double),
                ("latency_ms", C.c_double), ("footprint_bytes", C.c_double), ("admit_at_ms", C.c_double),
                ("done_at_ms", C.c_double), ("stats", StepStats),
                ("error", C.c_char * 256), ("setup_ms", C.c_double), ("solve_ms", C.c_double),
                ("finish_ms", C.c_double)]


class ErrorDetail(C.Structure):
    _fields_ = [("status", C.c_int), ("line", C.c_int64), ("id", C.c_int64), ("text", C.c_char * 512),
                ("message", C.c_char * 768)]


class ServerInfo(C.Structure):
    _fields_ = [("slots", C.c_int), ("preloaded_kernels", C.c_int), ("budget_bytes", C.c_double),
                ("pool_reserved_bytes", C.c_double), ("reservation", C.c_int)]


class LutDesc(C.Structure):
    _fields_ = [("n", C.c_int64), ("temperature", C.c_void_p), ("value", C.c_void_p)]


class MaterialDesc(C.Structure):
    _fields_ = [("name", C.c_char_p), ("youngs_modulus", LutDesc), ("poisson_ratio", LutDesc),
                ("thermal_expansion", LutDesc), ("reference_temperature", C.c_double)]


class AmplitudeDesc(C.Structure):
    _fields_ = [("n", C.c_int64), ("time", C.c_void_p), ("value", C.c_void_p), ("total_time", C.c_int),
                ("shift_x", C.c_double), ("shift_y", C.c_double)]


class RecordDesc(C.Structure):
    _fields_ = [("node_id", C.c_int64), ("dof", C.c_int32), ("amplitude", C.c_int32), ("value", C.c_double),
                ("origin_step", C.c_int64)]


class StepDesc(C.Structure):
    _fields_ = [("nlgeom", C.c_int), ("solver", C.c_int), ("increment", C.c_double * 4),
                ("max_increments", C.c_int64), ("n_loads", C.c_int64), ("loads", C.c_void_p),
                ("n_bcs", C.c_int64), ("bcs", C.c_void_p)]


class MeshDesc(C.Structure):
    _fields_ = [("n_nodes", C.c_int64), ("node_ids", C.c_void_p), ("xyz", C.c_void_p),
                ("n_c3d4", C.c_int64), ("c3d4_ids", C.c_void_p), ("c3d4_nodes", C.c_void_p),
                ("c3d4_material", C.c_void_p),
                ("n_c3d20", C.c_int64), ("c3d20_ids", C.c_void_p), ("c3d20_nodes", C.c_void_p),
                ("c3d20_material", C.c_void_p),
                ("n_materials", C.c_int), ("materials", C.c_void_p), ("n_amplitudes", C.c_int),
                ("amplitudes", C.c_void_p), ("n_steps", C.c_int), ("steps", C.c_void_p),
                ("default_temperature", C.c_double), ("n_initial_temperatures", C.c_int64),
                ("initial_temperature_ids", C.c_void_p), ("initial_temperatures", C.c_void_p)]


# name -> (restype, argtypes); every symbol of include/ferrix_b200.h
P = C.c_void_p
I64P = C.POINTER(C.c_int64)
# fx_increment_cb: int (*)(void* user, fx_model* model, int step_id, int inc_id, double global_time)
IncrementCallback = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double)

SIGNATURES = {
    "fx_default_solve_opts": (None, [C.POINTER(SolveOpts)]),
    "fx_ctx_create": (C.c_int, [C.c_int, C.POINTER(P)]),
    "fx_ctx_destroy": (None, [P]),
    "fx_ctx_last_error": (C.c_char_p, [P]),
    "fx_last_error_detail": (C.c_int, [P, C.POINTER(ErrorDetail)]),
    "fx_ctx_preloaded_kernels": (C.c_int, [P]),
    "fx_ctx_kernel_launches": (C.c_int64, [P]),
    "fx_ctx_stream": (C.c_void_p, [P]),
    "fx_model_from_inp": (C.c_int, [P, C.c_char_p, C.c_size_t, C.POINTER(P)]),
    "fx_model_from_arrays": (C.c_int, [P, C.POINTER(MeshDesc), C.POINTER(P)]),
    "fx_model_destroy": (None, [P]),
    "fx_model_sizes": (C.c_int, [P, I64P, I64P, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "fx_model_node_ids": (C.c_int, [P, P]),
    "fx_model_node_index": (C.c_int64, [P, C.c_int64]),
    "fx_model_set_default_temperature": (C.c_int, [P, C.c_double]),
    "fx_model_step_info": (C.c_int, [P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), P, I64P, I64P]),
    "fx_model_export": (C.c_int, [P, P, I64P, P, P, I64P, P, P]),
    "fx_model_step_records": (C.c_int, [P, C.c_int, C.c_int, P, P, P, P, P]),
    "fx_state_initialize": (C.c_int, [P]),
    "fx_state_get_displacements": (C.c_int, [P, P]),
    "fx_state_set_displacements": (C.c_int, [P, P]),
    "fx_state_get_temperatures": (C.c_int, [P, P, P]),
    "fx_state_set_temperatures": (C.c_int, [P, P, P]),
    "fx_step_solve": (C.c_int, [P, C.c_int, C.POINTER(SolveOpts), C.POINTER(StepStats)]),
    "fx_step_solve_cb": (C.c_int, [P, C.c_int, C.POINTER(SolveOpts), C.POINTER(StepStats), IncrementCallback, P]),
    "fx_vtk_series_init": (C.c_int, [C.c_char_p]),
    "fx_vtk_series_add": (C.c_int, [C.c_char_p, C.c_char_p, C.c_double]),
    "fx_vtk_series_finish": (C.c_int, [C.c_char_p]),
    "fx_assemble_csr": (C.c_int, [P, P, C.c_int, I64P, P, P, P, C.POINTER(C.c_double)]),
    "fx_internal_force": (C.c_int, [P, P, P, P]),
    "fx_thermal_force": (C.c_int, [P, P]),
    "fx_solve_csr": (C.c_int, [P, C.c_int64, P, P, P, P, P, C.POINTER(SolveOpts), C.POINTER(StepStats)]),
    "fx_model_drop_cache": (C.c_int, [P]),
    "fx_profile_spmv": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fx_profile_smoother": (C.c_int, [P, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fx_profile_assembly": (C.c_int, [P, C.c_int, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "fx_nodal_stress_strain": (C.c_int, [P, P, P]),
    "fx_write_vtk": (C.c_int, [P, C.c_char_p]),
    "fx_batch_solve": (C.c_int, [P, P, C.c_int, C.POINTER(SolveOpts), P, P]),
    "fx_default_server_opts": (None, [C.POINTER(ServerOpts)]),
    "fx_server_create": (C.c_int, [C.POINTER(ServerOpts), P]),
    "fx_server_submit": (C.c_int, [P, P, C.POINTER(C.c_int64)]),
    "fx_server_wait": (C.c_int, [P, C.c_int64, C.c_double, P, C.POINTER(RequestResult)]),
    "fx_server_get_info": (C.c_int, [P, C.POINTER(ServerInfo)]),
    "fx_server_destroy": (None, [P]),
    "fx_spmv_dot_noalloc": (C.c_int, [C.c_int, C.c_int64, P, P, P, P, P, P, P]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Loads the library (once). Raises OSError when it is missing."""
    global _lib
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"{path} not built; run `python -m ferrix_b200.build`")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def header_symbols(header: str) -> list:
    """Names of the functions declared in include/ferrix_b200.h."""
    import re
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fx_[a-z0-9_]+)\s*\(", text)))
