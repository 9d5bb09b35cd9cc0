"""ORACLE — test infrastructure only (never imported by the product path).

ctypes binding of oracle_elem.c (FP64 element/material/assembly restatement
of FerriX src/solver/mesh_lib/elements/*.rs, src/solver/material.rs and
src/solver/assembler.rs). Builds the shared library on first use when gcc
is available; the prebuilt oracle/_build/liboracle_elem.so is used otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

from .inp import FerrixError, ModelArrays

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle_elem.c")
LIB = os.path.join(HERE, "_build", "liboracle_elem.so")


def build(force: bool = False) -> str:
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O3", "-march=x86-64-v3", "-fPIC", "-shared", "-o", LIB, SRC, "-lm"])
    return LIB


_lib = None


class _Mats(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("e_off", "e_len", "nu_off", "nu_len", "a_off", "a_len",
                                            "tref", "lut_t", "lut_v")]


def lib():
    global _lib
    if _lib is None:
        path = LIB
        if os.path.exists(SRC):
            try:
                path = build()
            except (OSError, subprocess.CalledProcessError):
                path = LIB
        _lib = C.CDLL(path)
        P = C.c_void_p
        _lib.or_lut_interp.restype = C.c_double
        _lib.or_lut_interp.argtypes = [P, P, C.c_int, C.c_double]
        _lib.or_shape_c3d20.argtypes = [C.c_double] * 3 + [P, P]
        _lib.or_shape_c3d4.argtypes = [C.c_double] * 3 + [P, P]
        _lib.or_gauss_points.argtypes = [C.c_int, P, P]
        _lib.or_element_stiffness.argtypes = [C.c_int, P, C.c_int, P, P, P, P, P]
        _lib.or_assemble.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P, P, P, P, P]
        _lib.or_internal_force.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P, P, P]
        _lib.or_thermal_force.argtypes = [C.c_int, C.c_int, P, P, P, P, P, P, P, P]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _mats(m: ModelArrays):
    keep = [m.mat_e_off, m.mat_e_len, m.mat_nu_off, m.mat_nu_len, m.mat_a_off, m.mat_a_len, m.mat_tref,
            m.lut_t, m.lut_v]
    s = _Mats(*[a.ctypes.data for a in keep])
    return s, keep


_RC = {1: ("NumericalError", "Singular Jacobian"),
       2: ("InvalidModelState", "No Young's Modulus / Poisson's Ratio definition"),
       3: ("InvalidModelState", "Element has no material assigned.")}


def _check(rc, bad, eids):
    if rc:
        kind, msg = _RC[rc]
        raise FerrixError(kind, f"{msg} (element {int(eids[bad.value])})")


def lut_interp(t, v, temp):
    t = np.ascontiguousarray(t, dtype=np.float64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    return lib().or_lut_interp(_p(t), _p(v), len(t), float(temp))


def shape_c3d20(x, y, z):
    N = np.zeros(20)
    dN = np.zeros(60)
    lib().or_shape_c3d20(x, y, z, _p(N), _p(dN))
    return N, dN.reshape(3, 20)


def gauss_points(npe):
    pts = np.zeros(81)
    w = np.zeros(27)
    n = lib().or_gauss_points(npe, _p(pts), _p(w))
    return pts[: 3 * n].reshape(n, 3), w[:n]


def element_stiffness(m: ModelArrays, npe: int, k: int, u=None, t_cur=None):
    eids, conn, mats = m.groups[npe]
    ms, keep = _mats(m)
    ce = np.ascontiguousarray(conn[k])
    Ke = np.zeros((3 * npe, 3 * npe))
    rc = lib().or_element_stiffness(npe, _p(ce), int(mats[k]), _p(m.xyz), _p(u), _p(t_cur), C.byref(ms), _p(Ke))
    if rc:
        raise FerrixError(*_RC[rc])
    return Ke


def assemble(m: ModelArrays, u=None, t_cur=None):
    """Assembler::assemble -> (CSR K with duplicates summed like TriMat::to_csr, maxdiag)."""
    n = m.xyz.shape[0] * 3
    cap = sum(len(g[0]) * (3 * npe) ** 2 for npe, g in m.groups.items())
    rows = np.empty(cap, dtype=np.int64)
    cols = np.empty(cap, dtype=np.int64)
    vals = np.empty(cap, dtype=np.float64)
    nt = C.c_int64(0)
    md = C.c_double(0.0)
    bad = C.c_int(0)
    ms, keep = _mats(m)
    for npe, (eids, conn, mats) in sorted(m.groups.items()):
        rc = lib().or_assemble(npe, len(eids), _p(conn), _p(mats), _p(m.xyz), _p(u), _p(t_cur), C.byref(ms),
                               _p(rows), _p(cols), _p(vals), C.byref(nt), C.byref(md), C.byref(bad))
        _check(rc, bad, eids)
    k = nt.value
    K = sp.csr_matrix((vals[:k], (rows[:k], cols[:k])), shape=(n, n))
    K.sum_duplicates()
    return K, md.value


def internal_force(m: ModelArrays, u, uconf, t_init, t_cur):
    f = np.zeros(m.xyz.shape[0] * 3)
    bad = C.c_int(0)
    ms, keep = _mats(m)
    for npe, (eids, conn, mats) in sorted(m.groups.items()):
        rc = lib().or_internal_force(npe, len(eids), _p(conn), _p(mats), _p(m.xyz), _p(u), _p(uconf),
                                     _p(t_init), _p(t_cur), C.byref(ms), _p(f), C.byref(bad))
        _check(rc, bad, eids)
    return f


def thermal_force(m: ModelArrays, t_init, t_cur):
    f = np.zeros(m.xyz.shape[0] * 3)
    bad = C.c_int(0)
    ms, keep = _mats(m)
    for npe, (eids, conn, mats) in sorted(m.groups.items()):
        rc = lib().or_thermal_force(npe, len(eids), _p(conn), _p(mats), _p(m.xyz), _p(t_init), _p(t_cur),
                                    C.byref(ms), _p(f), C.byref(bad))
        _check(rc, bad, eids)
    return f
