"""The allocation-free SpMV entry point against the library's existing ones.

fx_spmv_dot_noalloc serves callers that may not allocate device memory where
they run (graph capture, memory owned by a host application's allocator,
real-time loops): it uses only scratch compiled into the library. Here it
computes y = K u and u.K u for the stiffness K returned by fx_assemble_csr;
the existing fx_internal_force computes the same K u matrix-free on a linear
deck (no thermal strain), so the two must agree to the FP64 force tolerance
used elsewhere (1e-11 of the largest entry). Two calls in a row with
different vectors check that the shared scratch carries nothing over.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_spmv_dot_noalloc_matches_existing_entry_points():
    import torch
    import ferrix_b200 as fx
    from ferrix_b200 import _lib, decks

    lib = _lib.load()
    ctx = fx.Context(0)
    try:
        p = fx.Project.from_inp_text(decks.c3d20_box(3, 3, 8), ctx)
        st = fx.SolutionState(p.num_dofs, p.num_nodes)
        st.initialize(p)
        ip, ind, dat, _ = p.assemble_csr(None, fx.PREC_FP64)
        n = p.num_dofs
        dev = torch.device("cuda:0")
        d_ip = torch.from_numpy(ip).to(dev)
        d_ind = torch.from_numpy(ind).to(dev)
        d_dat = torch.from_numpy(dat).to(dev)
        d_y = torch.empty(n, dtype=torch.float64, device=dev)
        d_dot = torch.empty(1, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev)
        rng = np.random.default_rng(5)
        for call in range(2):
            u = rng.normal(scale=1e-2, size=n)
            d_u = torch.from_numpy(u).to(dev)
            torch.cuda.synchronize()
            rc = lib.fx_spmv_dot_noalloc(0, n, C.c_void_p(d_ip.data_ptr()), C.c_void_p(d_ind.data_ptr()),
                                         C.c_void_p(d_dat.data_ptr()), C.c_void_p(d_u.data_ptr()),
                                         C.c_void_p(d_y.data_ptr()), C.c_void_p(d_dot.data_ptr()),
                                         C.c_void_p(stream.cuda_stream))
            assert rc == 0
            torch.cuda.synchronize()
            y = d_y.cpu().numpy()
            f = p.internal_force(u)  # existing entry point: K u, matrix-free in FP64
            scale = np.abs(f).max()
            assert np.abs(y - f).max() <= 1e-11 * scale, call
            dot = float(d_dot.cpu().item())
            assert abs(dot - float(u @ f)) <= 1e-11 * abs(float(u @ f)), call
        # sizes beyond the compiled-in scratch are refused before any work is queued
        assert lib.fx_spmv_dot_noalloc(0, 524_289, C.c_void_p(d_ip.data_ptr()), C.c_void_p(d_ind.data_ptr()),
                                       C.c_void_p(d_dat.data_ptr()), C.c_void_p(d_u.data_ptr()),
                                       C.c_void_p(d_y.data_ptr()), C.c_void_p(d_dot.data_ptr()),
                                       C.c_void_p(stream.cuda_stream)) == 18
        # y written in place of x would be read by other rows: refused on the host, nothing launched
        assert lib.fx_spmv_dot_noalloc(0, n, C.c_void_p(d_ip.data_ptr()), C.c_void_p(d_ind.data_ptr()),
                                       C.c_void_p(d_dat.data_ptr()), C.c_void_p(d_u.data_ptr()),
                                       C.c_void_p(d_u.data_ptr() + 8), C.c_void_p(d_dot.data_ptr()),
                                       C.c_void_p(stream.cuda_stream)) == 18
        p.close()
    finally:
        ctx.close()
