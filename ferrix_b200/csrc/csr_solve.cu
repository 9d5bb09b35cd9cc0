// fx_solve_csr: the Solver::solve seam (src/solver/solvers/mod.rs:18-43).
// A caller that already holds the assembled FP64 CSR matrix (sprs CsMat in
// the reference) hands it over; the matrix is regrouped into 3x3 blocks
// (rows padded to a multiple of 3 with identity rows), solved with the same
// batched PCG as the static step, and the FP64 true residual uses the
// caller's CSR matrix itself (one warp per row).
#include <algorithm>
#include <cstring>

#include "engine.hpp"

namespace fx {

__global__ void k_csr_residual(int64_t n, const int64_t* __restrict__ ip, const int64_t* __restrict__ ind,
                               const double* __restrict__ val, const double* __restrict__ x,
                               const double* __restrict__ b, double* __restrict__ r) {
    int64_t row = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    int lane = threadIdx.x & 31;
    if (row >= n) return;
    double acc = 0.0;
    for (int64_t k = ip[row] + lane; k < ip[row + 1]; k += 32) acc += val[k] * x[ind[k]];
    acc = warp_sum(acc);
    if (lane == 0) r[row] = b[row] - acc;
}

constexpr int kStagnated = -1;

template <typename T>
static int solve_csr_t(fx_ctx* ctx, int64_t n, const int64_t* ip, const int64_t* ind, const double* data,
                       const double* b, double* x, const fx_solve_opts& o, fx_step_stats* st, double accept_rtol = 0.0) {
    cudaStream_t s = ctx->stream;
    const int64_t nb = (n + 2) / 3;  // block rows
    const int64_t n3 = 3 * nb;
    if (nb >= (int64_t(1) << 30)) fail(FX_INVALID_ARGUMENT, "matrix too large");
    // block pattern per block row (host)
    std::vector<std::vector<int32_t>> rowcols(nb);
    for (int64_t r = 0; r < n; ++r)
        for (int64_t k = ip[r]; k < ip[r + 1]; ++k) {
            if (ind[k] < 0 || ind[k] >= n) fail(FX_INVALID_ARGUMENT, "column index out of range");
            rowcols[r / 3].push_back((int32_t)(ind[k] / 3));
        }
    BsrStructure S;
    S.n_rows = (int)nb;
    std::vector<int32_t> row_ptr(nb + 1, 0), goff(nb + 1, 0), diag(nb, -1);
    for (int64_t i = 0; i < nb; ++i) {
        auto& v = rowcols[i];
        v.push_back((int32_t)i);  // always a diagonal block
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end()), v.end());
        row_ptr[i + 1] = row_ptr[i] + (int32_t)v.size();
        goff[i + 1] = goff[i] + (int32_t)((v.size() + 3) / 4);
        diag[i] = (int32_t)(std::lower_bound(v.begin(), v.end(), (int32_t)i) - v.begin());
    }
    const int64_t G = goff[nb];
    S.n_groups = G;
    S.n_blocks = row_ptr[nb];
    std::vector<int32_t> cols(4 * G);
    std::vector<T> vals(36 * G, T(0));
    for (int64_t i = 0; i < nb; ++i) {
        const auto& v = rowcols[i];
        const int ng = goff[i + 1] - goff[i];
        for (int g = 0; g < ng * 4; ++g) cols[4 * (int64_t)goff[i] + g] = g < (int)v.size() ? v[g] : (int32_t)i;
        for (int rr = 0; rr < 3; ++rr) {
            int64_t r = 3 * i + rr;
            if (r >= n) {  // identity padding row
                int64_t kk = diag[i];
                vals[((int64_t)goff[i] * 9 + (int64_t)(3 * rr + rr) * ng + kk / 4) * 4 + (kk & 3)] = T(1);
                continue;
            }
            for (int64_t k = ip[r]; k < ip[r + 1]; ++k) {
                int32_t j = (int32_t)(ind[k] / 3);
                int c = (int)(ind[k] % 3);
                int64_t kk = std::lower_bound(v.begin(), v.end(), j) - v.begin();
                int64_t at = ((int64_t)goff[i] * 9 + (int64_t)(3 * rr + c) * ng + kk / 4) * 4 + (kk & 3);
                vals[at] = (T)((double)vals[at] + data[k]);
            }
        }
    }
    S.row_ptr.upload(row_ptr, s);
    S.goff.upload(goff, s);
    S.cols.upload(cols, s);
    S.diag_k.upload(diag, s);
    DBuf<T> d_vals, d_minv;
    d_vals.upload(vals, s);
    d_minv.alloc(9 * nb, s);
    launch_block_jacobi<T>(S, d_vals.ptr, d_minv.ptr, s);
    // FP64 CSR on the device for the true residual (padded rows: identity)
    std::vector<int64_t> ipp(n3 + 1);
    std::memcpy(ipp.data(), ip, (n + 1) * sizeof(int64_t));
    std::vector<int64_t> indp(ind, ind + ip[n]);
    std::vector<double> datp(data, data + ip[n]);
    for (int64_t r = n; r < n3; ++r) {
        indp.push_back(r);
        datp.push_back(1.0);
        ipp[r + 1] = ipp[r] + 1;
    }
    DBuf<int64_t> d_ip, d_ind;
    DBuf<double> d_dat, d_b, d_x;
    d_ip.upload(ipp, s);
    d_ind.upload(indp, s);
    d_dat.upload(datp, s);
    std::vector<double> bp(b, b + n);
    bp.resize(n3, 0.0);
    d_b.upload(bp, s);
    d_x.alloc(n3, s);
    PcgSystem<T> sys;
    sys.S = &S;
    sys.vals = d_vals.ptr;
    sys.minv = d_minv.ptr;
    sys.b = d_b.ptr;
    sys.x = d_x.ptr;
    const int64_t* pip = d_ip.ptr;
    const int64_t* pind = d_ind.ptr;
    const double* pdat = d_dat.ptr;
    sys.residual64 = [n3, pip, pind, pdat](const double* xx, const double* bb, double* r, cudaStream_t ss) {
        FX_LAUNCH(k_csr_residual, (unsigned)((n3 * 32 + 255) / 256), 256, 0, ss, n3, pip, pind, pdat, xx, bb, r);
    };
    PcgOptions po;
    po.rtol = sizeof(T) == 4 ? o.rtol * kMixedBjResidualFactor : o.rtol;
    po.accept_rtol = accept_rtol;
    po.max_iter = o.max_iter;
    po.poll = o.poll_interval;
    po.reliable_delta = o.reliable_delta;
    po.graphs = o.use_graphs != 0;
    EventTimer t;
    t.start(s);
    std::vector<PcgSystem<T>*> v{&sys};
    PcgBatch<T> batch;
    batch.solve(v, po, s, &ctx->launches);
    double ms = t.stop_ms(s);
    std::vector<double> xp(n3);
    d_x.download(xp.data(), n3, s);
    FX_CUDA_CHECK(cudaStreamSynchronize(s));
    std::memcpy(x, xp.data(), n * sizeof(double));
    if (st) {
        *st = fx_step_stats{};
        st->linear_solves = 1;
        st->pcg_iterations = sys.iterations;
        st->reliable_updates = sys.replacements;
        st->last_linear_relres = sys.relres;
        st->t_pcg_ms = ms;
        st->t_total_ms = ms;
        st->bsr_blocks = S.n_blocks;
    }
    if (sys.status == FX_NUMERICAL) fail(FX_NUMERICAL, "Mathematical error: PCG breakdown (matrix not positive definite)");
    if (sys.stagnated) return kStagnated;  // FP32 refinement stopped improving: the caller finishes in FP64
    if (sys.status == FX_CONVERGENCE)
        fail(FX_CONVERGENCE, "Solver failed to converge: PCG did not converge after " + std::to_string(sys.iterations) +
                                 " iterations");
    return sys.status;
}

// Scalar-CSR Jacobi PCG on the caller's matrix as given: the reference
// IterativeSolver (absolute sqrt(r.z) < tol, iterative.rs:26-136) when
// `absolute`, else the plain FP64 PCG with the relative stopping test.
static int solve_csr_scalar(fx_ctx* ctx, int64_t n, const int64_t* ip, const int64_t* ind, const double* data,
                            const double* b, double* x, const fx_solve_opts& o, bool absolute, fx_step_stats* st) {
    cudaStream_t s = ctx->stream;
    if (n >= (int64_t(1) << 31)) fail(FX_INVALID_ARGUMENT, "matrix too large");
    for (int64_t k = 0; k < ip[n]; ++k)
        if (ind[k] < 0 || ind[k] >= n) fail(FX_INVALID_ARGUMENT, "column index out of range");
    CsrSystem A;
    A.from_host(n, ip, ind, data, s);
    DBuf<double> d_b, d_x;
    d_b.upload(b, (size_t)n, s);
    d_x.alloc((size_t)n, s);
    PcgOptions po;
    po.rtol = o.rtol;
    po.max_iter = o.max_iter;
    po.poll = o.poll_interval;
    po.graphs = o.use_graphs != 0;
    long long iters = 0;
    double relres = 0.0;
    EventTimer t;
    t.start(s);
    const int rc = ctx->pcgcsr.solve(A, d_b.ptr, d_x.ptr, po, absolute, s, &ctx->launches, &iters, &relres);
    const double ms = t.stop_ms(s);
    d_x.download(x, (size_t)n, s);
    FX_CUDA_CHECK(cudaStreamSynchronize(s));
    if (st) {
        *st = fx_step_stats{};
        st->linear_solves = 1;
        st->pcg_iterations = iters;
        st->last_linear_relres = relres;
        st->t_pcg_ms = ms;
        st->t_total_ms = ms;
    }
    if (rc == FX_NUMERICAL) fail(FX_NUMERICAL, "Mathematical error: PCG breakdown (matrix not positive definite)");
    if (rc == FX_CONVERGENCE)
        fail(FX_CONVERGENCE,
             "Solver failed to converge: PCG did not converge after " + std::to_string(o.max_iter) + " iterations");
    return rc;
}

// A kernel of this file's module (preload_kernels() loads all of the module's kernels).
const void* kernels_anchor_csr_solve() { return reinterpret_cast<const void*>(&k_csr_residual); }

}  // namespace fx

using namespace fx;

extern "C" int fx_solve_csr(fx_ctx* ctx, int64_t n, const int64_t* indptr, const int64_t* indices,
                            const double* data, const double* b, double* x, const fx_solve_opts* opts,
                            fx_step_stats* stats) {
    if (!ctx || n <= 0 || !indptr || !indices || !data || !b || !x) return FX_INVALID_ARGUMENT;
    fx_solve_opts o;
    if (opts) o = *opts;
    else fx_default_solve_opts(&o);
    try {
        FX_CUDA_CHECK(cudaSetDevice(ctx->device));
        int64_t* saved = g_launch_counter;
        g_launch_counter = &ctx->launches;
        struct R {
            int64_t* v;
            ~R() { g_launch_counter = v; }
        } r{saved};
        if (o.reference_iterative || o.precision == FX_PREC_FP64_CSR)
            return solve_csr_scalar(ctx, n, indptr, indices, data, b, x, o, o.reference_iterative != 0, stats);
        if (o.precision == FX_PREC_FP64) return solve_csr_t<double>(ctx, n, indptr, indices, data, b, x, o, stats);
        const int rc = solve_csr_t<float>(ctx, n, indptr, indices, data, b, x, o, stats);
        if (rc != kStagnated) return rc;
        fx_step_stats first{};
        if (stats) first = *stats;
        fx_solve_opts o64 = o;  // the mixed solve's FP64 target (accepted at the caller's rtol where it stalls)
        o64.rtol = o.rtol * kMixedBjResidualFactor;
        const int rc64 = solve_csr_t<double>(ctx, n, indptr, indices, data, b, x, o64, stats, o.rtol);
        if (stats) {
            stats->pcg_iterations += first.pcg_iterations;
            stats->reliable_updates += first.reliable_updates;
            stats->t_pcg_ms += first.t_pcg_ms;
            stats->t_total_ms += first.t_total_ms;
            stats->fp64_fallbacks = 1;
        }
        return rc64;
    } catch (const Error& e) {
        ctx->last_error = e.what();
        ctx->last_detail.set(e);
        thread_error().set(e);
        return e.status;
    } catch (const std::exception& e) {
        ctx->last_error = e.what();
        ctx->last_detail.set(FX_GENERIC, e.what());
        thread_error().set(FX_GENERIC, e.what());
        return FX_GENERIC;
    }
}
