// Scalar-CSR FP64 Jacobi PCG on the GPU: the algorithm of the reference's
// IterativeSolver (src/solver/solvers/iterative.rs:26-136) with its
// DiagonalPreconditioner (src/solver/preconditioner.rs:36-58): x0 = 0,
// z = D^-1 r (1/d when |d| > 1e-9, else 1), row-wise CSR SpMV.
//
// Two uses: (1) the plain-FP64 comparator of the BSR3 solvers (relative stop
// on ||r||_D / ||b||_D like them); (2) reference semantics for SOLVER=ITERATIVE
// decks (absolute stop sqrt(r.z) < tol, max_iter, ConvergenceError beyond).
// One warp per matrix row; the direction update p = z + beta p is fused into
// the SpMV gather as in the BSR3 solver; scalar reductions are fixed-order.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <algorithm>

#include <vector>

#include "pcg_csr.hpp"

namespace fx {

constexpr int kCsrThreads = 256;

__device__ __forceinline__ double csr_block_sum(double v, double* sh) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    v = warp_sum(v);
    if (l == 0) sh[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int j = 0; j < (int)(blockDim.x >> 5); ++j) t += sh[j];
    __syncthreads();
    return t;
}

// partial -> part[blockIdx.x]; the last CTA sums all partials in order and
// runs `fin(total)` in thread 0.
template <typename F>
__device__ __forceinline__ void csr_last_reduce(double v, double* part, int* counter, double* sh, F fin) {
    __shared__ int s_last;
    double t = csr_block_sum(v, sh);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = t;
        __threadfence();
        s_last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    double acc = 0.0;
    for (int c = threadIdx.x; c < (int)gridDim.x; c += blockDim.x) acc += __ldcg(part + c);
    double tot = csr_block_sum(acc, sh);
    if (threadIdx.x == 0) {
        *counter = 0;
        fin(tot);
    }
}

struct CsrDev {
    int64_t n;
    const int64_t* ip;
    const int32_t* ind;
    const double* val;
    const double* dinv;
    double *x, *r, *z, *p0, *p1, *q, *part, *scal;
    int* status;
    int* counter;
};

__global__ void __launch_bounds__(kCsrThreads) k_csr_spmv(CsrDev D, int parity) {
    __shared__ double sh[32];
    __shared__ int s_run;
    if (threadIdx.x == 0) s_run = *(volatile int*)D.status == kRun;
    __syncthreads();
    if (!s_run) return;
    const double beta = D.scal[kBeta];
    const double* pold = parity ? D.p1 : D.p0;
    double* pnew = parity ? D.p0 : D.p1;
    const int lane = threadIdx.x & 31;
    const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
    double dot = 0.0;
    // uniform trip count per warp: every lane reaches the shuffles
    for (int64_t row = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); row < D.n; row += warps) {
        double acc = 0.0;
        for (int64_t k = D.ip[row] + lane; k < D.ip[row + 1]; k += 32) {
            int j = __ldcs(D.ind + k);
            acc += __ldcs(D.val + k) * (D.z[j] + beta * pold[j]);
        }
        acc = warp_sum(acc);
        if (lane == 0) {
            double pi = D.z[row] + beta * pold[row];
            pnew[row] = pi;
            D.q[row] = acc;
            dot += pi * acc;
        }
    }
    csr_last_reduce(dot, D.part, D.counter, sh, [&](double pq) {
        D.scal[kPq] = pq;
        if (!(pq > 0.0) || !isfinite(pq)) {
            *D.status = kBreak;
            D.scal[kAlpha] = 0.0;
        } else {
            D.scal[kAlpha] = D.scal[kRz] / pq;
        }
    });
}

__global__ void __launch_bounds__(kCsrThreads) k_csr_update(CsrDev D, int parity) {
    __shared__ double sh[32];
    __shared__ int s_run;
    if (threadIdx.x == 0) s_run = *(volatile int*)D.status == kRun;
    __syncthreads();
    if (!s_run) return;
    const double alpha = D.scal[kAlpha];
    const double* p = parity ? D.p0 : D.p1;
    double rz = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D.n; i += (int64_t)gridDim.x * blockDim.x) {
        D.x[i] += alpha * p[i];
        double r = D.r[i] - alpha * D.q[i];
        D.r[i] = r;
        double z = D.dinv[i] * r;
        D.z[i] = z;
        rz += r * z;
    }
    csr_last_reduce(rz, D.part, D.counter + 1, sh, [&](double rzn) {
        double rzo = D.scal[kRz];
        D.scal[kRzOld] = rzo;
        D.scal[kRz] = rzn;
        D.scal[kBeta] = rzo > 0.0 ? rzn / rzo : 0.0;
        D.scal[kIters] += 1.0;
        if (!isfinite(rzn) || rzn < 0.0) *D.status = kBreak;
        else if (rzn <= D.scal[kThresh]) *D.status = kConv;
    });
}

// r = b, z = D^-1 b, rz; threshold = rtol^2 rz0 (relative) or tol^2 (absolute)
__global__ void __launch_bounds__(kCsrThreads) k_csr_init(CsrDev D, const double* b, double tol2, int absolute) {
    __shared__ double sh[32];
    double rz = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < D.n; i += (int64_t)gridDim.x * blockDim.x) {
        double r = b[i];
        D.r[i] = r;
        D.x[i] = 0.0;
        D.p0[i] = 0.0;
        double z = D.dinv[i] * r;
        D.z[i] = z;
        rz += r * z;
    }
    csr_last_reduce(rz, D.part, D.counter + 2, sh, [&](double rz0) {
        D.scal[kRz] = rz0;
        D.scal[kBnorm] = rz0;
        D.scal[kBeta] = 0.0;
        D.scal[kIters] = 0.0;
        D.scal[kThresh] = absolute ? tol2 : tol2 * rz0;
        *D.status = rz0 <= D.scal[kThresh] ? kConv : kRun;
    });
}

__global__ void k_csr_dinv(int64_t n, const int64_t* __restrict__ ip, const int32_t* __restrict__ ind,
                           const double* __restrict__ val, double* __restrict__ dinv) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double d = 0.0;
    for (int64_t k = ip[i]; k < ip[i + 1]; ++k)
        if (ind[k] == i) d += val[k];
    dinv[i] = fabs(d) > 1e-9 ? 1.0 / d : 1.0;
}

// BSR3 (FP64) -> scalar CSR with int32 columns; row 3i+r holds 3*cnt_i entries
__global__ void k_bsr_to_csr32(int64_t nblk, const int32_t* __restrict__ blk_row, const int32_t* __restrict__ row_ptr,
                               const int32_t* __restrict__ goff, const int32_t* __restrict__ cols,
                               const double* __restrict__ vals, int64_t* __restrict__ indptr,
                               int32_t* __restrict__ indices, double* __restrict__ data) {
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    int i = blk_row[b];
    int k = (int)(b - row_ptr[i]);
    int64_t g0 = goff[i];
    int ng = goff[i + 1] - (int)g0;
    int j = cols[4 * g0 + k];
    int cnt = row_ptr[i + 1] - row_ptr[i];
    for (int r = 0; r < 3; ++r) {
        int64_t o = 9 * (int64_t)row_ptr[i] + 3 * (int64_t)r * cnt + 3 * k;
        for (int c = 0; c < 3; ++c) {
            indices[o + c] = 3 * j + c;
            data[o + c] = vals[(g0 * 9 + (int64_t)(3 * r + c) * ng + k / 4) * 4 + (k & 3)];
        }
    }
}

__global__ void k_csr_indptr(int n_nodes, const int32_t* __restrict__ row_ptr, int64_t* __restrict__ indptr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    int64_t cnt = row_ptr[i + 1] - row_ptr[i];
    for (int r = 0; r < 3; ++r) indptr[3 * i + r] = 9 * (int64_t)row_ptr[i] + 3 * r * cnt;
}

void CsrSystem::from_bsr(const BsrStructure& S, const double* vals64, cudaStream_t s) {
    n = 3 * (int64_t)S.n_rows;
    nnz = 9 * S.n_blocks;
    ip.alloc(n + 1, s);
    ind.alloc(nnz, s);
    val.alloc(nnz, s);
    dinv.alloc(n, s);
    FX_CUDA_CHECK(cudaMemcpyAsync(ip.ptr + n, &nnz, sizeof(int64_t), cudaMemcpyHostToDevice, s));
    if (S.n_rows) FX_LAUNCH(k_csr_indptr, (S.n_rows + 255) / 256, 256, 0, s, S.n_rows, S.row_ptr.ptr, ip.ptr);
    if (S.n_blocks)
        FX_LAUNCH(k_bsr_to_csr32, (unsigned)((S.n_blocks + 255) / 256), 256, 0, s, S.n_blocks, S.blk_row.ptr,
                  S.row_ptr.ptr, S.goff.ptr, S.cols.ptr, vals64, ip.ptr, ind.ptr, val.ptr);
    FX_LAUNCH(k_csr_dinv, (unsigned)((n + 255) / 256), 256, 0, s, n, ip.ptr, ind.ptr, val.ptr, dinv.ptr);
}

void CsrSystem::from_host(int64_t rows, const int64_t* h_ip, const int64_t* h_ind, const double* h_val,
                          cudaStream_t s) {
    n = rows;
    nnz = h_ip[rows];
    std::vector<int32_t> ind32((size_t)nnz);
    for (int64_t k = 0; k < nnz; ++k) ind32[(size_t)k] = (int32_t)h_ind[k];
    ip.upload(h_ip, (size_t)n + 1, s);
    ind.upload(ind32, s);
    val.upload(h_val, (size_t)nnz, s);
    dinv.alloc((size_t)n, s);
    FX_LAUNCH(k_csr_dinv, (unsigned)((n + 255) / 256), 256, 0, s, n, ip.ptr, ind.ptr, val.ptr, dinv.ptr);
    stream_wait(s, "csr upload");  // the host column copy must outlive the transfer
}

int CsrPcg::solve(CsrSystem& A, const double* b, double* x, const PcgOptions& opt, bool absolute, cudaStream_t s,
                  int64_t* launches, long long* iters_out, double* relres_out) {
    const int64_t n = A.n;
    r_.alloc(n, s);
    z_.alloc(n, s);
    p0_.alloc(n, s);
    p1_.alloc(n, s);
    q_.alloc(n, s);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int grid = sms * 8;
    part_.alloc(grid, s);
    scal_.alloc(kNScal, s);
    scal_.zero(s);
    status_.alloc(1, s);
    counter_.alloc(4, s);
    counter_.zero(s);
    CsrDev D{n, A.ip.ptr, A.ind.ptr, A.val.ptr, A.dinv.ptr, x, r_.ptr, z_.ptr, p0_.ptr, p1_.ptr, q_.ptr, part_.ptr,
             scal_.ptr, status_.ptr, counter_.ptr};
    const double tol2 = opt.rtol * opt.rtol;
    FX_LAUNCH(k_csr_init, grid, kCsrThreads, 0, s, D, b, tol2, absolute ? 1 : 0);
    const int poll = std::max(2, opt.poll & ~1);
    cudaGraphExec_t gexec = nullptr;
    if (opt.graphs && !debug_sync()) {
        cudaGraph_t g;
        int64_t* saved = g_launch_counter;
        g_launch_counter = nullptr;
        FX_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < poll; ++k) {
            FX_LAUNCH(k_csr_spmv, grid, kCsrThreads, 0, s, D, k & 1);
            FX_LAUNCH(k_csr_update, grid, kCsrThreads, 0, s, D, k & 1);
        }
        FX_CUDA_CHECK(cudaStreamEndCapture(s, &g));
        g_launch_counter = saved;
        FX_CUDA_CHECK(cudaGraphInstantiate(&gexec, g, 0));
        cudaGraphDestroy(g);
    }
    double sc[kNScal];
    int st = kRun;
    int rc = FX_OK;
    while (true) {
        FX_CUDA_CHECK(cudaMemcpyAsync(sc, scal_.ptr, sizeof(sc), cudaMemcpyDeviceToHost, s));
        FX_CUDA_CHECK(cudaMemcpyAsync(&st, status_.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
        stream_wait(s, "csr pcg poll");
        if (st == kConv) break;
        if (st == kBreak) {
            rc = FX_NUMERICAL;
            break;
        }
        if (sc[kIters] >= opt.max_iter) {
            rc = FX_CONVERGENCE;
            break;
        }
        if (gexec) {
            FX_CUDA_CHECK(cudaGraphLaunch(gexec, s));
        } else {
            int64_t* saved = g_launch_counter;
            g_launch_counter = nullptr;
            for (int k = 0; k < poll; ++k) {
                FX_LAUNCH(k_csr_spmv, grid, kCsrThreads, 0, s, D, k & 1);
                FX_LAUNCH(k_csr_update, grid, kCsrThreads, 0, s, D, k & 1);
            }
            g_launch_counter = saved;
        }
        if (launches) *launches += 2 * (int64_t)poll;
    }
    if (gexec) cudaGraphExecDestroy(gexec);
    if (iters_out) *iters_out = (long long)sc[kIters];
    if (relres_out) *relres_out = sc[kBnorm] > 0 ? std::sqrt(std::max(0.0, sc[kRz]) / sc[kBnorm]) : 0.0;
    return rc;
}

// A kernel of this file's module (preload_kernels() loads all of the module's kernels).
const void* kernels_anchor_pcg_csr() { return reinterpret_cast<const void*>(&k_csr_spmv); }

}  // namespace fx
