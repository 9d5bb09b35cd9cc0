// FP64 vector kernels of the Newton driver: residual assembly, BC-masked
// norms (static_step.rs:139-171) with a deterministic two-level reduction.
#include "common.hpp"
#include "kernels.hpp"

namespace fx {

__global__ void k_axpby(int64_t n, double a, const double* __restrict__ x, double b, const double* __restrict__ y,
                        double* __restrict__ out) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double xv = x ? x[i] : 0.0, yv = y ? y[i] : 0.0;
    out[i] = a * xv + b * yv;
}

void launch_axpby(int64_t n, double a, const double* x, double b, const double* y, double* out, cudaStream_t s) {
    if (n) FX_LAUNCH(k_axpby, (unsigned)((n + 255) / 256), 256, 0, s, n, a, x, b, y, out);
}

__global__ void k_scatter_set(int n, const int32_t* __restrict__ idx, const double* __restrict__ val,
                              double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[idx[i]] = val[i];
}

void launch_scatter_set(int n, const int32_t* idx, const double* val, double* out, cudaStream_t s) {
    if (n) FX_LAUNCH(k_scatter_set, (n + 255) / 256, 256, 0, s, n, idx, val, out);
}

__global__ void k_penalty_apply(int n, const int32_t* __restrict__ dof, const double* __restrict__ cnt,
                                const unsigned long long* __restrict__ maxdiag, const double* __restrict__ x,
                                double* __restrict__ out) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double md = __longlong_as_double((long long)*maxdiag);
    if (!(md > 0.0)) return;
    int d = dof[m];
    out[d] -= cnt[m] * (md * 1.0e6) * x[d];
}

void launch_penalty_apply(const BcView& bc, const unsigned long long* maxdiag, const double* x, double* out,
                          cudaStream_t s) {
    if (bc.n) FX_LAUNCH(k_penalty_apply, (bc.n + 255) / 256, 256, 0, s, bc.n, bc.dof, bc.cnt, maxdiag, x, out);
}

constexpr int kNormBlocks = 296;

__global__ void __launch_bounds__(256) k_masked_norms_partial(int64_t n, const double* __restrict__ a,
                                                              const double* __restrict__ b,
                                                              const uint8_t* __restrict__ mask,
                                                              double* __restrict__ partials) {
    double sa = 0.0, sb = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (mask && mask[i]) continue;
        double x = a[i], y = b[i];
        sa += x * x;
        sb += y * y;
    }
    __shared__ double sh[2][8];
    sa = warp_sum(sa);
    sb = warp_sum(sb);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        sh[0][w] = sa;
        sh[1][w] = sb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
            ta += sh[0][k];
            tb += sh[1][k];
        }
        partials[2 * blockIdx.x] = ta;
        partials[2 * blockIdx.x + 1] = tb;
    }
}

__global__ void k_sum_partials(int nb, const double* __restrict__ partials, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double ta = 0.0, tb = 0.0;
        for (int k = 0; k < nb; ++k) {
            ta += partials[2 * k];
            tb += partials[2 * k + 1];
        }
        out[0] = ta;
        out[1] = tb;
    }
}

void launch_masked_norms(int64_t n, const double* a, const double* b, const uint8_t* mask, double* partials,
                         double* out, cudaStream_t s) {
    FX_LAUNCH(k_masked_norms_partial, kNormBlocks, 256, 0, s, n, a, b, mask, partials);
    FX_LAUNCH(k_sum_partials, 1, 32, 0, s, kNormBlocks, partials, out);
}

// A kernel of this file's module (preload_kernels() loads all of the module's kernels).
const void* kernels_anchor_vectors() { return reinterpret_cast<const void*>(&k_axpby); }

}  // namespace fx
