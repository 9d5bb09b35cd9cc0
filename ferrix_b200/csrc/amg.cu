// Aggregation multigrid setup and V-cycle (see amg.hpp).
#include <cub/cub.cuh>

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstring>

#include <cuda_fp16.h>

#include "amg.hpp"
#include "coarse_row.cuh"

namespace fx {

namespace {

constexpr int kCoarseMaxDof = 1200;  // dense inverse at or below this size
constexpr int kMaxLevels = 8;

int bits_for(int64_t n) {
    int b = 1;
    while ((int64_t(1) << b) < n) ++b;
    return b;
}

template <typename Op>
void cub_call(Op op, DBuf<uint8_t>& tmp, cudaStream_t s) {
    size_t bytes = 0;
    FX_CUDA_CHECK(op(nullptr, bytes));
    if (tmp.n < bytes) tmp.alloc(bytes, s);
    FX_CUDA_CHECK(op(tmp.ptr, bytes));
}

// ------------------------------------------------------------------ aggregation

// org[0..2] = componentwise minimum of the n points c (one CTA)
__global__ void __launch_bounds__(1024) k_min3(int n, const double* __restrict__ c, double* __restrict__ org) {
    __shared__ double sh[3][32];
    double m[3] = {1e300, 1e300, 1e300};
    for (int i = threadIdx.x; i < n; i += blockDim.x)
#pragma unroll
        for (int d = 0; d < 3; ++d) m[d] = fmin(m[d], c[3 * (int64_t)i + d]);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        for (int o = 16; o > 0; o >>= 1) m[d] = fmin(m[d], __shfl_xor_sync(0xffffffffu, m[d], o));
        if (lane == 0) sh[d][w] = m[d];
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double v = 1e300;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v = fmin(v, sh[threadIdx.x][k]);
        org[threadIdx.x] = v;
    }
}

__global__ void k_cell_keys(int n, const double* __restrict__ c, const double* __restrict__ org, double inv_cell,
                            uint64_t* __restrict__ keys, int32_t* __restrict__ ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double ox = org[0], oy = org[1], oz = org[2];
    auto cell = [&](double v, double o) {
        double f = floor((v - o) * inv_cell);
        f = f < 0.0 ? 0.0 : (f > 2097151.0 ? 2097151.0 : f);
        return (uint64_t)f;
    };
    keys[i] = cell(c[3 * i], ox) | (cell(c[3 * i + 1], oy) << 21) | (cell(c[3 * i + 2], oz) << 42);
    ids[i] = i;
}

__global__ void k_heads64(int n, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

// agg[node] = rank of its cell; agg_ptr[a] = first sorted position of aggregate a
__global__ void k_agg_assign(int n, const int32_t* __restrict__ rank1, const int32_t* __restrict__ head,
                             const int32_t* __restrict__ sorted_ids, int32_t* __restrict__ agg,
                             int32_t* __restrict__ agg_ptr) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int a = rank1[i] - 1;
    agg[sorted_ids[i]] = a;
    if (head[i]) agg_ptr[a] = i;
}

__global__ void k_agg_centroid(int na, const int32_t* __restrict__ ptr, const int32_t* __restrict__ nodes,
                               const double* __restrict__ c, double* __restrict__ cent) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    double s0 = 0, s1 = 0, s2 = 0;
    int m = ptr[a + 1] - ptr[a];
    for (int k = ptr[a]; k < ptr[a + 1]; ++k) {
        int j = nodes[k];
        s0 += c[3 * j];
        s1 += c[3 * j + 1];
        s2 += c[3 * j + 2];
    }
    cent[3 * a] = s0 / m;
    cent[3 * a + 1] = s1 / m;
    cent[3 * a + 2] = s2 / m;
}

// Near-null-space row (d, col) of a member: level 0 rigid-body modes about the
// centroid; above, the member's R block from the previous QR.
__device__ __forceinline__ double nullspace_row(int bs, int j, int d, int col, const double* c, const double* cent,
                                                int a, const double* Rprev) {
    if (bs == 6) return Rprev[(size_t)j * 36 + d * 6 + col];
    double x = c[3 * j] - cent[3 * a], y = c[3 * j + 1] - cent[3 * a + 1], z = c[3 * j + 2] - cent[3 * a + 2];
    if (col < 3) return d == col ? 1.0 : 0.0;
    if (col == 3) return d == 0 ? -y : (d == 1 ? x : 0.0);   // rotation about z
    if (col == 4) return d == 1 ? -z : (d == 2 ? y : 0.0);   // rotation about x
    return d == 0 ? z : (d == 2 ? -x : 0.0);                  // rotation about y
}

// One warp per aggregate: Q (rows of the members, in place) and R (6x6).
__global__ void k_agg_qr(int na, const int32_t* __restrict__ ptr, const int32_t* __restrict__ nodes, int bs,
                         const double* __restrict__ c, const double* __restrict__ cent,
                         const double* __restrict__ Rprev, double* __restrict__ Q, double* __restrict__ Rnext) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= na) return;  // warp-uniform
    const int a = warp;
    const int p0 = ptr[a], m = ptr[a + 1] - ptr[a];
    const int rows = m * bs;
    auto qidx = [&](int r, int col) {
        int j = nodes[p0 + r / bs];
        return ((size_t)j * bs + (r % bs)) * 6 + col;
    };
    for (int r = lane; r < rows; r += 32) {
        int j = nodes[p0 + r / bs];
        for (int col = 0; col < 6; ++col) Q[qidx(r, col)] = nullspace_row(bs, j, r % bs, col, c, cent, a, Rprev);
    }
    __syncwarp();
    double R[36];
    for (int k = 0; k < 36; ++k) R[k] = 0.0;
    for (int col = 0; col < 6; ++col) {
        double n0 = 0.0;
        for (int r = lane; r < rows; r += 32) {
            double v = Q[qidx(r, col)];
            n0 += v * v;
        }
        n0 = sqrt(warp_sum(n0));
        for (int pass = 0; pass < 2; ++pass)
            for (int k = 0; k < col; ++k) {
                double dot = 0.0;
                for (int r = lane; r < rows; r += 32) dot += Q[qidx(r, k)] * Q[qidx(r, col)];
                dot = warp_sum(dot);
                R[k * 6 + col] += dot;
                for (int r = lane; r < rows; r += 32) Q[qidx(r, col)] -= dot * Q[qidx(r, k)];
                __syncwarp();
            }
        double nr = 0.0;
        for (int r = lane; r < rows; r += 32) {
            double v = Q[qidx(r, col)];
            nr += v * v;
        }
        nr = sqrt(warp_sum(nr));
        const bool keep = n0 > 0.0 && nr > 1e-10 * n0;
        R[col * 6 + col] = keep ? nr : 0.0;
        for (int r = lane; r < rows; r += 32) Q[qidx(r, col)] = keep ? Q[qidx(r, col)] / nr : 0.0;
        __syncwarp();
    }
    if (lane == 0)
        for (int k = 0; k < 36; ++k) Rnext[(size_t)a * 36 + k] = R[k];
}

// ------------------------------------------------------------------ Galerkin coarse matrix

// fine block (row i, col j) and its values at level 0 (planar BSR3) or above (row-major bs x bs)
struct FineView {
    int bs;
    const int32_t* blk_row;  // per block
    const int32_t* blk_col;  // per block (coarse levels); level 0 uses planar cols
    const double* vals;
    // level 0 planar
    const int32_t* row_ptr;
    const int32_t* goff;
    const int32_t* cols4;
    __device__ __forceinline__ int col(int64_t b, int i) const {
        if (bs == 6) return blk_col[b];
        int k = (int)(b - row_ptr[i]);
        return cols4[4 * (int64_t)goff[i] + k];
    }
    template <int BS>
    __device__ __forceinline__ void load(int64_t b, int i, double* v) const {
        if (BS == 6) {
#pragma unroll
            for (int k = 0; k < 36; ++k) v[k] = vals[b * 36 + k];
        } else {
            const int k = (int)(b - row_ptr[i]);
            const int64_t g0 = goff[i];
            const int ng = goff[i + 1] - (int)g0;
            const double* base = vals + (g0 * 9 + k / 4) * 4 + (k & 3);
#pragma unroll
            for (int t = 0; t < 9; ++t) v[t] = base[(int64_t)t * ng * 4];
        }
    }
};

__global__ void k_coarse_keys(int64_t nb, FineView F, const int32_t* __restrict__ agg, int nbits,
                              uint64_t* __restrict__ keys, int64_t* __restrict__ ids) {
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nb) return;
    int i = F.blk_row[b];
    int j = F.col(b, i);
    keys[b] = ((uint64_t)agg[i] << nbits) | (uint64_t)agg[j];
    ids[b] = b;
}

__global__ void k_heads_u64(int64_t n, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void k_coarse_blocks(int64_t n, const uint64_t* __restrict__ keys, const int32_t* __restrict__ bid,
                                int nbits, int64_t* __restrict__ seg, int32_t* __restrict__ crow,
                                int32_t* __restrict__ ccol, int32_t* __restrict__ cnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0 || keys[i] != keys[i - 1]) {
        int b = bid[i] - 1;
        seg[b] = i;
        int I = (int)(keys[i] >> nbits);
        crow[b] = I;
        ccol[b] = (int)(keys[i] & ((uint64_t(1) << nbits) - 1));
        atomicAdd(&cnt[I], 1);
    }
}

// Coarse block = sum over its fine blocks of Q_i^T A_ij Q_j. One warp per coarse
// block; lane k takes the k-th contiguous slice of the block's sorted fine blocks
// (row-major within a key, so each row's blocks are adjacent): T = sum_j A_ij Q_j
// is accumulated per row and Q_i^T T added when the row changes. The 36 sums are
// combined by a fixed butterfly: no atomics, the result does not depend on timing.
template <int BS>
__global__ void __launch_bounds__(128) k_galerkin(int64_t ncb, const int64_t* __restrict__ seg,
                                                  const int64_t* __restrict__ sorted_b, FineView F,
                                                  const double* __restrict__ Q, double* __restrict__ cvals) {
    const int64_t cb = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (cb >= ncb) return;  // warp-uniform
    const int64_t s0 = seg[cb], len = seg[cb + 1] - s0;
    const int64_t per = (len + 31) / 32;
    const int64_t a = s0 + lane * per, e = min(a + per, s0 + len);
    double acc[36];
#pragma unroll
    for (int k = 0; k < 36; ++k) acc[k] = 0.0;
    double T[BS * 6];
    int cur = -1;
    auto flush = [&]() {
        const double* Qi = Q + (size_t)cur * BS * 6;
#pragma unroll
        for (int k = 0; k < BS; ++k) {
            double q[6];
#pragma unroll
            for (int r = 0; r < 6; ++r) q[r] = Qi[k * 6 + r];
#pragma unroll
            for (int r = 0; r < 6; ++r)
#pragma unroll
                for (int c = 0; c < 6; ++c) acc[r * 6 + c] += q[r] * T[k * 6 + c];
        }
    };
    for (int64_t s = a; s < e; ++s) {
        const int64_t b = sorted_b[s];
        const int i = F.blk_row[b];
        const int j = F.col(b, i);
        if (i != cur) {
            if (cur >= 0) flush();
            cur = i;
#pragma unroll
            for (int k = 0; k < BS * 6; ++k) T[k] = 0.0;
        }
        const double* Qj = Q + (size_t)j * BS * 6;
        double v[BS * BS];
        F.load<BS>(b, i, v);
#pragma unroll
        for (int k = 0; k < BS; ++k) {
            double q[6];
#pragma unroll
            for (int c = 0; c < 6; ++c) q[c] = Qj[k * 6 + c];
#pragma unroll
            for (int r = 0; r < BS; ++r)
#pragma unroll
                for (int c = 0; c < 6; ++c) T[r * 6 + c] += v[r * BS + k] * q[c];
        }
    }
    if (cur >= 0) flush();
#pragma unroll
    for (int k = 0; k < 36; ++k) {
        const double t = warp_sum(acc[k]);
        if (lane == 0) cvals[cb * 36 + k] = t;
    }
}

__global__ void k_expand_rows(int n, const int32_t* __restrict__ row_ptr, int32_t* __restrict__ blk_row) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int b = row_ptr[i]; b < row_ptr[i + 1]; ++b) blk_row[b] = i;
}

// block inverse of the 6x6 diagonal blocks; DOFs with a vanishing pivot (rank-
// deficient aggregates) get zero rows/columns in the inverse
__global__ void k_block_inv6(int n, const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ cols,
                             const double* __restrict__ vals, double* __restrict__ dinv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double A[36], X[36];
    for (int k = 0; k < 36; ++k) {
        A[k] = 0.0;
        X[k] = 0.0;
    }
    for (int b = row_ptr[i]; b < row_ptr[i + 1]; ++b)
        if (cols[b] == i)
            for (int k = 0; k < 36; ++k) A[k] = vals[(int64_t)b * 36 + k];
    double dmax = 0.0;
    for (int k = 0; k < 6; ++k) dmax = fmax(dmax, fabs(A[k * 7]));
    bool dead[6];
    for (int k = 0; k < 6; ++k) {
        dead[k] = !(fabs(A[k * 7]) > 1e-12 * dmax);
        if (dead[k]) {
            for (int t = 0; t < 6; ++t) A[k * 6 + t] = A[t * 6 + k] = 0.0;
            A[k * 7] = 1.0;
        }
        X[k * 7] = 1.0;
    }
    // Gauss-Jordan (SPD block, no pivoting)
    for (int k = 0; k < 6; ++k) {
        double p = A[k * 7];
        if (p == 0.0) p = 1.0;
        double ip = 1.0 / p;
        for (int t = 0; t < 6; ++t) {
            A[k * 6 + t] *= ip;
            X[k * 6 + t] *= ip;
        }
        for (int r = 0; r < 6; ++r)
            if (r != k) {
                double f = A[r * 6 + k];
                for (int t = 0; t < 6; ++t) {
                    A[r * 6 + t] -= f * A[k * 6 + t];
                    X[r * 6 + t] -= f * X[k * 6 + t];
                }
            }
    }
    for (int k = 0; k < 6; ++k)
        if (dead[k])
            for (int t = 0; t < 6; ++t) X[k * 6 + t] = X[t * 6 + k] = 0.0;
    for (int k = 0; k < 36; ++k) dinv[(int64_t)i * 36 + k] = X[k];
}

// ------------------------------------------------------------------ level operators

// coarse levels: row-major 6x6 blocks, one warp per block row
__global__ void __launch_bounds__(256) k_ln_spmv(int n, const int32_t* __restrict__ row_ptr,
                                                 const int32_t* __restrict__ cols, const double* __restrict__ vals,
                                                 const double* __restrict__ x, const double* __restrict__ b,
                                                 double* __restrict__ y) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;  // warp-uniform
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int blk = row_ptr[warp] + lane; blk < row_ptr[warp + 1]; blk += 32) {
        const double* v = vals + (int64_t)blk * 36;
        const double* xx = x + 6 * (int64_t)cols[blk];
        double xv[6];
        for (int c = 0; c < 6; ++c) xv[c] = xx[c];
        for (int r = 0; r < 6; ++r) {
            double t = 0.0;
            for (int c = 0; c < 6; ++c) t += v[r * 6 + c] * xv[c];
            acc[r] += t;
        }
    }
    for (int r = 0; r < 6; ++r) acc[r] = warp_sum(acc[r]);
    if (lane < 6) {
        double v = acc[0];
        for (int r = 1; r < 6; ++r)
            if (lane == r) v = acc[r];
        y[6 * (int64_t)warp + lane] = b ? b[6 * (int64_t)warp + lane] - v : v;
    }
}

// Chebyshev start: d = D^-1 r / theta; x = (zero ? 0 : x) + d
__global__ void k_cheb_init(int n, int bs, const double* __restrict__ dinv, const double* __restrict__ r,
                            double* __restrict__ d, double* __restrict__ x, double inv_theta, int zero) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* Di = dinv + (int64_t)i * bs * bs;
    const double* ri = r + (int64_t)i * bs;
    for (int k = 0; k < bs; ++k) {
        double t = 0.0;
        for (int c = 0; c < bs; ++c) t += Di[k * bs + c] * ri[c];
        t *= inv_theta;
        d[(int64_t)i * bs + k] = t;
        x[(int64_t)i * bs + k] = zero ? t : x[(int64_t)i * bs + k] + t;
    }
}

// bc = Q^T rf per aggregate: one warp per aggregate, lanes over member rows
// Coarse Chebyshev start fused into the restriction (cs.dinv != null): with
// b = R r the first pre-smoothing step of the coarse level from x = 0 is
// d = c2 D^-1 b, xs = d, r = b (what k_cheb_start does there).
// b_c = Q^T r_f, warp per aggregate; each lane's rows are loaded four at a time
// before they are accumulated (in the same order as one row at a time).
__global__ void k_restrict(int na, const int32_t* __restrict__ ptr, const int32_t* __restrict__ nodes, int bs,
                           const double* __restrict__ Q, const double* __restrict__ rf, double* __restrict__ bc,
                           CoarseStart cs) {
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (a >= na) return;  // warp-uniform
    const int p0 = ptr[a], rows = (ptr[a + 1] - p0) * bs;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int r0 = lane; r0 < rows; r0 += 128) {
        double rv[4], qv[4][6];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int r = r0 + 32 * u;
            rv[u] = 0.0;
            if (r < rows) {
                const int j = nodes[p0 + r / bs];
                const int64_t row = (int64_t)j * bs + r % bs;
                rv[u] = rf[row];
#pragma unroll
                for (int c = 0; c < 6; ++c) qv[u][c] = Q[row * 6 + c];
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (r0 + 32 * u < rows) {
#pragma unroll
                for (int c = 0; c < 6; ++c) acc[c] += qv[u][c] * rv[u];
            }
    }
    double t[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) t[c] = warp_sum(acc[c]);  // every lane holds the sums
    if (lane < 6) {
        const int64_t o = (int64_t)a * 6 + lane;
        double tk = t[0];
#pragma unroll
        for (int c = 1; c < 6; ++c)
            if (lane == c) tk = t[c];
        bc[o] = tk;
        if (cs.dinv) {
            const double* Di = cs.dinv + (int64_t)a * 36 + lane * 6;
            double v = 0.0;
#pragma unroll
            for (int j = 0; j < 6; ++j) v += Di[j] * t[j];
            v *= cs.c2;
            cs.d[o] = v;
            cs.xs[o] = v;
            cs.r[o] = tk;
        }
    }
}

__global__ void k_prolong(int ndof, int bs, const int32_t* __restrict__ agg, const double* __restrict__ Q,
                          const double* __restrict__ xc, double* __restrict__ xf, double alpha) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ndof) return;
    int j = k / bs;
    const double* q = Q + (int64_t)k * 6;
    const double* x = xc + (int64_t)agg[j] * 6;
    double t = 0.0;
    for (int c = 0; c < 6; ++c) t += q[c] * x[c];
    xf[k] += alpha * t;
}

// ------------------------------------------------------------------ coarsest level

__global__ void k_dense_from_bsr(int n, const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ cols,
                                 const double* __restrict__ vals, double* __restrict__ A) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int nd = 6 * n;
    for (int b = row_ptr[i]; b < row_ptr[i + 1]; ++b)
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c)
                A[(int64_t)(6 * i + r) * nd + 6 * cols[b] + c] = vals[(int64_t)b * 36 + r * 6 + c];
}

// Coarsest level: in-place blocked Gauss-Jordan inverse of the dense SPD matrix
// (no pivoting), panels of kPanel pivots. Per panel K: the pivot block is
// inverted by one CTA (P), the panel rows become P A[K, j], every other row i
// gets A[i, j] -= A[i, K] (P A[K, j]) and A[i, K] = -A[i, K] P. DOFs with a
// vanishing diagonal are decoupled first and get zero rows/columns in the inverse.
constexpr int kPanel = 32;

__global__ void __launch_bounds__(1024) k_dense_decouple(int nd, double* __restrict__ A, uint8_t* __restrict__ dead,
                                                         double* __restrict__ diag) {
    __shared__ double s_red[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    double m = 0.0;
    for (int k = threadIdx.x; k < nd; k += blockDim.x) m = fmax(m, fabs(A[(int64_t)k * nd + k]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) s_red[warp] = m;
    __syncthreads();
    double dmax = 0.0;
    for (int w = 0; w < nw; ++w) dmax = fmax(dmax, s_red[w]);
    for (int k = threadIdx.x; k < nd; k += blockDim.x) dead[k] = !(fabs(A[(int64_t)k * nd + k]) > 1e-12 * dmax);
    __syncthreads();
    for (int r = warp; r < nd; r += nw)
        for (int c = lane; c < nd; c += 32)
            if (dead[r] || dead[c]) A[(int64_t)r * nd + c] = (r == c) ? 1.0 : 0.0;
    __syncthreads();
    for (int k = threadIdx.x; k < nd; k += blockDim.x) diag[k] = A[(int64_t)k * nd + k];  // before elimination
}

// A pivot of the elimination below kSingularPivot of its row's original
// diagonal means the coarse operator is singular: the rigid-body modes of an
// insufficiently constrained model lie in the coarse space (an SPD coarse
// matrix keeps each pivot at or above 1 / cond of the original diagonal).
constexpr double kSingularPivot = 1e-12;

// P = inverse of the pivot block A[k0:k0+b, k0:k0+b], written in place (one CTA, 32 warps);
// *singular |= 1 when a pivot is not above kSingularPivot times its original diagonal
__global__ void __launch_bounds__(1024) k_panel_inverse(int nd, int k0, int b, double* __restrict__ A,
                                                        const double* __restrict__ diag, int* __restrict__ singular) {
    __shared__ double S[kPanel][kPanel + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    S[w][lane] = (w < b && lane < b) ? A[(int64_t)(k0 + w) * nd + k0 + lane] : (w == lane ? 1.0 : 0.0);
    __syncthreads();
    for (int t = 0; t < b; ++t) {
        if (threadIdx.x == 0 && !(S[t][t] > kSingularPivot * diag[k0 + t])) *singular = 1;
        const double ip = 1.0 / S[t][t];
        __syncthreads();
        if (w == t && lane != t) S[t][lane] *= ip;
        __syncthreads();
        const double f = S[w][t];
        __syncthreads();
        if (w != t) {
            if (lane != t) S[w][lane] -= f * S[t][lane];
            else S[w][t] = -f * ip;
        }
        __syncthreads();
        if (threadIdx.x == 0) S[t][t] = ip;
        __syncthreads();
    }
    if (w < b && lane < b) A[(int64_t)(k0 + w) * nd + k0 + lane] = S[w][lane];
}

__device__ __forceinline__ void load_panel(int nd, int k0, int b, const double* A, double (*P)[kPanel]) {
    for (int e = threadIdx.x; e < kPanel * kPanel; e += blockDim.x) {
        const int r = e / kPanel, c = e % kPanel;
        P[r][c] = (r < b && c < b) ? A[(int64_t)(k0 + r) * nd + k0 + c] : 0.0;
    }
    __syncthreads();
}

// panel rows: A[K, j] = P A[K, j] for every column j outside K (one thread per column)
__global__ void __launch_bounds__(128) k_panel_rows(int nd, int k0, int b, double* __restrict__ A) {
    __shared__ double P[kPanel][kPanel];
    load_panel(nd, k0, b, A, P);
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nd || (j >= k0 && j < k0 + b)) return;
    double col[kPanel];
#pragma unroll
    for (int t = 0; t < kPanel; ++t) col[t] = t < b ? A[(int64_t)(k0 + t) * nd + j] : 0.0;
    for (int r = 0; r < b; ++r) {
        double s = 0.0;
#pragma unroll
        for (int t = 0; t < kPanel; ++t) s += P[r][t] * col[t];
        A[(int64_t)(k0 + r) * nd + j] = s;
    }
}

// A[i, j] -= A[i, K] A[K, j] for every i, j outside K: one 32 x 32 tile per CTA,
// both factors staged in shared memory (k0 is a multiple of 32, so the panel's
// rows and columns are whole tiles, which are skipped)
__global__ void __launch_bounds__(256) k_panel_update(int nd, int k0, int b, double* __restrict__ A) {
    __shared__ double Lt[32][33];  // A[i0 + r, k0 + t]
    __shared__ double Rt[32][33];  // A[k0 + t, j0 + c]
    const int i0 = blockIdx.y * 32, j0 = blockIdx.x * 32;
    if (i0 == k0 || j0 == k0) return;  // CTA-uniform
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (int r = ty; r < 32; r += 8) {
        const int i = i0 + r, j = j0 + tx;
        Lt[r][tx] = (i < nd && tx < b) ? A[(int64_t)i * nd + k0 + tx] : 0.0;
        Rt[r][tx] = (r < b && j < nd) ? A[(int64_t)(k0 + r) * nd + j] : 0.0;
    }
    __syncthreads();
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int t = 0; t < 32; ++t) {
        const double rv = Rt[t][tx];
#pragma unroll
        for (int u = 0; u < 4; ++u) acc[u] += Lt[ty + 8 * u][t] * rv;
    }
    const int j = j0 + tx;
    if (j >= nd) return;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int i = i0 + ty + 8 * u;
        if (i < nd) A[(int64_t)i * nd + j] -= acc[u];
    }
}

// after the update: A[i, K] = -A[i, K] P for every row i outside K (one warp per row)
__global__ void __launch_bounds__(256) k_panel_cols(int nd, int k0, int b, double* __restrict__ A) {
    __shared__ double P[kPanel][kPanel];
    load_panel(nd, k0, b, A, P);
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (i >= nd || (i >= k0 && i < k0 + b)) return;  // warp-uniform
    double* Ai = A + (int64_t)i * nd;
    const double a = lane < b ? Ai[k0 + lane] : 0.0;
    double acc = 0.0;
    for (int s = 0; s < b; ++s) acc += __shfl_sync(0xffffffffu, a, s) * P[s][lane];
    if (lane < b) Ai[k0 + lane] = -acc;
}

__global__ void __launch_bounds__(256) k_dense_zero_dead(int nd, double* __restrict__ A,
                                                         const uint8_t* __restrict__ dead) {
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (r >= nd) return;
    for (int c = lane; c < nd; c += 32)
        if (dead[r] || dead[c]) A[(int64_t)r * nd + c] = 0.0;
}

__global__ void k_dense_matvec(int nd, const double* __restrict__ A, const double* __restrict__ x,
                               double* __restrict__ y) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= nd) return;
    const double t = dense_row_dot<false>(A + (int64_t)warp * nd, x, nd, lane);
    if (lane == 0) y[warp] = t;
}

// deterministic dot product of two vectors into out[0] (two launches)
__global__ void k_dot_part(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ part) {
    __shared__ double sh[8];
    double t = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        t += a[i] * b[i];
    t = warp_sum(t);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
        part[blockIdx.x] = s;
    }
}

__global__ void k_sum_part(int nb, const double* __restrict__ part, double* __restrict__ out) {
    double t = 0.0;
    for (int k = threadIdx.x; k < nb; k += 32) t += part[k];
    t = warp_sum(t);
    if (threadIdx.x == 0) *out = t;
}

// x = d / sqrt(*nrm2), the norm read on the device
// x = d / |d| (x may be d itself)
__global__ void k_normalize(int64_t n, const double* __restrict__ nrm2, const double* d, double* x) {
    const double v = *nrm2;
    const double inv = v > 0.0 ? 1.0 / sqrt(v) : 1.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        x[i] = d[i] * inv;
}

__global__ void k_fill_hash(int64_t n, double* __restrict__ v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    v[i] = (double)(h & 0xFFFFF) / 1048576.0 + 0.5;
}


unsigned grid_for(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// ---- outer PCG scalars: S[0] r.z, S[1] p.q, S[2] r.D^-1 r, S[3] b.D^-1 b, S[4] beta, S[5] alpha, S[6] breakdown
__global__ void k_fin(int nb, const double* __restrict__ part, double* __restrict__ S, int what) {
    double t = 0.0;  // fixed lane assignment and tree: deterministic
    for (int k = threadIdx.x; k < nb; k += 32) t += part[k];
    t = warp_sum(t);
    if (threadIdx.x != 0) return;
    if (what == 0) {  // p.q -> alpha
        S[1] = t;
        if (!(t > 0.0) || !isfinite(t)) {
            S[6] = 1.0;
            S[5] = 0.0;
        } else {
            S[5] = S[0] / t;
        }
    } else if (what == 1) {  // r.D^-1 r
        S[2] = t;
    } else if (what == 2) {  // r.z -> beta
        S[4] = S[0] > 0.0 ? t / S[0] : 0.0;
        S[0] = t;
    } else if (what == 3) {  // initial: r.z and b.D^-1 b
        S[0] = t;
        S[4] = 0.0;
    }
}

// partial r . D^-1 r without the update (start of the solve)
__global__ void k_rdr_part(int n, const double* __restrict__ r, const double* __restrict__ dinv,
                           double* __restrict__ part) {
    __shared__ double sh[8];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double* D = dinv + 9 * (int64_t)i;
        const double* rv = r + 3 * (int64_t)i;
        for (int c = 0; c < 3; ++c) acc += rv[c] * (D[3 * c] * rv[0] + D[3 * c + 1] * rv[1] + D[3 * c + 2] * rv[2]);
    }
    acc = warp_sum(acc);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
        part[blockIdx.x] = s;
    }
}

__global__ void k_xpby(int64_t n, const double* __restrict__ z, const double* __restrict__ S, double* __restrict__ p) {
    const double beta = S[4];
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        p[i] = z[i] + beta * p[i];
}


// ------------------------------------------------------------------ level 0: fused operators
// One pass over the planar BSR3 matrix (8 lanes per block row, FP64 accumulation,
// values in VT = double or float) followed by a row-local epilogue:
//   kL0Resid  y = b - A v (y = A v without b)
//   kL0RUpd   r -= A v
//   kL0Cheb0  r = b - A v; d = c2 D^-1 r; xo = v + d             (first Chebyshev step from v = x)
//   kL0ChebK  r -= A v; d = c1 v + c2 D^-1 r; xo += d            (later steps, v = previous direction)
//   kL0Apply  y = A v
// With dot = 1 the CTA partials of v.y give alpha = r.z / p.q; with dot = 2 the
// partials of b.xo give r.z and beta (the last V-cycle step of the outer CG).
// The last CTA to finish sums the partials in a fixed order.
enum : int { kL0Resid = 0, kL0RUpd = 1, kL0Cheb0 = 2, kL0ChebK = 3, kL0Apply = 4 };

template <typename VT>
struct L0Op {
    int n;
    const int32_t* goff;
    const int32_t* cols;
    const VT* vals;
    const double* v;
    const double* b;
    double* y;
    double* r;
    double* d_out;
    double* xo;
    const double* dinv;
    double c1, c2;
    int dot;
    const double* zold;  // dot = 2 with a flexible outer CG: the previous preconditioned residual
    double* part;
    int* counter;
    double* S;
    // FP32 smoother vectors (mixed precision): the gathered vector as float4 per
    // node (x, y, z, 0) and the new direction written into the same layout; with FP16
    // values and kL0H16Vec the directions are four halves per node (8 bytes) instead
    const float4* v4;
    float* d4_out;
    // FP16 values of the diagonally scaled matrix S A S (S = diag(a_ii)^-1/2): sqrt(a_ii)
    // per node; the gathered float4 vectors then hold sqrt(a_jj) v_j
    const float4* sq4;
    // FP16 smoother directions (kL0H16Vec): {2^k, 2^-k}, the V-cycle's scale of the
    // stored directions (null: 1)
    const float* hs;
};

__device__ __forceinline__ void ld4v(const float* p, float o[4]) {
    const float4 v = __ldcs(reinterpret_cast<const float4*>(p));
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}
__device__ __forceinline__ void ld4v(const __half* p, float o[4]) {
    const uint2 v = __ldcs(reinterpret_cast<const uint2*>(p));
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b.x;
    o[3] = b.y;
}
__device__ __forceinline__ void unpack_h4(uint2 v, float o[4]) {
    const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&v.x));
    const float2 b = __half22float2(*reinterpret_cast<const __half2*>(&v.y));
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b.x;
    o[3] = b.y;
}
template <typename T>
__device__ __forceinline__ void unpack_h4(uint2, T*) {}
__device__ __forceinline__ void ld4v(const double* p, double o[4]) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(p));
    const double2 b = __ldcs(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b.x;
    o[3] = b.y;
}

// Fixed-order CTA sums of (v, v2), then the last CTA to arrive reduces all CTA
// partials and finalises the outer CG scalars: mode 1 alpha = r.z / p.q; mode 2
// beta = (r.z_new - r.z_old) / r.z_prev (Polak-Ribiere, flexible CG; v2 = 0 for
// the plain form) and r.z.
__device__ __forceinline__ void cta_dot_finalize(double v, double v2, int mode, double* part, int* counter,
                                                 double* S) {
    __shared__ double sh[2][32];
    __shared__ int s_last;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    v = warp_sum(v);
    v2 = warp_sum(v2);
    if (lane == 0) {
        sh[0][w] = v;
        sh[1][w] = v2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0, t2 = 0.0;
        for (int k = 0; k < nw; ++k) {
            t += sh[0][k];
            t2 += sh[1][k];
        }
        part[2 * blockIdx.x] = t;
        part[2 * blockIdx.x + 1] = t2;
        __threadfence();
        s_last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || w != 0) return;
    __threadfence();
    double t = 0.0, t2 = 0.0;
    for (int k = lane; k < (int)gridDim.x; k += 32) {
        t += __ldcg(part + 2 * k);
        t2 += __ldcg(part + 2 * k + 1);
    }
    t = warp_sum(t);
    t2 = warp_sum(t2);
    if (lane != 0) return;
    *counter = 0;
    if (mode == 1) {  // p.q -> alpha
        S[1] = t;
        if (!(t > 0.0) || !isfinite(t)) {
            S[6] = 1.0;
            S[5] = 0.0;
        } else {
            S[5] = S[0] / t;
        }
    } else {  // new r.z -> beta
        S[4] = S[0] > 0.0 ? (t - t2) / S[0] : 0.0;
        S[0] = t;
    }
}

#ifndef FX_L0_MIN_BLOCKS
#define FX_L0_MIN_BLOCKS 2
#endif
constexpr int kL0MinBlocks = FX_L0_MIN_BLOCKS;  // 256-thread CTAs resident per SM (2: at most 128 registers)
// The outer CG's q = K p (FP64 values, mode kL0Apply) compiled for its own CTAs per SM (2: on
// the 417k-DOF box a default solve took 51.5-51.7 ms, against 53.4 with 3 (80 registers)
// and 55.0 with 4 (64 registers, spilling))
#ifndef FX_L0_MIN_BLOCKS_APPLY
#define FX_L0_MIN_BLOCKS_APPLY 2
#endif
constexpr int kL0MinBlocksApply = FX_L0_MIN_BLOCKS_APPLY;
// FP16 values: its loads are half as wide as the FP32 form's, so it is latency-bound and
// needs more warps and more loads in flight. Measured per Chebyshev step on the 417k-DOF
// C3D20 box (B200): 57.7 us at 2 CTAs per SM; 54.8 at 3 (85 registers); 61.5 at 4 with
// spills; 50.5 at 4 with the row's epilogue operands loaded after the gathers (no spills
// at 64 registers); 48.1 with, in addition, each group's nine plane loads issued before
// its column ids (FX_L0_VFIRST_H). The FP32 / FP64 forms spill and slow down at those
// budgets, so they keep 2 CTAs per SM.
#ifndef FX_L0_VFIRST_H
#define FX_L0_VFIRST_H 1
#endif
#ifndef FX_L0_LATE_EPI_H
#define FX_L0_LATE_EPI_H 1
#endif
#ifndef FX_L0_MIN_BLOCKS_H
#define FX_L0_MIN_BLOCKS_H 4
#endif
constexpr int kL0MinBlocksH = FX_L0_MIN_BLOCKS_H;
// FP16 smoother: the Chebyshev directions as four halves per node (8 bytes) instead of
// a float4 (the prolongated iterate stays FP32). The directions shrink with the outer
// CG's residual, by 1e8 and more over a solve, so unscaled they fall below FP16's
// subnormal range and the smoothing stops; they are stored times a power of two taken
// from the residual the V-cycle smooths.
#ifndef FX_L0_H16VEC
#define FX_L0_H16VEC 1
#endif
constexpr bool kL0H16Vec = FX_L0_H16VEC != 0;
// With the FP16 smoother, the level-0 eigenvalue estimate's products also come from the FP16
// scaled matrix (1); else from an FP32 copy of the FP64 values made for it (0). On the
// 417k-DOF box: multigrid setup 5.17 -> 4.92 ms, the same 100 CG iterations.
#ifndef FX_AMG_EST_F16
#define FX_AMG_EST_F16 1
#endif
constexpr bool kAmgEstF16 = FX_AMG_EST_F16 != 0;
// the stored directions' 2-norm is about 2^kH16Exp: a direction entry overflows only if the
// residual grows by about 2^(15 - kH16Exp) from one outer iteration to the next, and the
// entries of a vector of 1e7 nodes still sit ~10 binades above the smallest normal FP16
constexpr int kH16Exp = 8;

// {2^k, 2^-k} with 2^k sqrt(rdr) in [2^(kH16Exp-1), 2^kH16Exp), rdr = r.D^-1 r of the
// residual the V-cycle smooths: the smoother's directions c D^-1 r scaled by sqrt(a_ii)
// have a 2-norm of about sqrt(rdr). A power of two scales exactly, so the FP16 roundings
// are those of an FP16 whose range is centred on the vector.
__device__ __forceinline__ float2 h16_scale(double rdr) {
    if (!(rdr > 0.0) || !isfinite(rdr)) return make_float2(1.0f, 1.0f);
    int e;
    frexp(sqrt(rdr), &e);
    const int k = max(-100, min(100, kH16Exp - e));
    return make_float2(ldexpf(1.0f, k), ldexpf(1.0f, -k));
}

// FP16 bits of x rounded to nearest, clamped to the finite range (a direction that
// outgrows the lagged scale saturates instead of turning the smoother's sums into inf)
__device__ __forceinline__ uint32_t h16_bits(float x) {
    return __half_as_ushort(__float2half_rn(fminf(fmaxf(x, -65504.0f), 65504.0f)));
}

#ifndef FX_L0_LANES
#define FX_L0_LANES 8
#endif
constexpr int kL0Lanes = FX_L0_LANES;          // lanes per block row (8 or 4)
constexpr int kL0RowsPerWarp = 32 / kL0Lanes;
constexpr int kL0LaneShift = kL0Lanes == 8 ? 3 : 2;
#ifndef FX_L0_UNROLL
#define FX_L0_UNROLL 2
#endif
constexpr int kL0Unroll = FX_L0_UNROLL;  // groups of a row in flight per lane

// G32: gathers from o.v4 (FP32, 16 B per node) and writes the direction into
// o.d4_out; the row's own FP64 values still come from o.v where the mode needs
// them (Cheb0: the iterate), else from o.v4.
template <typename VT, int MODE, bool G32 = false>
__global__ void __launch_bounds__(256, std::is_same<VT, __half>::value ? kL0MinBlocksH
                                      : (MODE == kL0Apply ? kL0MinBlocksApply : kL0MinBlocks))
    k_l0_op(L0Op<VT> o) {
    // FP16 values (of the scaled matrix): FP32 gathers of the scaled vectors, row sums
    // scaled back by sqrt(a_ii), directions written scaled
    constexpr bool H = std::is_same<VT, __half>::value;
    // FP16 values: the row-local epilogue operands are loaded after the gathers
    // (FX_L0_LATE_EPI_H), which frees their registers during the gather loop
    constexpr bool kL0LateEpi = H && FX_L0_LATE_EPI_H;
    constexpr bool kL0VFirst = H && FX_L0_VFIRST_H;
    // FP16 directions: written by the Chebyshev steps, gathered by all but the step from
    // the (FP32) iterate; 2^-k is applied to the row sums, after the gathers
    constexpr bool kH16 = H && G32 && kL0H16Vec;
    constexpr bool kH16g = kH16 && (MODE == kL0ChebK || MODE == kL0RUpd);
    const int sub = threadIdx.x & (kL0Lanes - 1);
    const int row0 = (blockIdx.x * blockDim.x + threadIdx.x) >> kL0LaneShift;
    const int rows_per_grid = (gridDim.x * blockDim.x) >> kL0LaneShift;
    // uniform trip count per warp: the warp's rows share one base
    const int nb = ((o.n + kL0RowsPerWarp - 1) / kL0RowsPerWarp) * kL0RowsPerWarp;
    const double* __restrict__ v = o.v;
    double dsum = 0.0, dsum2 = 0.0;
    for (int base = row0 - (row0 & (kL0RowsPerWarp - 1)); base < nb; base += rows_per_grid) {
        const int row = base + (row0 & (kL0RowsPerWarp - 1));
        const bool valid = row < o.n;
        const int g0 = valid ? o.goff[row] : 0;
        const int ng = valid ? o.goff[row + 1] - g0 : 0;
        // row-local operands of the epilogue, loaded before the gathers so that their latency overlaps
        const int64_t o3 = 3 * (int64_t)row;
        const int c = sub < 3 ? sub : 0;
        const bool epi = valid && sub < 3;
        double src3[3] = {0.0, 0.0, 0.0}, Dr[3] = {0.0, 0.0, 0.0}, vc = 0.0, xoc = 0.0, bc = 0.0, zoc = 0.0;
        float4 sqi = make_float4(1.f, 1.f, 1.f, 0.f);
        float2 hsc = make_float2(1.f, 1.f);  // {2^k, 2^-k}: .x is read where the direction is stored
        auto load_epi = [&]() {
        if (H && epi) sqi = __ldg(o.sq4 + row);
        if (kH16g && epi && o.hs) hsc.y = __ldg(o.hs + 1);
        if (epi) {
            if (MODE == kL0Cheb0 || MODE == kL0ChebK) {
                const double* src = MODE == kL0Cheb0 ? o.b : o.r;
#pragma unroll
                for (int kk = 0; kk < 3; ++kk) {
                    src3[kk] = src[o3 + kk];
                    Dr[kk] = o.dinv[9 * (int64_t)row + 3 * c + kk];
                }
                if (G32 && MODE == kL0ChebK) {
                    const float* own = reinterpret_cast<const float*>(o.v4 + row);
                    if constexpr (kH16)
                        vc = (double)(__half2float(reinterpret_cast<const __half*>(o.v4)[4 * (int64_t)row + c]) *
                                      hsc.y);
                    else vc = (double)own[c];
                    if (H) vc /= (double)(c == 0 ? sqi.x : (c == 1 ? sqi.y : sqi.z));
                } else {
                    vc = v[o3 + c];
                }
                if (MODE == kL0ChebK) xoc = o.xo[o3 + c];
                if (o.dot) bc = o.b[o3 + c];
                if (o.dot && o.zold) zoc = o.zold[o3 + c];
            } else if (MODE == kL0Apply) {
                vc = v[o3 + c];
            } else if (MODE == kL0Resid) {
                bc = o.b ? o.b[o3 + c] : 0.0;
            } else {
                src3[0] = o.r[o3 + c];
            }
        }
        };
        if (!kL0LateEpi) load_epi();
        double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll kL0Unroll
        for (int g = sub; g < ng; g += kL0Lanes) {
            // FP16 values (kL0VFirst): the group's nine 8-byte plane loads are issued before
            // the column ids and the gathers that depend on them
            uint2 raw[kL0VFirst ? 9 : 1];
            if constexpr (kL0VFirst) {
                const __half* vh = reinterpret_cast<const __half*>(o.vals) + ((int64_t)g0 * 9 + g) * 4;
#pragma unroll
                for (int k = 0; k < 9; ++k)
                    raw[k] = __ldcs(reinterpret_cast<const uint2*>(vh + (int64_t)k * ng * 4));
            }
            const int4 cc = __ldg(reinterpret_cast<const int4*>(o.cols) + g0 + g);
            const int cj[4] = {cc.x, cc.y, cc.z, cc.w};
            // FP32 values with FP32 gathered vectors: the group's 4 blocks are summed in
            // FP32 (no FP64 conversions of the 36 values) and added to the FP64 row sums
            using GT = typename std::conditional<G32, float, double>::type;
            GT xv[4][3];
            if (G32) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if constexpr (kH16g) {
                        const uint2 u = __ldg(reinterpret_cast<const uint2*>(o.v4) + cj[q]);
                        const float2 a = __half22float2(*reinterpret_cast<const __half2*>(&u.x));
                        xv[q][0] = a.x;
                        xv[q][1] = a.y;
                        xv[q][2] = __half2float(__ushort_as_half((unsigned short)(u.y & 0xffffu)));
                    } else {
                        const float4 t = __ldg(o.v4 + cj[q]);
                        xv[q][0] = t.x;
                        xv[q][1] = t.y;
                        xv[q][2] = t.z;
                    }
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int k = 0; k < 3; ++k) xv[q][k] = (GT)__ldg(v + 3 * (int64_t)cj[q] + k);
            }
            const VT* vb = o.vals + ((int64_t)g0 * 9 + g) * 4;
            const int64_t pl = (int64_t)ng * 4;
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                using MT = typename std::conditional<H, float, VT>::type;
                MT m0[4], m1[4], m2[4];
                if constexpr (kL0VFirst) {
                    unpack_h4(raw[3 * r], m0);
                    unpack_h4(raw[3 * r + 1], m1);
                    unpack_h4(raw[3 * r + 2], m2);
                } else {
                    ld4v(vb + (3 * r) * pl, m0);
                    ld4v(vb + (3 * r + 1) * pl, m1);
                    ld4v(vb + (3 * r + 2) * pl, m2);
                }
                GT t = 0;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    t += (GT)m0[q] * xv[q][0] + (GT)m1[q] * xv[q][1] + (GT)m2[q] * xv[q][2];
                acc[r] += (double)t;
            }
        }
#pragma unroll
        for (int s = kL0Lanes / 2; s > 0; s >>= 1)
#pragma unroll
            for (int r = 0; r < 3; ++r) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], s);
        if (kL0LateEpi) load_epi();
        // epilogue: lane c of the row's 8 handles component c
        if (H) {  // (A v)_i = sqrt(a_ii) (S A S (sqrt(a_jj) v_j))_i; FP16 directions: times 2^-k
            const double u = kH16g ? (double)hsc.y : 1.0;
            acc[0] *= (double)sqi.x * u;
            acc[1] *= (double)sqi.y * u;
            acc[2] *= (double)sqi.z * u;
        }
        const double axc = c == 0 ? acc[0] : (c == 1 ? acc[1] : acc[2]);
        __syncwarp();  // every lane's reads of r (above) are ordered before any lane writes r[c]
        if (!epi) continue;
        if (MODE == kL0Resid) {
            o.y[o3 + c] = o.b ? bc - axc : axc;
        } else if (MODE == kL0RUpd) {
            o.r[o3 + c] = src3[0] - axc;
        } else if (MODE == kL0Apply) {
            o.y[o3 + c] = axc;
            dsum += vc * axc;
        } else {  // Chebyshev steps
            const double rr[3] = {src3[0] - acc[0], src3[1] - acc[1], src3[2] - acc[2]};
            const double z = Dr[0] * rr[0] + Dr[1] * rr[1] + Dr[2] * rr[2];
            o.r[o3 + c] = c == 0 ? rr[0] : (c == 1 ? rr[1] : rr[2]);
            const double dn = (MODE == kL0Cheb0 ? 0.0 : o.c1 * vc) + o.c2 * z;
            if (kH16) {
                if (o.hs) hsc.x = __ldg(o.hs);
                reinterpret_cast<unsigned short*>(o.d4_out)[4 * (int64_t)row + c] = (unsigned short)h16_bits(
                    (float)(dn * (double)(c == 0 ? sqi.x : (c == 1 ? sqi.y : sqi.z))) * hsc.x);
            } else if (G32) o.d4_out[4 * (int64_t)row + c] = (float)(H ? dn * (double)(c == 0 ? sqi.x : (c == 1 ? sqi.y : sqi.z)) : dn);
            else o.d_out[o3 + c] = dn;
            const double xn = (MODE == kL0Cheb0 ? vc : xoc) + dn;
            o.xo[o3 + c] = xn;
            if (o.dot) {
                dsum += bc * xn;
                dsum2 += bc * zoc;
            }
        }
    }
    if (o.dot) cta_dot_finalize(dsum, dsum2, o.dot, o.part, o.counter, o.S);
}

// ---- K-cycle on a coarse level (one CTA; the level has at most a few 10k DOF)
// Two steps of a flexible CG for A x = b preconditioned by the next cycle:
//   z1 = B(b), v1 = A z1, alpha1 = z1.b / z1.v1, x = alpha1 z1, r = b - alpha1 v1;
//   z2 = B(r), v2 = A z2, w = z2 - (z2.v1 / z1.v1) z1, x += (w.r / w.Aw) w.
template <int NV>
__device__ __forceinline__ void block_sums(double (&v)[NV], double* sh /* [NV][32] */) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k * 32 + w] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NV; ++k) {  // every thread sums in the same fixed order
        double t = 0.0;
        for (int j = 0; j < nw; ++j) t += sh[k * 32 + j];
        v[k] = t;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(1024) k_kcycle1(int64_t n, const double* __restrict__ b,
                                                  const double* __restrict__ z1, const double* __restrict__ v1,
                                                  double* __restrict__ x, double* __restrict__ r,
                                                  double* __restrict__ kc) {
    __shared__ double sh[2 * 32];
    double s[2] = {0.0, 0.0};
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        s[0] += z1[i] * b[i];
        s[1] += z1[i] * v1[i];
    }
    block_sums<2>(s, sh);
    const double sigma = s[1];
    const double alpha = sigma > 0.0 && isfinite(sigma) ? s[0] / sigma : 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        x[i] = alpha * z1[i];
        r[i] = b[i] - alpha * v1[i];
    }
    if (threadIdx.x == 0) kc[0] = sigma;
}

__global__ void __launch_bounds__(1024) k_kcycle2(int64_t n, const double* __restrict__ z1,
                                                  const double* __restrict__ v1, const double* __restrict__ z2,
                                                  const double* __restrict__ v2, const double* __restrict__ r,
                                                  double* __restrict__ x, const double* __restrict__ kc) {
    __shared__ double sh[2 * 32];
    const double sigma = kc[0];
    double g[1] = {0.0};
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) g[0] += z2[i] * v1[i];
    block_sums<1>(g, sh);
    const double beta = sigma > 0.0 && isfinite(sigma) ? g[0] / sigma : 0.0;
    double s[2] = {0.0, 0.0};
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        const double w = z2[i] - beta * z1[i];
        const double aw = v2[i] - beta * v1[i];
        s[0] += w * r[i];
        s[1] += w * aw;
    }
    block_sums<2>(s, sh);
    const double alpha = s[1] > 0.0 && isfinite(s[1]) ? s[0] / s[1] : 0.0;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) x[i] += alpha * (z2[i] - beta * z1[i]);
}

// ---- coarse levels (row-major 6x6 block CSR): SpMV fused with the smoother
// update, one warp per block row, a lane per block of the row (coarse_row6); the
// same modes as the fine-level operator (kL0Resid, kL0RUpd, kL0Cheb0, kL0ChebK).
// Threads per CTA of the coarse-level kernels (warp per block row / aggregate).
#ifndef FX_LN_THREADS
#define FX_LN_THREADS 128
#endif
constexpr int kLnThreads = FX_LN_THREADS;
// CTAs per SM the coarse-level operators are compiled for: 4 x 128 threads leaves 128
// registers, enough for a lane's whole 6x6 block and its gathered 6-vector in flight
// without spills. On the 417k-DOF box a default solve took 51.9-52.4 ms with 4, against
// 52.9-53.2 with 6 (80 registers), 52.5-53.2 with 7 (72, spilling) and 52.3-52.5 with 8
// (64, the epilogue operands loaded after the row sums, FX_LN_LATE_EPI).
#ifndef FX_LN_MIN_BLOCKS
#define FX_LN_MIN_BLOCKS 4
#endif
constexpr int kLnMinBlocks = FX_LN_MIN_BLOCKS;
#ifndef FX_LN_LATE_EPI
#define FX_LN_LATE_EPI 0
#endif
constexpr bool kLnLateEpi = FX_LN_LATE_EPI != 0;  // epilogue operands loaded after the row sums

struct LnOp {
    int n;
    const int32_t* row_ptr;
    const int32_t* cols;
    const double* vals;
    const double* v;
    const double* b;
    double* y;
    double* r;
    double* d_out;
    double* xo;
    const double* dinv;  // 6x6 block inverses
    double c1, c2;
};

template <int MODE>
__global__ void __launch_bounds__(kLnThreads, kLnMinBlocks) k_ln_op(LnOp o) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= o.n) return;  // warp-uniform
    const int64_t o6 = 6 * (int64_t)row;
    const int c = lane < 6 ? lane : 0;
    const bool epi = lane < 6;
    double src6[6] = {0, 0, 0, 0, 0, 0}, Dr[6] = {0, 0, 0, 0, 0, 0}, vc = 0.0, xoc = 0.0, bc = 0.0;
    auto load_epi = [&]() {  // row-local operands of the epilogue
    if (epi) {
        if (MODE == kL0Cheb0 || MODE == kL0ChebK) {
            const double* src = MODE == kL0Cheb0 ? o.b : o.r;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                src6[k] = src[o6 + k];
                Dr[k] = o.dinv[36 * (int64_t)row + 6 * c + k];
            }
            vc = o.v[o6 + c];
            if (MODE == kL0ChebK) xoc = o.xo[o6 + c];
        } else if (MODE == kL0Resid) {
            bc = o.b ? o.b[o6 + c] : 0.0;
        } else {
            src6[0] = o.r[o6 + c];
        }
    }
    };
    if (!kLnLateEpi) load_epi();
    // lanes over the row's blocks; every lane ends with the six row sums
    const int b0 = o.row_ptr[row];
    double acc[6];
    coarse_row6<false>(o.cols, o.vals, o.v, b0, o.row_ptr[row + 1] - b0, lane, acc);
    if (kLnLateEpi) load_epi();
    double axc = acc[0];
#pragma unroll
    for (int r = 1; r < 6; ++r)
        if (c == r) axc = acc[r];
    __syncwarp();  // every lane's reads of r are ordered before any lane writes r[c]
    if (!epi) return;
    if (MODE == kL0Resid) {
        o.y[o6 + c] = o.b ? bc - axc : axc;
    } else if (MODE == kL0RUpd) {
        o.r[o6 + c] = src6[0] - axc;
    } else {
        double z = 0.0, rc = 0.0;
#pragma unroll
        for (int k = 0; k < 6; ++k) {
            const double rk = src6[k] - acc[k];
            z += Dr[k] * rk;
            if (k == c) rc = rk;
        }
        o.r[o6 + c] = rc;
        const double dn = (MODE == kL0Cheb0 ? 0.0 : o.c1 * vc) + o.c2 * z;
        o.d_out[o6 + c] = dn;
        o.xo[o6 + c] = (MODE == kL0Cheb0 ? vc : xoc) + dn;
    }
}

// FP32 copy of a node's three components for the smoother's gathers; with the FP16
// scaled matrix (sq4 != null) multiplied by sqrt(a_ii) per component.
__device__ __forceinline__ float4 scaled4(const double t[3], const float4* __restrict__ sq4, int i) {
    if (!sq4) return make_float4((float)t[0], (float)t[1], (float)t[2], 0.0f);
    const float4 q = sq4[i];
    return make_float4((float)(t[0] * (double)q.x), (float)(t[1] * (double)q.y), (float)(t[2] * (double)q.z), 0.0f);
}

// Stores node i of a smoother direction: float4 per node, or with the FP16 scaled matrix
// (sq4 != null) and kL0H16Vec four halves per node (8 bytes), times hs = 2^k, in the same buffer.
__device__ __forceinline__ void store_dir4(float4* __restrict__ base, int i, const double t[3],
                                           const float4* __restrict__ sq4, float hs) {
    const float4 f = scaled4(t, sq4, i);
    if (kL0H16Vec && sq4) {
        uint2 u;
        u.x = h16_bits(f.x * hs) | (h16_bits(f.y * hs) << 16);
        u.y = h16_bits(f.z * hs);
        reinterpret_cast<uint2*>(base)[i] = u;
    } else {
        base[i] = f;
    }
}

// x4[i] = the float4 of node i's three components scaled by sqrt(a_ii) (the FP16
// operator's gathered vector), from an FP64 vector
__global__ void k_scaled4(int n, const double* __restrict__ x, const float4* __restrict__ sq4, float4* __restrict__ x4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double t[3] = {x[3 * (int64_t)i], x[3 * (int64_t)i + 1], x[3 * (int64_t)i + 2]};
    x4[i] = scaled4(t, sq4, i);
}

// first smoothing step from x = 0 at any level: d = c2 D^-1 b; x = d; r = b
__global__ void k_cheb_start(int n, int bs, const double* __restrict__ dinv, const double* __restrict__ b,
                             double* __restrict__ r, double* __restrict__ d, double* __restrict__ x, double c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t o = (int64_t)i * bs;
    const double* Di = dinv + (int64_t)i * bs * bs;
    for (int k = 0; k < bs; ++k) {
        double t = 0.0;
        for (int j = 0; j < bs; ++j) t += Di[k * bs + j] * b[o + j];
        t *= c2;
        d[o + k] = t;
        x[o + k] = t;
    }
    for (int k = 0; k < bs; ++k) r[o + k] = b[o + k];
}

// first pre-smoothing step from x = 0: d = c2 D^-1 b; x = d; r = b
// (d4 != null: the direction as float4 per node instead of d; hs != null: FP16 directions,
// whose scale for this V-cycle is taken from *rdr = b.D^-1 b and published in hs)
__global__ void k_l0_cheb_start(int n, const double* __restrict__ dinv, const double* __restrict__ b,
                                double* __restrict__ r, double* __restrict__ d, float4* __restrict__ d4,
                                double* __restrict__ x, double c2, const float4* __restrict__ sq4,
                                const double* __restrict__ rdr, float* __restrict__ hs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float2 hsc = hs ? h16_scale(*rdr) : make_float2(1.0f, 1.0f);
    if (hs && i == 0) {  // read by the V-cycle's later launches only
        hs[0] = hsc.x;
        hs[1] = hsc.y;
    }
    const int64_t o3 = 3 * (int64_t)i;
    const double bb[3] = {b[o3], b[o3 + 1], b[o3 + 2]};
    const double* D = dinv + 9 * (int64_t)i;
    double t[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        t[c] = c2 * (D[3 * c] * bb[0] + D[3 * c + 1] * bb[1] + D[3 * c + 2] * bb[2]);
        r[o3 + c] = bb[c];
        x[o3 + c] = t[c];
    }
    if (d4) store_dir4(d4, i, t, sq4, hsc.x);
    else
        for (int c = 0; c < 3; ++c) d[o3 + c] = t[c];
}

// fine level: x += Q xc (3 rows per node) and the FP32 copy of x for the smoother gathers
__global__ void k_prolong0(int n, const int32_t* __restrict__ agg, const double* __restrict__ Q,
                           const double* __restrict__ xc, double* __restrict__ xf, float4* __restrict__ x4,
                           double alpha, const float4* __restrict__ sq4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double* x = xc + (int64_t)agg[i] * 6;
    double out[3];
    for (int k = 0; k < 3; ++k) {
        const double* q = Q + (3 * (int64_t)i + k) * 6;
        double t = 0.0;
        for (int c = 0; c < 6; ++c) t += q[c] * x[c];
        out[k] = xf[3 * (int64_t)i + k] + alpha * t;
        xf[3 * (int64_t)i + k] = out[k];
    }
    x4[i] = scaled4(out, sq4, i);
}

// The CG update fused with the first step of the V-cycle that follows it:
// x += alpha p, r -= alpha q, r.D^-1 r reduced by the last CTA into S[2], and
// with b = the new r: r0 = b, x0 = d = c2 D^-1 b (what k_l0_cheb_start does).
// hs != null (FP16 directions): the V-cycle's scale comes from S[2] as this launch
// finds it, the previous residual's r.D^-1 r (the new one is reduced only at the end),
// and the last CTA publishes it in hs for the V-cycle's later launches.
__global__ void __launch_bounds__(256) k_amg_update_start(int n, double* __restrict__ S, const double* __restrict__ p,
                                                          const double* __restrict__ q, double* __restrict__ x,
                                                          double* __restrict__ r, const double* __restrict__ dinv,
                                                          double* __restrict__ part, int* __restrict__ counter,
                                                          double* __restrict__ r0, double* __restrict__ x0,
                                                          double* __restrict__ d0, float4* __restrict__ d4,
                                                          double c2, const float4* __restrict__ sq4,
                                                          float* __restrict__ hs) {
    __shared__ double sh[32];
    __shared__ int s_last;
    const double alpha = S[5];
    const float2 hsc = hs ? h16_scale(S[2]) : make_float2(1.0f, 1.0f);
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int64_t o3 = 3 * (int64_t)i;
        double rv[3];
        for (int c = 0; c < 3; ++c) {
            x[o3 + c] += alpha * p[o3 + c];
            rv[c] = r[o3 + c] - alpha * q[o3 + c];
            r[o3 + c] = rv[c];
            r0[o3 + c] = rv[c];
        }
        const double* D = dinv + 9 * (int64_t)i;
        double t[3];
        for (int c = 0; c < 3; ++c) {
            const double dr = D[3 * c] * rv[0] + D[3 * c + 1] * rv[1] + D[3 * c + 2] * rv[2];
            acc += rv[c] * dr;
            t[c] = c2 * dr;
            x0[o3 + c] = t[c];
        }
        if (d4) store_dir4(d4, i, t, sq4, hsc.x);
        else
            for (int c = 0; c < 3; ++c) d0[o3 + c] = t[c];
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    acc = warp_sum(acc);
    if (lane == 0) sh[w] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tt = 0.0;
        for (int k = 0; k < nw; ++k) tt += sh[k];
        part[blockIdx.x] = tt;
        __threadfence();
        s_last = atomicAdd(counter, 1) == (int)gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last || w != 0) return;
    __threadfence();
    double tt = 0.0;
    for (int k = lane; k < (int)gridDim.x; k += 32) tt += __ldcg(part + k);
    tt = warp_sum(tt);
    if (lane == 0) {
        S[2] = tt;
        *counter = 0;
        if (hs) {
            hs[0] = hsc.x;
            hs[1] = hsc.y;
        }
    }
}

// sqrt of the fine matrix's diagonal per DOF (float4 per node; 1 where a node has no
// diagonal block or a non-positive diagonal)
__global__ void k_diag_sqrt(int n, const int32_t* __restrict__ goff, const int32_t* __restrict__ diag_k,
                            const double* __restrict__ vals, float4* __restrict__ sq4) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int kk = diag_k[i];
    float o[3] = {1.f, 1.f, 1.f};
    if (kk >= 0) {
        const int64_t g0 = goff[i], ng = goff[i + 1] - g0;
        for (int c = 0; c < 3; ++c) {
            const double a = vals[(g0 * 9 + (int64_t)(4 * c) * ng + kk / 4) * 4 + (kk & 3)];
            if (a > 0.0) o[c] = (float)sqrt(a);
        }
    }
    sq4[i] = make_float4(o[0], o[1], o[2], 0.f);
}

// FP16 copy of the scaled matrix S A S, S = diag(sqrt(a_ii))^-1 with the float square
// roots of k_diag_sqrt (the smoother scales its vectors by the same values): |entries| <= 1
// for a symmetric positive definite matrix. Warp per block row; lane `it` takes plane
// e = it / ng of group g = it % ng, whose 4 values are the row's vec4 number it (planar
// layout), so a warp reads consecutive 32-byte vectors; the scale is an FP32 reciprocal
// of sqrt(a_ii) sqrt(a_jj) (its rounding, ~6e-8, is far below FP16's).
__global__ void k_vals_to_f16(int n, const int32_t* __restrict__ goff, const int32_t* __restrict__ cols,
                              const double* __restrict__ vals, const float4* __restrict__ sq4, __half* __restrict__ out) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (row >= n) return;
    const int64_t g0 = goff[row];
    const int ng = goff[row + 1] - (int)g0;
    const float4 sr = sq4[row];
    for (int it = lane; it < 9 * ng; it += 32) {
        const int e = it / ng, g = it - e * ng;
        const int4 cc = __ldg(reinterpret_cast<const int4*>(cols) + g0 + g);
        const int cj[4] = {cc.x, cc.y, cc.z, cc.w};
        const int cr = e / 3, ccomp = e - 3 * cr;
        const float si = cr == 0 ? sr.x : (cr == 1 ? sr.y : sr.z);
        const double2* src = reinterpret_cast<const double2*>(vals + (g0 * 9 + it) * 4);
        const double2 v01 = __ldcs(src), v23 = __ldcs(src + 1);
        const double v[4] = {v01.x, v01.y, v23.x, v23.y};
        __half h[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 t = __ldg(sq4 + cj[q]);
            const float sj = ccomp == 0 ? t.x : (ccomp == 1 ? t.y : t.z);
            h[q] = __double2half(v[q] * (double)(1.0f / (si * sj)));
        }
        uint2 packed;
        packed.x = (uint32_t)__half_as_ushort(h[0]) | ((uint32_t)__half_as_ushort(h[1]) << 16);
        packed.y = (uint32_t)__half_as_ushort(h[2]) | ((uint32_t)__half_as_ushort(h[3]) << 16);
        reinterpret_cast<uint2*>(out)[g0 * 9 + it] = packed;
    }
}

__global__ void k_f64_to_f32(int64_t n, const double* __restrict__ a, float* __restrict__ b) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = (float)a[i];
}

}  // namespace

// ------------------------------------------------------------------ host side

// Grid of the level-0 operators: at most one wave of resident CTAs (grid-stride rows);
// h: the FP16-value kernels, which have their own register budget; apply: the outer CG's
// FP64 q = K p (kL0MinBlocksApply).
static unsigned l0_grid(int n, bool h = false, bool apply = false) {
    thread_local int cached_dev = -1, cached_cap[3] = {0, 0, 0};  // per host thread: contexts live on one thread each
    int dev = 0;
    FX_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev != cached_dev) {
        int sms = 0, per_sm = 0, per_sm_h = 0, per_sm_a = 0;
        FX_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        FX_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_l0_op<double, kL0ChebK>, 256, 0));
        FX_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_h, k_l0_op<__half, kL0ChebK, true>, 256,
                                                                    0));
        FX_CUDA_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_a, k_l0_op<double, kL0Apply>, 256, 0));
        cached_cap[0] = std::max(1, sms * std::max(1, per_sm));
        cached_cap[1] = std::max(1, sms * std::max(1, per_sm_h));
        cached_cap[2] = std::max(1, sms * std::max(1, per_sm_a));
        cached_dev = dev;
    }
    return (unsigned)std::min<int64_t>(grid_for((int64_t)n * kL0Lanes), cached_cap[apply ? 2 : (h ? 1 : 0)]);
}

// Slots of the partial-sum buffer a level-0 operator with a dot product needs: two per CTA
// of the largest level-0 grid (the FP16 kernels run more CTAs per SM than the others).
static int64_t l0_part_slots(int n) {
    return 2 * (int64_t)std::max({l0_grid(n, false), l0_grid(n, true), l0_grid(n, false, true)});
}

template <typename VT>
static L0Op<VT> l0_op(const AmgLevel& l, const VT* vals) {
    L0Op<VT> o{};
    o.n = l.n;
    o.goff = l.S0->goff.ptr;
    o.cols = l.S0->cols.ptr;
    o.vals = vals;
    o.dinv = l.dinv0;
    return o;
}

static void level_spmv(const AmgLevel& l, const double* x, const double* b, double* y, cudaStream_t s) {
    if (l.S0) {
        L0Op<double> o = l0_op<double>(l, l.vals0);
        o.v = x;
        o.b = b;
        o.y = y;
        FX_LAUNCH((k_l0_op<double, kL0Resid>), l0_grid(l.n), 256, 0, s, o);
    } else {
        FX_LAUNCH(k_ln_spmv, grid_for((int64_t)l.n * 32), 256, 0, s, l.n, l.row_ptr.ptr, l.cols.ptr, l.vals.ptr, x, b,
                  y);
    }
}

// red[nb] = a . b (deterministic, stays on the device)
static void dot_dev(const double* a, const double* b, int64_t n, DBuf<double>& red, cudaStream_t s) {
    const int nb = 296;
    if (red.n < (size_t)nb + 1) red.alloc(nb + 1, s);
    FX_LAUNCH(k_dot_part, nb, 256, 0, s, n, a, b, red.ptr);
    FX_LAUNCH(k_sum_part, 1, 32, 0, s, nb, red.ptr, red.ptr + nb);
}

// Largest eigenvalue of D^-1 A by 12 power iterations from a fixed hashed start
// vector, normalised on the device; one host read at the end.
// (level 0: with vals16 / sq4 the products come from the FP16 scaled matrix the smoother
// reads, through float4 copies of x in l.x4; else from vals32, an FP32 copy, when given)
// warm: start from the vector the previous estimate on this level ended with (a
// refresh after a small change of the matrix) and iterate 4 times instead of 12.
static void estimate_lmax(AmgLevel& l, DBuf<double>& red, cudaStream_t s, const float* vals32, bool warm,
                          const __half* vals16 = nullptr, const float4* sq4 = nullptr) {
    const int64_t nd = (int64_t)l.n * l.bs;
    const int nb = 296;
    const bool from_ev = warm && l.ev.n == (size_t)nd;
    if (from_ev)
        FX_CUDA_CHECK(cudaMemcpyAsync(l.x.ptr, l.ev.ptr, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    else
        FX_LAUNCH(k_fill_hash, grid_for(nd), 256, 0, s, nd, l.x.ptr);
    dot_dev(l.x.ptr, l.x.ptr, nd, red, s);
    FX_LAUNCH(k_normalize, grid_for(nd), 256, 0, s, nd, red.ptr + nb, l.x.ptr, l.x.ptr);
    const int iters = from_ev ? 4 : 12;
    for (int it = 0; it < iters; ++it) {
        if (l.S0 && vals16 && sq4) {  // t = A x, |x| = 1, from the FP16 scaled matrix
            float4* x4 = reinterpret_cast<float4*>(l.x4.ptr);
            FX_LAUNCH(k_scaled4, grid_for(l.n), 256, 0, s, l.n, l.x.ptr, sq4, x4);
            L0Op<__half> o = l0_op<__half>(l, vals16);
            o.v4 = x4;
            o.y = l.t.ptr;
            o.sq4 = sq4;
            FX_LAUNCH((k_l0_op<__half, kL0Resid, true>), l0_grid(l.n, true), 256, 0, s, o);
        } else if (l.S0 && vals32) {  // t = A x, |x| = 1
            L0Op<float> o = l0_op<float>(l, vals32);
            o.v = l.x.ptr;
            o.y = l.t.ptr;
            FX_LAUNCH((k_l0_op<float, kL0Resid>), l0_grid(l.n), 256, 0, s, o);
        } else {
            level_spmv(l, l.x.ptr, nullptr, l.t.ptr, s);
        }
        FX_LAUNCH(k_cheb_init, grid_for(l.n), 256, 0, s, l.n, l.bs, l.dinv_ptr(), l.t.ptr, l.d.ptr, l.r.ptr, 1.0,
                  1);  // d = D^-1 A x
        dot_dev(l.d.ptr, l.d.ptr, nd, red, s);
        FX_LAUNCH(k_normalize, grid_for(nd), 256, 0, s, nd, red.ptr + nb, l.d.ptr, l.x.ptr);
    }
    l.ev.alloc(nd, s);
    FX_CUDA_CHECK(cudaMemcpyAsync(l.ev.ptr, l.x.ptr, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    double nd2 = 0.0;
    FX_CUDA_CHECK(cudaMemcpyAsync(&nd2, red.ptr + nb, sizeof(double), cudaMemcpyDeviceToHost, s));
    stream_wait(s, "amg eigenvalue estimate");
    l.lmax = 1.1 * (nd2 > 0.0 ? std::sqrt(nd2) : 1.0);
}

// The fine level of a Galerkin product as the kernels read it: the planar BSR3
// at level 0, row-major 6x6 block CSR (with each block's row) above.
static FineView fine_view(const AmgLevel& l) {
    FineView F{};
    F.bs = l.bs;
    if (l.S0) {
        F.blk_row = l.S0->blk_row.ptr;
        F.vals = l.vals0;
        F.row_ptr = l.S0->row_ptr.ptr;
        F.goff = l.S0->goff.ptr;
        F.cols4 = l.S0->cols.ptr;
    } else {
        F.blk_row = l.gal_rows.ptr;
        F.blk_col = l.cols.ptr;
        F.vals = l.vals.ptr;
    }
    return F;
}

// c.vals = Q^T A Q over lf's Galerkin map (fixed-order sums per coarse block)
static void galerkin(const AmgLevel& lf, AmgLevel& c, cudaStream_t s) {
    const FineView F = fine_view(lf);
    const int64_t ncb = c.nblocks;
    if (F.bs == 3)
        FX_LAUNCH(k_galerkin<3>, grid_for(ncb * 32, 128), 128, 0, s, ncb, lf.gal_seg.ptr, lf.gal_blk.ptr, F, lf.Q.ptr,
                  c.vals.ptr);
    else
        FX_LAUNCH(k_galerkin<6>, grid_for(ncb * 32, 128), 128, 0, s, ncb, lf.gal_seg.ptr, lf.gal_blk.ptr, F, lf.Q.ptr,
                  c.vals.ptr);
}

// Dense inverse of the coarsest level's matrix (blocked Gauss-Jordan); fails
// with FX_NUMERICAL when the matrix is singular (rigid-body modes).
void Amg::coarsest_inverse(AmgLevel& l, cudaStream_t s) {
    const int64_t nd = (int64_t)l.n * l.bs;
    l.dense_inv.alloc((size_t)nd * nd, s);
    l.dense_inv.zero(s);
    FX_LAUNCH(k_dense_from_bsr, grid_for(l.n, 64), 64, 0, s, l.n, l.row_ptr.ptr, l.cols.ptr, l.vals.ptr,
              l.dense_inv.ptr);
    DBuf<uint8_t> dead;
    dead.alloc(nd, s);
    DBuf<double> diag0;
    DBuf<int> singular;
    diag0.alloc(nd, s);
    singular.alloc(1, s);
    singular.zero(s);
    FX_LAUNCH(k_dense_decouple, 1, 1024, 0, s, (int)nd, l.dense_inv.ptr, dead.ptr, diag0.ptr);
    for (int k0 = 0; k0 < (int)nd; k0 += kPanel) {
        const int b = std::min<int>(kPanel, (int)nd - k0);
        FX_LAUNCH(k_panel_inverse, 1, 1024, 0, s, (int)nd, k0, b, l.dense_inv.ptr, diag0.ptr, singular.ptr);
        FX_LAUNCH(k_panel_rows, grid_for(nd, 128), 128, 0, s, (int)nd, k0, b, l.dense_inv.ptr);
        const unsigned tiles = (unsigned)((nd + 31) / 32);
        FX_LAUNCH(k_panel_update, dim3(tiles, tiles), 256, 0, s, (int)nd, k0, b, l.dense_inv.ptr);
        FX_LAUNCH(k_panel_cols, grid_for(nd * 32), 256, 0, s, (int)nd, k0, b, l.dense_inv.ptr);
    }
    FX_LAUNCH(k_dense_zero_dead, grid_for(nd * 32), 256, 0, s, (int)nd, l.dense_inv.ptr, dead.ptr);
    int sing = 0;
    FX_CUDA_CHECK(cudaMemcpyAsync(&sing, singular.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    stream_wait(s, "amg coarse inverse");
    if (sing)
        fail(FX_NUMERICAL, "Mathematical error: the multigrid coarse operator is singular (system not "
                           "positive definite). Check for rigid body modes!");
}

void Amg::setup(const BsrStructure& S0, const double* vals0, const double* dinv0, const double* xyz, int n_nodes,
                double cell0, cudaStream_t s, AmgStats* st) {
    EventTimer timer;
    timer.start(s);
    L.clear();
    L.reserve(kMaxLevels);
    L.emplace_back();
    {
        AmgLevel& l0 = L[0];
        l0.n = n_nodes;
        l0.bs = 3;
        l0.S0 = &S0;
        l0.vals0 = vals0;
        l0.dinv0 = dinv0;
        l0.nblocks = S0.n_blocks;
    }
    // the level-0 points and their origin (cell keys of every level are taken from it)
    DBuf<double> coords, cent, Rprev, Rnext, org;
    coords.alloc(3 * (size_t)n_nodes, s);
    FX_CUDA_CHECK(cudaMemcpyAsync(coords.ptr, xyz, 3 * (size_t)n_nodes * sizeof(double), cudaMemcpyDeviceToDevice, s));
    org.alloc(3, s);
    FX_LAUNCH(k_min3, 1, 1024, 0, s, n_nodes, coords.ptr, org.ptr);
    double cell = cell0;
    for (int lev = 0;; ++lev) {
        AmgLevel& l = L[lev];
        const int64_t nd = (int64_t)l.n * l.bs;
        for (DBuf<double>* v : {&l.x, &l.b, &l.r, &l.d, &l.t}) v->alloc(nd, s);
        if (lev > 0) l.xs.alloc(nd, s);
        if (lev == 0)
            for (DBuf<float>* v : {&l.d4a, &l.d4b, &l.x4}) {
                v->alloc(4 * (size_t)l.n, s);
                v->zero(s);  // the fourth component stays 0
            }
        if (lev > 0) {
            l.dinv.alloc((size_t)l.n * 36, s);
            FX_LAUNCH(k_block_inv6, grid_for(l.n, 128), 128, 0, s, l.n, l.row_ptr.ptr, l.cols.ptr, l.vals.ptr,
                      l.dinv.ptr);
        }
        if (lev > 0 && (nd <= kCoarseMaxDof || lev + 1 >= kMaxLevels)) {
            l.coarsest = true;
            coarsest_inverse(l, s);
            break;
        }
        estimate_lmax(l, red_, s, lev == 0 ? vals0_f32_ : nullptr, false,
                      lev == 0 && kAmgEstF16 ? vals0_f16_ : nullptr, sq4_);
        // ---- aggregation by cells
        DBuf<uint64_t> keys, keys_s;
        DBuf<int32_t> ids, ids_s, head, rank1;
        keys.alloc(l.n, s);
        keys_s.alloc(l.n, s);
        ids.alloc(l.n, s);
        ids_s.alloc(l.n, s);
        FX_LAUNCH(k_cell_keys, grid_for(l.n), 256, 0, s, l.n, coords.ptr, org.ptr, 1.0 / cell, keys.ptr,
                  ids.ptr);
        cub_call([&](void* t, size_t& b) {
            return cub::DeviceRadixSort::SortPairs(t, b, keys.ptr, keys_s.ptr, ids.ptr, ids_s.ptr, l.n, 0, 63, s);
        }, tmp_, s);
        head.alloc(l.n, s);
        rank1.alloc(l.n, s);
        FX_LAUNCH(k_heads64, grid_for(l.n), 256, 0, s, l.n, keys_s.ptr, head.ptr);
        cub_call([&](void* t, size_t& b) { return cub::DeviceScan::InclusiveSum(t, b, head.ptr, rank1.ptr, l.n, s); },
                 tmp_, s);
        int na = 0;
        FX_CUDA_CHECK(cudaMemcpyAsync(&na, rank1.ptr + l.n - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        stream_wait(s, "amg aggregates");
        if (na >= l.n) {  // cells too small to aggregate: grow and retry this level
            if (l.n <= 1) fail(FX_GENERIC, "multigrid: a single block row cannot be coarsened");
            cell *= 1.5;
            --lev;
            continue;
        }
        l.n_agg = na;
        l.agg.alloc(l.n, s);
        l.agg_ptr.alloc(na + 1, s);
        FX_LAUNCH(k_agg_assign, grid_for(l.n), 256, 0, s, l.n, rank1.ptr, head.ptr, ids_s.ptr, l.agg.ptr,
                  l.agg_ptr.ptr);
        FX_CUDA_CHECK(cudaMemcpyAsync(l.agg_ptr.ptr + na, &l.n, sizeof(int), cudaMemcpyHostToDevice, s));
        l.agg_nodes = std::move(ids_s);
        cent.alloc((size_t)na * 3, s);
        FX_LAUNCH(k_agg_centroid, grid_for(na), 256, 0, s, na, l.agg_ptr.ptr, l.agg_nodes.ptr, coords.ptr, cent.ptr);
        // ---- tentative prolongator
        l.Q.alloc((size_t)nd * 6, s);
        Rnext.alloc((size_t)na * 36, s);
        FX_LAUNCH(k_agg_qr, grid_for((int64_t)na * 32), 256, 0, s, na, l.agg_ptr.ptr, l.agg_nodes.ptr, l.bs,
                  coords.ptr, cent.ptr, Rprev.ptr, l.Q.ptr, Rnext.ptr);
        // ---- Galerkin coarse matrix
        if (!l.S0) {
            l.gal_rows.alloc(l.nblocks, s);
            FX_LAUNCH(k_expand_rows, grid_for(l.n), 256, 0, s, l.n, l.row_ptr.ptr, l.gal_rows.ptr);
        }
        const FineView F = fine_view(l);
        const int nbits = bits_for(na > 1 ? na : 2);
        DBuf<uint64_t> ck, ck_s;
        DBuf<int64_t> cb, cb_s;
        ck.alloc(l.nblocks, s);
        ck_s.alloc(l.nblocks, s);
        cb.alloc(l.nblocks, s);
        cb_s.alloc(l.nblocks, s);
        FX_LAUNCH(k_coarse_keys, grid_for(l.nblocks), 256, 0, s, l.nblocks, F, l.agg.ptr, nbits, ck.ptr, cb.ptr);
        cub_call([&](void* t, size_t& b) {
            return cub::DeviceRadixSort::SortPairs(t, b, ck.ptr, ck_s.ptr, cb.ptr, cb_s.ptr, l.nblocks, 0, 2 * nbits,
                                                   s);
        }, tmp_, s);
        ck.release();
        cb.release();
        DBuf<int32_t> chead, cbid;
        chead.alloc(l.nblocks, s);
        cbid.alloc(l.nblocks, s);
        FX_LAUNCH(k_heads_u64, grid_for(l.nblocks), 256, 0, s, l.nblocks, ck_s.ptr, chead.ptr);
        cub_call([&](void* t, size_t& b) {
            return cub::DeviceScan::InclusiveSum(t, b, chead.ptr, cbid.ptr, l.nblocks, s);
        }, tmp_, s);
        int ncb = 0;
        FX_CUDA_CHECK(cudaMemcpyAsync(&ncb, cbid.ptr + l.nblocks - 1, sizeof(int), cudaMemcpyDeviceToHost, s));
        stream_wait(s, "amg coarse blocks");
        L.emplace_back();
        AmgLevel& c = L.back();
        AmgLevel& lf = L[L.size() - 2];
        c.n = na;
        c.bs = 6;
        c.nblocks = ncb;
        DBuf<int64_t> seg;
        DBuf<int32_t> crow, cnt;
        seg.alloc(ncb + 1, s);
        crow.alloc(ncb, s);
        c.cols.alloc(ncb, s);
        cnt.alloc(na, s);
        cnt.zero(s);
        FX_LAUNCH(k_coarse_blocks, grid_for(lf.nblocks), 256, 0, s, lf.nblocks, ck_s.ptr, cbid.ptr, nbits, seg.ptr,
                  crow.ptr, c.cols.ptr, cnt.ptr);
        const int64_t nbf = lf.nblocks;
        FX_CUDA_CHECK(cudaMemcpyAsync(seg.ptr + ncb, &nbf, sizeof(int64_t), cudaMemcpyHostToDevice, s));
        c.row_ptr.alloc(na + 1, s);
        FX_CUDA_CHECK(cudaMemsetAsync(c.row_ptr.ptr, 0, sizeof(int32_t), s));
        cub_call([&](void* t, size_t& b) {
            return cub::DeviceScan::InclusiveSum(t, b, cnt.ptr, c.row_ptr.ptr + 1, na, s);
        }, tmp_, s);
        c.vals.alloc((size_t)ncb * 36, s);
        lf.gal_seg = std::move(seg);  // kept for refresh()
        lf.gal_blk = std::move(cb_s);
        galerkin(lf, c, s);
        stream_wait(s, "amg galerkin");
        // next level points and near-null-space
        coords = std::move(cent);
        Rprev = std::move(Rnext);
        cell *= 2.0;
    }
    if (L.size() > 2) {  // K-cycle work vectors on the first coarse level
        AmgLevel& l1 = L[1];
        const int64_t nd1 = (int64_t)l1.n * l1.bs;
        for (auto& v : l1.kc) v.alloc(nd1, s);
        l1.kcs.alloc(8, s);
        l1.kcs.zero(s);
    }
    if (st) {
        st->levels = (int)L.size();
        st->sizes.clear();
        for (auto& l : L) st->sizes.push_back(l.n * l.bs);
        st->setup_ms = timer.stop_ms(s);
    }
}

void Amg::refresh(const double* vals0, const double* dinv0, cudaStream_t s, AmgStats* st) {
    EventTimer timer;
    timer.start(s);
    L[0].vals0 = vals0;
    L[0].dinv0 = dinv0;
    for (size_t lev = 0; lev < L.size(); ++lev) {  // the numeric steps of setup(), in its order
        AmgLevel& l = L[lev];
        if (lev > 0)
            FX_LAUNCH(k_block_inv6, grid_for(l.n, 128), 128, 0, s, l.n, l.row_ptr.ptr, l.cols.ptr, l.vals.ptr,
                      l.dinv.ptr);
        if (l.coarsest) {
            coarsest_inverse(l, s);
            break;
        }
        estimate_lmax(l, red_, s, lev == 0 ? vals0_f32_ : nullptr, true,
                      lev == 0 && kAmgEstF16 ? vals0_f16_ : nullptr, sq4_);
        galerkin(l, L[lev + 1], s);
    }
    if (st) {
        st->levels = (int)L.size();
        st->sizes.clear();
        for (auto& l : L) st->sizes.push_back(l.n * l.bs);
        st->setup_ms = timer.stop_ms(s);
    }
}

// Chebyshev polynomial smoother on D^-1 A over [lmax/30, lmax] (degree = steps):
// d_1 = D^-1 r_0 / theta, then r_k = r_{k-1} - A d_k,
// d_{k+1} = rho_k rho_{k-1} d_k + (2 rho_k / delta) D^-1 r_k with
// rho_0 = delta / theta, rho_k = 1 / (2 theta / delta - rho_{k-1}); x += every d.
struct ChebCoef {
    double c2_start;
    double c1[8], c2[8];
};
// kind 1: fourth-kind Chebyshev smoother (Lottes, "Optimal polynomial smoothers
// for multigrid V-cycles", Numer. Linear Algebra Appl. 2023): d_1 = 4/(3 rho)
// D^-1 r_0, d_k = (2k-3)/(2k+1) d_{k-1} + (8k-4)/((2k+1) rho) D^-1 r_{k-1}, rho =
// the lambda_max estimate; no lower eigenvalue bound needed.
static ChebCoef cheb_coef(double lmax, int degree, int kind, double ratio) {
    if (kind == 1) {
        ChebCoef k{};
        k.c2_start = 4.0 / (3.0 * lmax);
        for (int s = 1; s < degree; ++s) {
            const int i = s + 1;  // step index of the recurrence (the start is step 1)
            k.c1[s] = (2.0 * i - 3.0) / (2.0 * i + 1.0);
            k.c2[s] = (8.0 * i - 4.0) / ((2.0 * i + 1.0) * lmax);
        }
        return k;
    }
    const double lmin = lmax / ratio;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    const double sigma = theta / delta;
    ChebCoef k{};
    k.c2_start = 1.0 / theta;
    double rho = 1.0 / sigma;
    for (int s = 1; s < degree; ++s) {
        const double rho1 = 1.0 / (2.0 * sigma - rho);
        k.c1[s] = rho1 * rho;
        k.c2[s] = 2.0 * rho1 / delta;
        rho = rho1;
    }
    return k;
}

static LnOp ln_op(const AmgLevel& l) {
    LnOp o{};
    o.n = l.n;
    o.row_ptr = l.row_ptr.ptr;
    o.cols = l.cols.ptr;
    o.vals = l.vals.ptr;
    o.dinv = l.dinv.ptr;
    return o;
}

// Cycle at a coarse level (6x6 blocks) for A x = b (b and x of that level's size):
// Chebyshev pre-smoothing from x = 0 into the scratch iterate xs (start kernel,
// then SpMVs fused with the updates), the residual, the coarse correction added
// to xs, and post-smoothing that reads xs and writes the result into x.
CoarseStart Amg::coarse_start(int m) const {
    CoarseStart cs{};
    const AmgLevel& c = L[m];
    if (c.coarsest || (kcycle_ && m == 1)) return cs;  // dense solve; K-cycle calls the cycle on other vectors
    cs.dinv = c.dinv.ptr;
    cs.r = c.r.ptr;
    cs.d = c.d.ptr;
    cs.xs = c.xs.ptr;
    cs.c2 = cheb_coef(c.lmax, degree_, cheb_kind_, cheb_ratio_).c2_start;
    return cs;
}

void Amg::cycle(int lev, const double* b, double* x, cudaStream_t s, bool started) {
    AmgLevel& l = L[lev];
    const int64_t nd = (int64_t)l.n * l.bs;
    if (l.coarsest) {
        FX_LAUNCH(k_dense_matvec, grid_for(nd * 32, kLnThreads), kLnThreads, 0, s, (int)nd, l.dense_inv.ptr, b, x);
        return;
    }
    AmgLevel& c = L[lev + 1];
    // coarse_row6 reads the 6x6 blocks and the gathered 6-vectors as 16-byte pairs
    if ((reinterpret_cast<uintptr_t>(l.vals.ptr) | reinterpret_cast<uintptr_t>(l.d.ptr) |
         reinterpret_cast<uintptr_t>(l.t.ptr) | reinterpret_cast<uintptr_t>(l.xs.ptr)) & 15)
        fail(FX_GENERIC, "multigrid: coarse-level buffers not 16-byte aligned");
    const ChebCoef k = cheb_coef(l.lmax, degree_, cheb_kind_, cheb_ratio_);
    const unsigned grid = grid_for((int64_t)l.n * 32, kLnThreads);
    double* dA = l.d.ptr;
    double* dB = l.t.ptr;
    double* xs = l.xs.ptr;
    if (!started)
        FX_LAUNCH(k_cheb_start, grid_for(l.n), 256, 0, s, l.n, l.bs, l.dinv.ptr, b, l.r.ptr, dA, xs, k.c2_start);
    for (int st = 1; st < degree_; ++st) {
        LnOp o = ln_op(l);
        o.v = dA;
        o.r = l.r.ptr;
        o.d_out = dB;
        o.xo = xs;
        o.c1 = k.c1[st];
        o.c2 = k.c2[st];
        FX_LAUNCH(k_ln_op<kL0ChebK>, grid, kLnThreads, 0, s, o);
        std::swap(dA, dB);
    }
    {
        LnOp o = ln_op(l);
        o.v = dA;
        o.r = l.r.ptr;
        FX_LAUNCH(k_ln_op<kL0RUpd>, grid, kLnThreads, 0, s, o);  // r = b - A xs
    }
    FX_LAUNCH(k_restrict, grid_for((int64_t)l.n_agg * 32, kLnThreads), kLnThreads, 0, s, l.n_agg, l.agg_ptr.ptr, l.agg_nodes.ptr, l.bs,
              l.Q.ptr, l.r.ptr, c.b.ptr, coarse_start(lev + 1));
    coarse(lev + 1, s);
    FX_LAUNCH(k_prolong, grid_for(nd), 256, 0, s, (int)nd, l.bs, l.agg.ptr, l.Q.ptr, c.x.ptr, xs, alpha_);
    {
        LnOp o = ln_op(l);
        o.v = xs;
        o.b = b;
        o.r = l.r.ptr;
        o.d_out = dA;
        o.xo = x;
        o.c2 = k.c2_start;
        FX_LAUNCH(k_ln_op<kL0Cheb0>, grid, kLnThreads, 0, s, o);
    }
    for (int st = 1; st < degree_; ++st) {
        LnOp o = ln_op(l);
        o.v = dA;
        o.r = l.r.ptr;
        o.d_out = dB;
        o.xo = x;
        o.c1 = k.c1[st];
        o.c2 = k.c2[st];
        FX_LAUNCH(k_ln_op<kL0ChebK>, grid, kLnThreads, 0, s, o);
        std::swap(dA, dB);
    }
}

// Coarse correction at level m: L[m].x ~ A_m^-1 L[m].b, by a K-cycle at the first
// coarse level (when it is not the coarsest) and V-cycles below.
void Amg::coarse(int m, cudaStream_t s) {
    AmgLevel& l = L[m];
    if (!(kcycle_ && m == 1 && !l.coarsest)) {
        cycle(m, l.b.ptr, l.x.ptr, s, coarse_start(m).dinv != nullptr);
        return;
    }
    const int64_t nd = (int64_t)l.n * l.bs;
    double *z1 = l.kc[0].ptr, *v1 = l.kc[1].ptr, *r = l.kc[2].ptr, *z2 = l.kc[3].ptr, *v2 = l.kc[4].ptr;
    cycle(m, l.b.ptr, z1, s);
    level_spmv(l, z1, nullptr, v1, s);
    FX_LAUNCH(k_kcycle1, 1, 1024, 0, s, nd, l.b.ptr, z1, v1, l.x.ptr, r, l.kcs.ptr);
    cycle(m, r, z2, s);
    level_spmv(l, z2, nullptr, v2, s);
    FX_LAUNCH(k_kcycle2, 1, 1024, 0, s, nd, z1, v1, z2, v2, r, l.x.ptr, l.kcs.ptr);
}

// Level 0 with the fused operators: pre-smoothing from x = 0 (one elementwise
// start, degree-1 fused steps, one fused residual update), coarse correction,
// post-smoothing written straight into z. With S != null the last step also
// reduces r.z and beta for the outer CG.
template <typename VT>
void Amg::vcycle0(const VT* vals, const double* b, double* z, double* S, double* part, int* counter,
                  const double* zold, cudaStream_t s, bool started) {
    AmgLevel& l = L[0];
    AmgLevel& c = L[1];
    const int64_t nd = (int64_t)l.n * 3;
    const ChebCoef k = cheb_coef(l.lmax, degree_, cheb_kind_, cheb_ratio_);
    const unsigned grid = l0_grid(l.n, std::is_same<VT, __half>::value);
    // FP32 or FP16 values: the smoother's gathered vectors are FP32 (float4 per node),
    // with FP16 values FP16 directions (kL0H16Vec) scaled by the V-cycle's power of two
    constexpr bool g32 = !std::is_same<VT, double>::value;
    float* hs = std::is_same<VT, __half>::value ? h16_scale_slot() : nullptr;
    double* dA = l.d.ptr;
    double* dB = l.t.ptr;
    float4* dA4 = reinterpret_cast<float4*>(l.d4a.ptr);
    float4* dB4 = reinterpret_cast<float4*>(l.d4b.ptr);
    float4* x4 = reinterpret_cast<float4*>(l.x4.ptr);
    if (!started)
        FX_LAUNCH(k_l0_cheb_start, grid_for(l.n), 256, 0, s, l.n, l.dinv0, b, l.r.ptr, dA, g32 ? dA4 : nullptr,
                  l.x.ptr, k.c2_start, sq4_, rdr_, hs);
    auto op = [&]() {
        L0Op<VT> o = l0_op<VT>(l, vals);
        o.sq4 = sq4_;
        o.hs = hs;
        return o;
    };
    for (int st = 1; st < degree_; ++st) {
        L0Op<VT> o = op();
        o.v = dA;
        o.v4 = dA4;
        o.r = l.r.ptr;
        o.d_out = dB;
        o.d4_out = reinterpret_cast<float*>(dB4);
        o.xo = l.x.ptr;
        o.c1 = k.c1[st];
        o.c2 = k.c2[st];
        FX_LAUNCH((k_l0_op<VT, kL0ChebK, g32>), grid, 256, 0, s, o);
        std::swap(dA, dB);
        std::swap(dA4, dB4);
    }
    {
        L0Op<VT> o = op();
        o.v = dA;
        o.v4 = dA4;
        o.r = l.r.ptr;
        FX_LAUNCH((k_l0_op<VT, kL0RUpd, g32>), grid, 256, 0, s, o);  // r = b - A x
    }
    if (fused_coarse_ && !kcycle_ && desc_.ptr) {  // restriction, coarse levels, prolongation: one launch
        launch_coarse_grid(desc_.ptr, gbar_.ptr, gflag_, g32, degree_, alpha_, s);
    } else {
        FX_LAUNCH(k_restrict, grid_for((int64_t)l.n_agg * 32, kLnThreads), kLnThreads, 0, s, l.n_agg, l.agg_ptr.ptr, l.agg_nodes.ptr, 3,
                  l.Q.ptr, l.r.ptr, c.b.ptr, coarse_start(1));
        coarse(1, s);
        if (g32)
            FX_LAUNCH(k_prolong0, grid_for(l.n), 256, 0, s, l.n, l.agg.ptr, l.Q.ptr, c.x.ptr, l.x.ptr, x4, alpha_,
                      sq4_);
        else FX_LAUNCH(k_prolong, grid_for(nd), 256, 0, s, (int)nd, 3, l.agg.ptr, l.Q.ptr, c.x.ptr, l.x.ptr, alpha_);
    }
    for (int st = 0; st < degree_; ++st) {
        L0Op<VT> o = op();
        o.b = b;
        o.r = l.r.ptr;
        o.xo = z;
        if (st == 0) {  // from the iterate: r = b - A x, d = D^-1 r / theta, z = x + d
            o.v = l.x.ptr;
            o.v4 = x4;
            o.d_out = dA;
            o.d4_out = reinterpret_cast<float*>(dA4);
            o.c2 = k.c2_start;
        } else {
            o.v = dA;
            o.v4 = dA4;
            o.d_out = dB;
            o.d4_out = reinterpret_cast<float*>(dB4);
            o.c1 = k.c1[st];
            o.c2 = k.c2[st];
        }
        if (st == degree_ - 1 && S) {
            if (2 * (int64_t)grid > part_slots_)
                fail(FX_GENERIC, "multigrid: partial-sum buffer smaller than the smoother grid");
            o.dot = 2;
            o.zold = zold;
            o.part = part;
            o.counter = counter;
            o.S = S;
        }
        if (st == 0) FX_LAUNCH((k_l0_op<VT, kL0Cheb0, g32>), grid, 256, 0, s, o);
        else {
            FX_LAUNCH((k_l0_op<VT, kL0ChebK, g32>), grid, 256, 0, s, o);
            std::swap(dA, dB);
            std::swap(dA4, dB4);
        }
    }
}

void Amg::apply(const double* r, double* z, double* S, double* part, int* counter, const double* zold,
                cudaStream_t s, bool started) {
    if (vals0_f16_) vcycle0<__half>(vals0_f16_, r, z, S, part, counter, zold, s, started);
    else if (vals0_f32_) vcycle0<float>(vals0_f32_, r, z, S, part, counter, zold, s, started);
    else vcycle0<double>(L[0].vals0, r, z, S, part, counter, zold, s, started);
}

Amg::Start0 Amg::start0() const {
    const AmgLevel& l = L[0];
    Start0 o{};
    o.r = l.r.ptr;
    o.x = l.x.ptr;
    o.d = l.d.ptr;
    o.d4 = vals0_f32_ || vals0_f16_ ? reinterpret_cast<float4*>(l.d4a.ptr) : nullptr;
    o.c2 = cheb_coef(l.lmax, degree_, cheb_kind_, cheb_ratio_).c2_start;
    o.sq4 = sq4_;
    o.hs = vals0_f16_ ? h16_scale_slot() : nullptr;
    return o;
}

// the scale slot of FP16 smoother directions (null: the directions are FP32, or unscaled)
float* Amg::h16_scale_slot() const { return kL0H16Vec && rdr_ ? hs_ : nullptr; }

// ------------------------------------------------------------------ AMG-preconditioned CG (FP64)

double profile_smoother_op(const BsrStructure& S, const double* vals64, const double* dinv64, bool fp32, bool fp16,
                           int reps, cudaStream_t s, double* bytes) {
    fp32 = fp32 || fp16;
    const int n = S.n_rows;
    const int64_t nd = 3 * (int64_t)n;
    DBuf<float> v32;
    DBuf<__half> v16;
    DBuf<float4> sq4;
    if (fp16) {
        sq4.alloc((size_t)n, s);
        FX_LAUNCH(k_diag_sqrt, grid_for(n), 256, 0, s, n, S.goff.ptr, S.diag_k.ptr, vals64, sq4.ptr);
        v16.alloc((size_t)S.n_groups * 36, s);
        FX_LAUNCH(k_vals_to_f16, grid_for((int64_t)n * 32), 256, 0, s, n, S.goff.ptr, S.cols.ptr, vals64, sq4.ptr,
                  v16.ptr);
    } else if (fp32) {
        const int64_t nv = (int64_t)S.n_groups * 36;
        v32.alloc(nv, s);
        FX_LAUNCH(k_f64_to_f32, 148 * 8, 256, 0, s, nv, vals64, v32.ptr);
    }
    DBuf<double> v, r, d, xo;
    for (DBuf<double>* b : {&v, &r, &d, &xo}) {
        b->alloc(nd, s);
        FX_LAUNCH(k_fill_hash, grid_for(nd), 256, 0, s, nd, b->ptr);
    }
    DBuf<float> v4, d4;  // FP32 smoother vectors (float4 per node), as in the V-cycle
    if (fp32) {
        v4.alloc(4 * (size_t)n, s);
        d4.alloc(4 * (size_t)n, s);
        v4.zero(s);
        d4.zero(s);
    }
    AmgLevel l;
    l.n = n;
    l.S0 = &S;
    l.vals0 = vals64;
    l.dinv0 = dinv64;
    const unsigned grid = l0_grid(n, fp16);
    auto launch = [&]() {
        if (fp16) {
            L0Op<__half> o = l0_op<__half>(l, v16.ptr);
            o.v = v.ptr;
            o.v4 = reinterpret_cast<const float4*>(v4.ptr);
            o.r = r.ptr;
            o.d_out = d.ptr;
            o.d4_out = d4.ptr;
            o.xo = xo.ptr;
            o.c1 = 0.5;
            o.c2 = 1e-9;
            o.sq4 = sq4.ptr;
            FX_LAUNCH((k_l0_op<__half, kL0ChebK, true>), grid, 256, 0, s, o);
        } else if (fp32) {
            L0Op<float> o = l0_op<float>(l, v32.ptr);
            o.v = v.ptr;
            o.v4 = reinterpret_cast<const float4*>(v4.ptr);
            o.r = r.ptr;
            o.d_out = d.ptr;
            o.d4_out = d4.ptr;
            o.xo = xo.ptr;
            o.c1 = 0.5;
            o.c2 = 1e-9;
            FX_LAUNCH((k_l0_op<float, kL0ChebK, true>), grid, 256, 0, s, o);
        } else {
            L0Op<double> o = l0_op<double>(l, vals64);
            o.v = v.ptr;
            o.r = r.ptr;
            o.d_out = d.ptr;
            o.xo = xo.ptr;
            o.c1 = 0.5;
            o.c2 = 1e-9;
            FX_LAUNCH((k_l0_op<double, kL0ChebK>), grid, 256, 0, s, o);
        }
    };
    for (int k = 0; k < 3; ++k) launch();
    EventTimer t;
    t.start(s);
    for (int k = 0; k < reps; ++k) launch();
    const double ms = t.stop_ms(s) / reps;
    // compulsory bytes: matrix values + column indices once, row offsets, and per
    // node the gathered direction (24 B FP64 / 16 B float4), r read+write (48), the
    // new direction (24 / 16), iterate read+write (48) and the 3x3 block inverse (72)
    // (FP16: 2-byte values, the 16-byte scales of each row, and with kL0H16Vec 8-byte
    // directions gathered and written)
    const double vb = fp16 ? 2.0 : (fp32 ? 4.0 : 8.0);
    const double per_node = fp16 && kL0H16Vec ? 184.0 : (fp32 ? 200.0 : 216.0);
    *bytes = (double)S.n_blocks * (9.0 * vb + 4.0) + 4.0 * (n + 1) + per_node * n + (fp16 ? 16.0 * n : 0.0);
    return ms;
}

void Amg::describe(ClInst& o) const {
    const AmgLevel& l0 = L[0];
    o.n = l0.n;
    o.levels = (int)L.size();
    o.goff = l0.S0->goff.ptr;
    o.cols = l0.S0->cols.ptr;
    o.vals64 = l0.vals0;
    o.vals32 = vals0_f32_;
    o.dinv0 = l0.dinv0;
    o.sq4 = sq4_;
    o.agg = l0.agg.ptr;
    o.agg_ptr = l0.agg_ptr.ptr;
    o.agg_nodes = l0.agg_nodes.ptr;
    o.Q = l0.Q.ptr;
    o.n_agg = l0.n_agg;
    o.lr = l0.r.ptr;
    o.lx = l0.x.ptr;
    o.ld = l0.d.ptr;
    o.lt = l0.t.ptr;
    o.d4a = l0.d4a.ptr;
    o.d4b = l0.d4b.ptr;
    o.x4 = l0.x4.ptr;
    const ChebCoef k0 = cheb_coef(l0.lmax, degree_, cheb_kind_, cheb_ratio_);
    o.c2_start = k0.c2_start;
    for (int i = 0; i < 8; ++i) {
        o.c1[i] = k0.c1[i];
        o.c2[i] = k0.c2[i];
    }
    for (size_t m = 1; m < L.size() && m < (size_t)kClMaxLevels; ++m) {
        const AmgLevel& l = L[m];
        ClLevel& c = o.lev[m];
        c.n = l.n;
        c.coarsest = l.coarsest ? 1 : 0;
        c.n_agg = l.n_agg;
        c.row_ptr = l.row_ptr.ptr;
        c.cols = l.cols.ptr;
        c.vals = l.vals.ptr;
        c.dinv = l.dinv.ptr;
        c.dense_inv = l.dense_inv.ptr;
        c.agg = l.agg.ptr;
        c.agg_ptr = l.agg_ptr.ptr;
        c.agg_nodes = l.agg_nodes.ptr;
        c.Q = l.Q.ptr;
        c.x = l.x.ptr;
        c.b = l.b.ptr;
        c.r = l.r.ptr;
        c.d = l.d.ptr;
        c.t = l.t.ptr;
        c.xs = l.xs.ptr;
        for (const void* q : {(const void*)c.vals, (const void*)c.x, (const void*)c.b, (const void*)c.d,
                              (const void*)c.t, (const void*)c.xs})
            if (reinterpret_cast<uintptr_t>(q) & 15)  // coarse_row6's 16-byte loads
                fail(FX_GENERIC, "multigrid: coarse-level buffers not 16-byte aligned");
        if (!l.coarsest) {
            const ChebCoef k = cheb_coef(l.lmax, degree_, cheb_kind_, cheb_ratio_);
            c.c2_start = k.c2_start;
            for (int i = 0; i < 8; ++i) {
                c.c1[i] = k.c1[i];
                c.c2[i] = k.c2[i];
            }
        }
    }
}

void AmgPcg::prepare(const BsrStructure& S, const double* vals64, const double* dinv64, const double* xyz,
                     double cell0, const PcgOptions& opt, cudaStream_t s, AmgStats* st, bool reuse, bool persistent) {
    const int n = S.n_rows;
    const int64_t nd = 3 * (int64_t)n;
    if (opt.amg_degree < 1 || opt.amg_degree > 8) fail(FX_INVALID_ARGUMENT, "multigrid smoother degree must be 1..8");
    const float* v32 = nullptr;
    const bool f16 = opt.amg_fp32 && opt.amg_fp16 && !persistent;
    if (f16) {  // FP16 values of S A S and the scales
        sq4_.alloc((size_t)n, s);
        FX_LAUNCH(k_diag_sqrt, grid_for(n), 256, 0, s, n, S.goff.ptr, S.diag_k.ptr, vals64, sq4_.ptr);
        vals16_.alloc((size_t)S.n_groups * 36, s);
        FX_LAUNCH(k_vals_to_f16, grid_for((int64_t)n * 32), 256, 0, s, n, S.goff.ptr, S.cols.ptr, vals64, sq4_.ptr,
                  vals16_.ptr);
    }
    // FP32 values: the FP32 smoother's; with the FP16 smoother only when the level-0
    // eigenvalue estimate reads them (kAmgEstF16 off) instead of the FP16 values
    if (opt.amg_fp32 && (!f16 || !kAmgEstF16)) {
        const int64_t nv = (int64_t)S.n_groups * 36;
        vals32_.alloc(nv, s);
        FX_LAUNCH(k_f64_to_f32, 148 * 8, 256, 0, s, nv, vals64, vals32_.ptr);
        v32 = vals32_.ptr;
    }
    amg.set_smoother(opt.amg_degree, v32);  // before setup: its eigenvalue estimate uses v32
    if (f16) amg.set_smoother_f16(vals16_.ptr, sq4_.ptr);
    if (reuse && amg.built_for == S.id && !amg.L.empty() && amg.L[0].n == n) {
        amg.refresh(vals64, dinv64, s, st);
    } else {
        amg.built_for = 0;  // (a failed setup leaves nothing to reuse)
        amg.setup(S, vals64, dinv64, xyz, n, cell0, s, st);
        amg.built_for = S.id;
    }
    amg.set_cycle(opt.amg_kcycle);
    amg.set_smoother_kind(opt.amg_cheb_kind);
    amg.set_overcorrect(opt.amg_overcorrect);
    amg.set_cheb_ratio(opt.amg_cheb_ratio);
    S_ = &S;
    vals64_ = vals64;
    dinv64_ = dinv64;
    r_.alloc(nd, s);
    z_.alloc(nd, s);
    p_.alloc(nd, s);
    q_.alloc(nd, s);
    const int nb = 296;
    part_.alloc(std::max<int64_t>(nb, l0_part_slots(n)), s);
    amg.set_part_slots((int64_t)part_.n);
    sc_.alloc(8, s);
    sc_.zero(s);
    hs_.alloc(2, s);
    amg.set_smoother_scale(f16 ? sc_.ptr + 2 : nullptr, f16 ? hs_.ptr : nullptr);  // S[2] = r.D^-1 r
    counter_.alloc(1, s);
    counter_.zero(s);
    // the fused coarse cycle reads the hierarchy from a device descriptor, re-uploaded
    // after every setup / refresh (new eigenvalue estimates, new Chebyshev coefficients);
    // a barrier timeout sets S[7]
    amg.set_fused_coarse(opt.amg_fused_coarse && !opt.amg_kcycle, sc_.ptr + 7);
    if (opt.amg_fused_coarse && !opt.amg_kcycle) amg.upload_descriptor(s);
}

void Amg::upload_descriptor(cudaStream_t s) {
    ClInst h{};
    describe(h);
    desc_.upload(&h, 1, s);
    gbar_.alloc(1, s);
    gbar_.zero(s);
}

ClInst AmgPcg::describe(const double* b, double* x) const {
    ClInst o{};
    amg.describe(o);
    o.b = b;
    o.x = x;
    o.r = r_.ptr;
    o.z = z_.ptr;
    o.p = p_.ptr;
    o.q = q_.ptr;
    return o;
}

double AmgPcg::true_relres(const double* b, const double* x, cudaStream_t s) {
    const int n = S_->n_rows;
    const int nb = 296;
    level_spmv(amg.L[0], x, b, q_.ptr, s);
    FX_LAUNCH(k_rdr_part, nb, 256, 0, s, n, q_.ptr, dinv64_, part_.ptr);
    FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 1);
    FX_LAUNCH(k_rdr_part, nb, 256, 0, s, n, b, dinv64_, part_.ptr);
    FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr + 4, 1);
    double h[8];
    FX_CUDA_CHECK(cudaMemcpyAsync(h, sc_.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
    stream_wait(s, "amg true residual");
    return h[6] > 0.0 ? std::sqrt(std::max(0.0, h[2]) / h[6]) : 0.0;
}

int AmgPcg::solve(const BsrStructure& S, const double* vals64, const double* dinv64, const double* xyz,
                  double cell0, const double* b, double* x, const PcgOptions& opt, cudaStream_t s,
                  int64_t* launches, long long* iters, double* relres, AmgStats* st, bool reuse) {
    const int n = S.n_rows;
    const int64_t nd = 3 * (int64_t)n;
    prepare(S, vals64, dinv64, xyz, cell0, opt, s, st, reuse);
    const int nb = 296;
    const unsigned g0 = l0_grid(n, false, true);  // q = K p
    if (2 * (int64_t)g0 > (int64_t)part_.n) fail(FX_GENERIC, "multigrid: partial-sum buffer smaller than the CG grid");
    FX_CUDA_CHECK(cudaMemsetAsync(x, 0, nd * sizeof(double), s));
    FX_CUDA_CHECK(cudaMemcpyAsync(r_.ptr, b, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    // ||b||_D, z = V(b) with r.z, p = z
    FX_LAUNCH(k_rdr_part, nb, 256, 0, s, n, r_.ptr, dinv64, part_.ptr);
    FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 1);
    FX_CUDA_CHECK(cudaMemcpyAsync(sc_.ptr + 3, sc_.ptr + 2, sizeof(double), cudaMemcpyDeviceToDevice, s));
    z2_.alloc(nd, s);
    amg.apply(r_.ptr, z_.ptr, nullptr, nullptr, nullptr, nullptr, s);
    FX_LAUNCH(k_dot_part, nb, 256, 0, s, nd, r_.ptr, z_.ptr, part_.ptr);
    FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 3);
    FX_CUDA_CHECK(cudaMemcpyAsync(p_.ptr, z_.ptr, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    const AmgLevel& l0 = amg.L[0];
    // flexible CG (the K-cycle makes the preconditioner vary slightly between
    // iterations): z alternates between two buffers so that r.z_old is at hand
    // the CG update and p = z + beta p with a thread per node / entry (all of them in
    // flight at once), the update's grid within the partial-sum slots it reduces into
    const unsigned gu = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(n), (int64_t)part_.n));
    const unsigned gx = (unsigned)std::min<int64_t>(grid_for(nd), 4096);
    int parity = 0;
    auto iteration = [&]() {
        double* zn = parity ? z_.ptr : z2_.ptr;
        const double* zo = parity ? z2_.ptr : z_.ptr;
        parity ^= 1;
        L0Op<double> o = l0_op<double>(l0, vals64);
        o.v = p_.ptr;
        o.y = q_.ptr;
        o.dot = 1;
        o.part = part_.ptr;
        o.counter = counter_.ptr;
        o.S = sc_.ptr;
        FX_LAUNCH((k_l0_op<double, kL0Apply>), g0, 256, 0, s, o);  // q = A p, alpha
        const Amg::Start0 s0 = amg.start0();
        FX_LAUNCH(k_amg_update_start, gu, 256, 0, s, n, sc_.ptr, p_.ptr, q_.ptr, x, r_.ptr, dinv64, part_.ptr,
                  counter_.ptr, s0.r, s0.x, s0.d, s0.d4, s0.c2, s0.sq4, s0.hs);  // x, r, r.D^-1 r; the V-cycle's first step
        amg.apply(r_.ptr, zn, sc_.ptr, part_.ptr, counter_.ptr, amg.kcycle() ? zo : nullptr, s, true);  // z, r.z, beta
        FX_LAUNCH(k_xpby, gx, 256, 0, s, nd, zn, sc_.ptr, p_.ptr);
    };
    // Four iterations per graph replay between host checks. (A device-side loop
    // as a WHILE graph node, one or four iterations per body, measured 1-7 %
    // slower per iteration on B200 than these host-polled replays.)
    const int per_poll = 4;
    cudaGraphExec_t gexec = nullptr;
    int64_t per_iter_launches = 0;
    if (opt.graphs && !debug_sync()) {
        cudaGraph_t g;
        int64_t count = 0;
        int64_t* saved = g_launch_counter;
        g_launch_counter = &count;
        FX_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        for (int k = 0; k < per_poll; ++k) iteration();
        const cudaError_t ce = cudaStreamEndCapture(s, &g);
        g_launch_counter = saved;
        FX_CUDA_CHECK(ce);
        per_iter_launches = count;
        FX_CUDA_CHECK(cudaGraphInstantiate(&gexec, g, 0));
        cudaGraphDestroy(g);
    }
    double h[8];
    long long it = 0;
    int rc = FX_OK;
    const double rtol2 = opt.rtol * opt.rtol;
    while (true) {
        FX_CUDA_CHECK(cudaMemcpyAsync(h, sc_.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
        stream_wait(s, "amg pcg poll");
        if (h[7] != 0.0) fail(FX_TIMEOUT, "multigrid: a grid barrier of the coarse cycle timed out");
        if (h[6] != 0.0) {
            rc = FX_NUMERICAL;
            break;
        }
        if (h[3] <= 0.0 || h[2] <= rtol2 * h[3]) break;
        if (it >= opt.max_iter) {
            rc = FX_CONVERGENCE;
            break;
        }
        if (gexec) {
            FX_CUDA_CHECK(cudaGraphLaunch(gexec, s));
            if (launches) *launches += per_iter_launches;
        } else {
            for (int k = 0; k < per_poll; ++k) iteration();
        }
        it += per_poll;
    }
    if (gexec) cudaGraphExecDestroy(gexec);
    // true residual of the assembled FP64 system in the block-Jacobi norm
    level_spmv(l0, x, b, q_.ptr, s);
    FX_LAUNCH(k_rdr_part, nb, 256, 0, s, n, q_.ptr, dinv64, part_.ptr);
    FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 1);
    FX_CUDA_CHECK(cudaMemcpyAsync(h, sc_.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
    stream_wait(s, "amg pcg final");
    if (iters) *iters = it;
    if (relres) *relres = h[3] > 0.0 ? std::sqrt(std::max(0.0, h[2]) / h[3]) : 0.0;
    return rc;
}

// A kernel of this file's module (preload_kernels() loads all of the module's kernels).
const void* kernels_anchor_amg() { return reinterpret_cast<const void*>(&k_xpby); }

}  // namespace fx
