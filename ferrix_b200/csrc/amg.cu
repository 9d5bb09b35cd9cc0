// Aggregation multigrid setup and V-cycle (see amg.hpp).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "amg.hpp"

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

__global__ void k_cell_keys(int n, const double* __restrict__ c, double ox, double oy, double oz, double inv_cell,
                            uint64_t* __restrict__ keys, int32_t* __restrict__ ids) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
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
    __device__ __forceinline__ double val(int64_t b, int i, int r, int c) const {
        if (bs == 6) return vals[b * 36 + r * 6 + c];
        int k = (int)(b - row_ptr[i]);
        int64_t g0 = goff[i];
        int ng = goff[i + 1] - (int)g0;
        return vals[(g0 * 9 + (int64_t)(3 * r + c) * ng + k / 4) * 4 + (k & 3)];
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

// coarse block = sum over its fine blocks of Q_i^T A_ij Q_j (fixed order)
__global__ void k_galerkin(int64_t ncb, const int64_t* __restrict__ seg, const int64_t* __restrict__ sorted_b,
                           FineView F, const double* __restrict__ Q, double* __restrict__ cvals) {
    int64_t cb = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (cb >= ncb) return;
    const int bs = F.bs;
    double acc[36];
    for (int k = 0; k < 36; ++k) acc[k] = 0.0;
    for (int64_t s = seg[cb]; s < seg[cb + 1]; ++s) {
        int64_t b = sorted_b[s];
        int i = F.blk_row[b];
        int j = F.col(b, i);
        const double* Qi = Q + (size_t)i * bs * 6;
        const double* Qj = Q + (size_t)j * bs * 6;
        double T[6 * 6];  // A_ij Q_j (bs x 6)
        for (int r = 0; r < bs; ++r)
            for (int c = 0; c < 6; ++c) {
                double t = 0.0;
                for (int k = 0; k < bs; ++k) t += F.val(b, i, r, k) * Qj[k * 6 + c];
                T[r * 6 + c] = t;
            }
        for (int r = 0; r < 6; ++r)
            for (int c = 0; c < 6; ++c) {
                double t = 0.0;
                for (int k = 0; k < bs; ++k) t += Qi[k * 6 + r] * T[k * 6 + c];
                acc[r * 6 + c] += t;
            }
    }
    for (int k = 0; k < 36; ++k) cvals[cb * 36 + k] = acc[k];
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

// y = A x (b == null) or y = b - A x, level 0 planar BSR3, 8 lanes per row
__global__ void __launch_bounds__(256) k_l0_spmv(int n, const int32_t* __restrict__ goff,
                                                 const int32_t* __restrict__ cols, const double* __restrict__ vals,
                                                 const double* __restrict__ x, const double* __restrict__ b,
                                                 double* __restrict__ y) {
    const int sub = threadIdx.x & 7;
    const int row0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 3;
    const int rows_per_grid = (gridDim.x * blockDim.x) >> 3;
    const int nb = ((n + 3) / 4) * 4;  // uniform trip count per warp (4 rows per warp)
    for (int base = row0 - (row0 & 3); base < nb; base += rows_per_grid) {
        const int row = base + (row0 & 3);
        const bool valid = row < n;
        const int g0 = valid ? goff[row] : 0;
        const int ng = valid ? goff[row + 1] - g0 : 0;
        double a0 = 0, a1 = 0, a2 = 0;
        for (int g = sub; g < ng; g += 8) {
            const int4 cc = __ldg(reinterpret_cast<const int4*>(cols) + g0 + g);
            const int cj[4] = {cc.x, cc.y, cc.z, cc.w};
            const double* vb = vals + ((int64_t)g0 * 9 + g) * 4;
            const int64_t pl = (int64_t)ng * 4;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const double x0 = x[3 * cj[q]], x1 = x[3 * cj[q] + 1], x2 = x[3 * cj[q] + 2];
                a0 += vb[0 * pl + q] * x0 + vb[1 * pl + q] * x1 + vb[2 * pl + q] * x2;
                a1 += vb[3 * pl + q] * x0 + vb[4 * pl + q] * x1 + vb[5 * pl + q] * x2;
                a2 += vb[6 * pl + q] * x0 + vb[7 * pl + q] * x1 + vb[8 * pl + q] * x2;
            }
        }
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
        if (valid && sub == 0) {
            if (b) {
                y[3 * row] = b[3 * row] - a0;
                y[3 * row + 1] = b[3 * row + 1] - a1;
                y[3 * row + 2] = b[3 * row + 2] - a2;
            } else {
                y[3 * row] = a0;
                y[3 * row + 1] = a1;
                y[3 * row + 2] = a2;
            }
        }
    }
}

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

// Chebyshev step: r -= t; d = c1 d + c2 D^-1 r; x += d
__global__ void k_cheb_step(int n, int bs, const double* __restrict__ dinv, double* __restrict__ r,
                            const double* __restrict__ t, double* __restrict__ d, double* __restrict__ x, double c1,
                            double c2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t o = (int64_t)i * bs;
    double rr[6];
    for (int k = 0; k < bs; ++k) {
        rr[k] = r[o + k] - t[o + k];
        r[o + k] = rr[k];
    }
    const double* Di = dinv + (int64_t)i * bs * bs;
    for (int k = 0; k < bs; ++k) {
        double z = 0.0;
        for (int c = 0; c < bs; ++c) z += Di[k * bs + c] * rr[c];
        double dn = c1 * d[o + k] + c2 * z;
        d[o + k] = dn;
        x[o + k] += dn;
    }
}

__global__ void k_restrict(int na, const int32_t* __restrict__ ptr, const int32_t* __restrict__ nodes, int bs,
                           const double* __restrict__ Q, const double* __restrict__ rf, double* __restrict__ bc) {
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= na) return;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int p = ptr[a]; p < ptr[a + 1]; ++p) {
        int j = nodes[p];
        for (int d = 0; d < bs; ++d) {
            double rv = rf[(int64_t)j * bs + d];
            const double* q = Q + ((int64_t)j * bs + d) * 6;
            for (int c = 0; c < 6; ++c) acc[c] += q[c] * rv;
        }
    }
    for (int c = 0; c < 6; ++c) bc[(int64_t)a * 6 + c] = acc[c];
}

__global__ void k_prolong(int ndof, int bs, const int32_t* __restrict__ agg, const double* __restrict__ Q,
                          const double* __restrict__ xc, double* __restrict__ xf) {
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= ndof) return;
    int j = k / bs;
    const double* q = Q + (int64_t)k * 6;
    const double* x = xc + (int64_t)agg[j] * 6;
    double t = 0.0;
    for (int c = 0; c < 6; ++c) t += q[c] * x[c];
    xf[k] += t;
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

// In-place Gauss-Jordan inverse of an SPD matrix (one CTA); DOFs with a vanishing
// diagonal are decoupled first and get zero rows/columns in the inverse.
__global__ void __launch_bounds__(1024) k_dense_inverse(int nd, double* __restrict__ A, uint8_t* __restrict__ dead) {
    __shared__ double s_dmax;
    if (threadIdx.x == 0) {
        double m = 0.0;
        for (int k = 0; k < nd; ++k) m = fmax(m, fabs(A[(int64_t)k * nd + k]));
        s_dmax = m;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nd; k += blockDim.x) dead[k] = !(fabs(A[(int64_t)k * nd + k]) > 1e-12 * s_dmax);
    __syncthreads();
    for (int64_t e = threadIdx.x; e < (int64_t)nd * nd; e += blockDim.x) {
        int r = (int)(e / nd), c = (int)(e % nd);
        if (dead[r] || dead[c]) A[e] = (r == c) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int k = 0; k < nd; ++k) {
        const double ip = 1.0 / A[(int64_t)k * nd + k];
        __syncthreads();
        for (int c = threadIdx.x; c < nd; c += blockDim.x)
            if (c != k) A[(int64_t)k * nd + c] *= ip;
        __syncthreads();
        for (int64_t e = threadIdx.x; e < (int64_t)nd * nd; e += blockDim.x) {
            int r = (int)(e / nd), c = (int)(e % nd);
            if (r == k || c == k) continue;
            A[e] -= A[(int64_t)r * nd + k] * A[(int64_t)k * nd + c];
        }
        __syncthreads();
        for (int r = threadIdx.x; r < nd; r += blockDim.x)
            if (r != k) A[(int64_t)r * nd + k] *= -ip;
        __syncthreads();
        if (threadIdx.x == 0) A[(int64_t)k * nd + k] = ip;
        __syncthreads();
    }
    for (int64_t e = threadIdx.x; e < (int64_t)nd * nd; e += blockDim.x) {
        int r = (int)(e / nd), c = (int)(e % nd);
        if (dead[r] || dead[c]) A[e] = 0.0;
    }
}

__global__ void k_dense_matvec(int nd, const double* __restrict__ A, const double* __restrict__ x,
                               double* __restrict__ y) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= nd) return;
    double t = 0.0;
    for (int c = lane; c < nd; c += 32) t += A[(int64_t)warp * nd + c] * x[c];
    t = warp_sum(t);
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
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < nb; ++k) s += part[k];
        *out = s;
    }
}

__global__ void k_fill_hash(int64_t n, double* __restrict__ v) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull;
    h ^= h >> 29;
    v[i] = (double)(h & 0xFFFFF) / 1048576.0 + 0.5;
}

__global__ void k_scale(int64_t n, double a, const double* __restrict__ x, double* __restrict__ y) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = a * x[i];
}

unsigned grid_for(int64_t n, int t = 256) { return (unsigned)((n + t - 1) / t); }

// ---- outer PCG scalars: S[0] r.z, S[1] p.q, S[2] r.D^-1 r, S[3] b.D^-1 b, S[4] beta, S[5] alpha, S[6] breakdown
__global__ void k_fin(int nb, const double* __restrict__ part, double* __restrict__ S, int what) {
    if (threadIdx.x != 0) return;
    double t = 0.0;
    for (int k = 0; k < nb; ++k) t += part[k];
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

// x += alpha p, r -= alpha q, partial r . D^-1 r (3x3 blocks)
__global__ void k_amg_update(int n, const double* __restrict__ S, const double* __restrict__ p,
                             const double* __restrict__ q, double* __restrict__ x, double* __restrict__ r,
                             const double* __restrict__ dinv, double* __restrict__ part) {
    __shared__ double sh[8];
    const double alpha = S[5];
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double rv[3];
        for (int c = 0; c < 3; ++c) {
            x[3 * i + c] += alpha * p[3 * i + c];
            rv[c] = r[3 * i + c] - alpha * q[3 * i + c];
            r[3 * i + c] = rv[c];
        }
        const double* D = dinv + 9 * (int64_t)i;
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

}  // namespace

// ------------------------------------------------------------------ host side

static void level_spmv(const AmgLevel& l, const double* x, const double* b, double* y, cudaStream_t s) {
    if (l.S0) {
        int blocks = std::min<int64_t>(grid_for((int64_t)l.n * 8), 148 * 16);
        FX_LAUNCH(k_l0_spmv, blocks, 256, 0, s, l.n, l.S0->goff.ptr, l.S0->cols.ptr, l.vals0, x, b, y);
    } else {
        FX_LAUNCH(k_ln_spmv, grid_for((int64_t)l.n * 32), 256, 0, s, l.n, l.row_ptr.ptr, l.cols.ptr, l.vals.ptr, x, b,
                  y);
    }
}

static double dot(const double* a, const double* b, int64_t n, DBuf<double>& red, cudaStream_t s) {
    const int nb = 296;
    red.alloc(nb + 1, s);
    FX_LAUNCH(k_dot_part, nb, 256, 0, s, n, a, b, red.ptr);
    FX_LAUNCH(k_sum_part, 1, 32, 0, s, nb, red.ptr, red.ptr + nb);
    double v = 0.0;
    FX_CUDA_CHECK(cudaMemcpyAsync(&v, red.ptr + nb, sizeof(double), cudaMemcpyDeviceToHost, s));
    stream_wait(s, "amg dot");
    return v;
}

static void estimate_lmax(AmgLevel& l, DBuf<double>& red, cudaStream_t s) {
    const int64_t nd = (int64_t)l.n * l.bs;
    FX_LAUNCH(k_fill_hash, grid_for(nd), 256, 0, s, nd, l.x.ptr);
    double lam = 1.0;
    for (int it = 0; it < 12; ++it) {
        level_spmv(l, l.x.ptr, nullptr, l.t.ptr, s);                 // t = A x
        FX_LAUNCH(k_cheb_init, grid_for(l.n), 256, 0, s, l.n, l.bs, l.dinv_ptr(), l.t.ptr, l.d.ptr, l.r.ptr, 1.0,
                  1);                                                 // d = D^-1 A x
        double nd2 = dot(l.d.ptr, l.d.ptr, nd, red, s);
        double nx2 = dot(l.x.ptr, l.x.ptr, nd, red, s);
        lam = nx2 > 0 ? std::sqrt(nd2 / nx2) : 1.0;
        double inv = nd2 > 0 ? 1.0 / std::sqrt(nd2) : 1.0;
        FX_LAUNCH(k_scale, grid_for(nd), 256, 0, s, nd, inv, l.d.ptr, l.x.ptr);
    }
    l.lmax = 1.1 * lam;
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
    // host copy of the level-0 points' origin
    std::vector<double> hx(3 * (size_t)n_nodes);
    FX_CUDA_CHECK(cudaMemcpyAsync(hx.data(), xyz, hx.size() * sizeof(double), cudaMemcpyDeviceToHost, s));
    stream_wait(s, "amg coords");
    double o[3] = {1e300, 1e300, 1e300};
    for (int i = 0; i < n_nodes; ++i)
        for (int d = 0; d < 3; ++d) o[d] = std::min(o[d], hx[3 * (size_t)i + d]);
    DBuf<double> coords, cent, Rprev, Rnext;
    coords.upload(hx, s);
    double cell = cell0;
    for (int lev = 0;; ++lev) {
        AmgLevel& l = L[lev];
        const int64_t nd = (int64_t)l.n * l.bs;
        for (DBuf<double>* v : {&l.x, &l.b, &l.r, &l.d, &l.t}) v->alloc(nd, s);
        if (lev > 0) {
            l.dinv.alloc((size_t)l.n * 36, s);
            FX_LAUNCH(k_block_inv6, grid_for(l.n, 128), 128, 0, s, l.n, l.row_ptr.ptr, l.cols.ptr, l.vals.ptr,
                      l.dinv.ptr);
        }
        if (lev > 0 && (nd <= kCoarseMaxDof || lev + 1 >= kMaxLevels)) {
            l.coarsest = true;
            l.dense_inv.alloc((size_t)nd * nd, s);
            l.dense_inv.zero(s);
            FX_LAUNCH(k_dense_from_bsr, grid_for(l.n, 64), 64, 0, s, l.n, l.row_ptr.ptr, l.cols.ptr, l.vals.ptr,
                      l.dense_inv.ptr);
            DBuf<uint8_t> dead;
            dead.alloc(nd, s);
            FX_LAUNCH(k_dense_inverse, 1, 1024, 0, s, (int)nd, l.dense_inv.ptr, dead.ptr);
            stream_wait(s, "amg coarse inverse");
            break;
        }
        estimate_lmax(l, red_, s);
        // ---- aggregation by cells
        DBuf<uint64_t> keys, keys_s;
        DBuf<int32_t> ids, ids_s, head, rank1;
        keys.alloc(l.n, s);
        keys_s.alloc(l.n, s);
        ids.alloc(l.n, s);
        ids_s.alloc(l.n, s);
        FX_LAUNCH(k_cell_keys, grid_for(l.n), 256, 0, s, l.n, coords.ptr, o[0], o[1], o[2], 1.0 / cell, keys.ptr,
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
        FineView F{};
        F.bs = l.bs;
        DBuf<int32_t> blk_row_c;
        if (l.S0) {
            F.blk_row = l.S0->blk_row.ptr;
            F.vals = l.vals0;
            F.row_ptr = l.S0->row_ptr.ptr;
            F.goff = l.S0->goff.ptr;
            F.cols4 = l.S0->cols.ptr;
        } else {
            blk_row_c.alloc(l.nblocks, s);
            FX_LAUNCH(k_expand_rows, grid_for(l.n), 256, 0, s, l.n, l.row_ptr.ptr, blk_row_c.ptr);
            F.blk_row = blk_row_c.ptr;
            F.blk_col = l.cols.ptr;
            F.vals = l.vals.ptr;
        }
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
        FX_LAUNCH(k_galerkin, grid_for(ncb, 128), 128, 0, s, (int64_t)ncb, seg.ptr, cb_s.ptr, F, lf.Q.ptr,
                  c.vals.ptr);
        stream_wait(s, "amg galerkin");
        // next level points and near-null-space
        coords = std::move(cent);
        Rprev = std::move(Rnext);
        cell *= 2.0;
    }
    if (st) {
        st->levels = (int)L.size();
        st->sizes.clear();
        for (auto& l : L) st->sizes.push_back(l.n * l.bs);
        st->setup_ms = timer.stop_ms(s);
    }
}

// Chebyshev polynomial smoother of degree 2 on D^-1 A over [lmax/30, lmax].
static void smooth(AmgLevel& l, bool zero_x, cudaStream_t s) {
    const double lmax = l.lmax, lmin = lmax / 30.0;
    const double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin);
    const double sigma = theta / delta;
    const double rho = 1.0 / sigma;
    const double rho1 = 1.0 / (2.0 * sigma - rho);
    const int64_t nd = (int64_t)l.n * l.bs;
    if (zero_x) FX_CUDA_CHECK(cudaMemcpyAsync(l.r.ptr, l.b.ptr, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    else level_spmv(l, l.x.ptr, l.b.ptr, l.r.ptr, s);  // r = b - A x
    FX_LAUNCH(k_cheb_init, grid_for(l.n), 256, 0, s, l.n, l.bs, l.dinv_ptr(), l.r.ptr, l.d.ptr, l.x.ptr, 1.0 / theta,
              zero_x ? 1 : 0);
    level_spmv(l, l.d.ptr, nullptr, l.t.ptr, s);  // t = A d
    FX_LAUNCH(k_cheb_step, grid_for(l.n), 256, 0, s, l.n, l.bs, l.dinv_ptr(), l.r.ptr, l.t.ptr, l.d.ptr, l.x.ptr,
              rho1 * rho, 2.0 * rho1 / delta);
}

void Amg::vcycle(int lev, cudaStream_t s) {
    AmgLevel& l = L[lev];
    const int64_t nd = (int64_t)l.n * l.bs;
    if (l.coarsest) {
        FX_LAUNCH(k_dense_matvec, grid_for(nd * 32), 256, 0, s, (int)nd, l.dense_inv.ptr, l.b.ptr, l.x.ptr);
        return;
    }
    AmgLevel& c = L[lev + 1];
    smooth(l, true, s);
    level_spmv(l, l.x.ptr, l.b.ptr, l.r.ptr, s);  // r = b - A x
    FX_LAUNCH(k_restrict, grid_for(l.n_agg), 256, 0, s, l.n_agg, l.agg_ptr.ptr, l.agg_nodes.ptr, l.bs, l.Q.ptr,
              l.r.ptr, c.b.ptr);
    vcycle(lev + 1, s);
    FX_LAUNCH(k_prolong, grid_for(nd), 256, 0, s, (int)nd, l.bs, l.agg.ptr, l.Q.ptr, c.x.ptr, l.x.ptr);
    smooth(l, false, s);
}

void Amg::apply(const double* r, double* z, cudaStream_t s) {
    AmgLevel& l = L[0];
    const int64_t nd = (int64_t)l.n * l.bs;
    FX_CUDA_CHECK(cudaMemcpyAsync(l.b.ptr, r, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    vcycle(0, s);
    FX_CUDA_CHECK(cudaMemcpyAsync(z, l.x.ptr, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
}

// ------------------------------------------------------------------ AMG-preconditioned CG (FP64)

int AmgPcg::solve(const BsrStructure& S, const double* vals64, const double* dinv64, const double* xyz,
                  double cell0, const double* b, double* x, const PcgOptions& opt, cudaStream_t s,
                  int64_t* launches, long long* iters, double* relres, AmgStats* st) {
    const int n = S.n_rows;
    const int64_t nd = 3 * (int64_t)n;
    amg.setup(S, vals64, dinv64, xyz, n, cell0, s, st);
    AmgLevel& l0 = amg.L[0];
    r_.alloc(nd, s);
    z_.alloc(nd, s);
    p_.alloc(nd, s);
    q_.alloc(nd, s);
    const int nb = 296;
    part_.alloc(nb, s);
    sc_.alloc(8, s);
    sc_.zero(s);
    FX_CUDA_CHECK(cudaMemsetAsync(x, 0, nd * sizeof(double), s));
    FX_CUDA_CHECK(cudaMemcpyAsync(r_.ptr, b, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    // ||b||_D, z = V(b), rz, p = z
    FX_LAUNCH(k_rdr_part, nb, 256, 0, s, n, r_.ptr, dinv64, part_.ptr);
    FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 1);
    FX_CUDA_CHECK(cudaMemcpyAsync(sc_.ptr + 3, sc_.ptr + 2, sizeof(double), cudaMemcpyDeviceToDevice, s));
    amg.apply(r_.ptr, z_.ptr, s);
    FX_LAUNCH(k_dot_part, nb, 256, 0, s, nd, r_.ptr, z_.ptr, part_.ptr);
    FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 3);
    FX_CUDA_CHECK(cudaMemcpyAsync(p_.ptr, z_.ptr, nd * sizeof(double), cudaMemcpyDeviceToDevice, s));
    auto iteration = [&]() {
        const int spmv_grid = (int)std::min<int64_t>(grid_for((int64_t)n * 8), 148 * 16);
        FX_LAUNCH(k_l0_spmv, spmv_grid, 256, 0, s, n, S.goff.ptr, S.cols.ptr, vals64, p_.ptr, nullptr, q_.ptr);
        FX_LAUNCH(k_dot_part, nb, 256, 0, s, nd, p_.ptr, q_.ptr, part_.ptr);
        FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 0);
        FX_LAUNCH(k_amg_update, nb, 256, 0, s, n, sc_.ptr, p_.ptr, q_.ptr, x, r_.ptr, dinv64, part_.ptr);
        FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 1);
        amg.apply(r_.ptr, z_.ptr, s);
        FX_LAUNCH(k_dot_part, nb, 256, 0, s, nd, r_.ptr, z_.ptr, part_.ptr);
        FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 2);
        FX_LAUNCH(k_xpby, nb, 256, 0, s, nd, z_.ptr, sc_.ptr, p_.ptr);
    };
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
        FX_CUDA_CHECK(cudaStreamEndCapture(s, &g));
        g_launch_counter = saved;
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
    const int spmv_grid = (int)std::min<int64_t>(grid_for((int64_t)n * 8), 148 * 16);
    FX_LAUNCH(k_l0_spmv, spmv_grid, 256, 0, s, n, S.goff.ptr, S.cols.ptr, vals64, x, b, q_.ptr);
    FX_LAUNCH(k_rdr_part, nb, 256, 0, s, n, q_.ptr, dinv64, part_.ptr);
    FX_LAUNCH(k_fin, 1, 32, 0, s, nb, part_.ptr, sc_.ptr, 1);
    FX_CUDA_CHECK(cudaMemcpyAsync(h, sc_.ptr, sizeof(h), cudaMemcpyDeviceToHost, s));
    stream_wait(s, "amg pcg final");
    if (iters) *iters = it;
    if (relres) *relres = h[3] > 0.0 ? std::sqrt(std::max(0.0, h[2]) / h[3]) : 0.0;
    (void)l0;
    return rc;
}

}  // namespace fx
