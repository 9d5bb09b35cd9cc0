// One warp's sums of a coarse-level block row (row-major 6x6 block CSR): lane l
// handles the row's blocks l, l + 32, ..., each whole (its 36 values, its column id
// and the 6 gathered source values), and the six row sums are reduced over the warp
// by a fixed xor tree, so that every lane ends with the same six sums. Per row, the
// loads form three dependent steps (row pointer; column ids and values; gathered
// sources) whatever the row's length up to 32 blocks. Shared by the per-step coarse
// kernels and the persistent / cooperative coarse kernels, which must produce the
// same sums.
#pragma once

#include <cstdint>

namespace fx {

// Loads of the source vector: through L2 only (CG = true) when other CTAs of the
// same launch write it, the default path otherwise.
template <bool CG>
__device__ __forceinline__ double2 coarse_ld2(const double* p) {
    if constexpr (CG) return __ldcg(reinterpret_cast<const double2*>(p));
    else return *reinterpret_cast<const double2*>(p);
}

// acc[r] = sum over the row's blocks b0 .. b0 + nblk - 1 of (block row r) . v(col), in
// every lane of the warp. The lane's blocks are summed in block order; the lanes' sums
// are added by xor shuffles over 16, 8, 4, 2, 1 (both partners add the same two values,
// so all lanes hold identical bits).
template <bool CG>
__device__ __forceinline__ void coarse_row6(const int32_t* __restrict__ cols, const double* __restrict__ vals,
                                            const double* v, int b0, int nblk, int lane, double (&acc)[6]) {
#pragma unroll
    for (int r = 0; r < 6; ++r) acc[r] = 0.0;
    for (int j = lane; j < nblk; j += 32) {
        const int64_t blk = b0 + j;
        const int col = __ldg(cols + blk);
        const double2* a = reinterpret_cast<const double2*>(vals + blk * 36);
        double2 m[18];
#pragma unroll
        for (int k = 0; k < 18; ++k) m[k] = __ldg(a + k);
        const double* xs = v + 6 * (int64_t)col;
        const double2 x0 = coarse_ld2<CG>(xs), x1 = coarse_ld2<CG>(xs + 2), x2 = coarse_ld2<CG>(xs + 4);
#pragma unroll
        for (int r = 0; r < 6; ++r)
            acc[r] += m[3 * r].x * x0.x + m[3 * r].y * x0.y + m[3 * r + 1].x * x1.x + m[3 * r + 1].y * x1.y +
                      m[3 * r + 2].x * x2.x + m[3 * r + 2].y * x2.y;
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1)
#pragma unroll
        for (int r = 0; r < 6; ++r) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], s);
}

// One row of the coarsest level's dense inverse times x, summed by a warp: lane l adds
// A[c] x[c] for c = l, l + 32, ... in that order (8 columns' loads in flight before their
// products), then the lanes' sums by an xor tree. Shared by the per-step and the
// persistent / cooperative coarse kernels.
template <bool CG>
__device__ __forceinline__ double dense_row_dot(const double* __restrict__ a, const double* x, int nd, int lane) {
    constexpr int U = 8;
    double t = 0.0;
    for (int c0 = lane; c0 < nd; c0 += 32 * U) {
        double av[U], xv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int c = c0 + 32 * u;
            av[u] = c < nd ? __ldg(a + c) : 0.0;
            xv[u] = c < nd ? (CG ? __ldcg(x + c) : x[c]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (c0 + 32 * u < nd) t += av[u] * xv[u];
    }
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) t += __shfl_xor_sync(0xffffffffu, t, s);
    return t;
}

}  // namespace fx
