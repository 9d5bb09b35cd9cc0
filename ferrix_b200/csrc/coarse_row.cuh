// One warp's partial sums of a coarse-level row (row-major 6x6 block CSR): lane
// l < 30 handles block row l % 6 of the row's blocks l / 6 + 5 m, so consecutive
// lanes read consecutive 48-byte block rows. Shared by the per-step coarse kernels
// and the persistent cluster kernels, which must produce the same sums.
#pragma once

#include <cstdint>

namespace fx {

// Loads of the source vector: through L2 only (CG = true) when other CTAs of the
// same launch write it, the default path otherwise.
template <bool CG>
__device__ __forceinline__ double coarse_ld(const double* p) {
    if constexpr (CG) return __ldcg(p);
    else return *p;
}

// Partial sum sum_items vals(item) . v(col(item)) of this lane over items it = lane,
// lane + 30, ... < items (6 per block). U items' loads (column ids, block rows, gathered
// sources) are issued before their products, so that U column-index -> gather chains are
// in flight; the products are still added in item order, so the sum is the same for every
// U (and as item-by-item accumulation).
template <bool CG, int U>
__device__ __forceinline__ double coarse_row_part(const int32_t* __restrict__ cols,
                                                  const double* __restrict__ vals, const double* v, int b0,
                                                  int items, int lane) {
    double t = 0.0;
    if (lane >= 30) return t;
    int it = lane;
    if constexpr (U > 1) {
        for (; it + 30 * (U - 1) < items; it += 30 * U) {
            int kb[U], col[U];
#pragma unroll
            for (int q = 0; q < U; ++q) {
                kb[q] = (it + 30 * q) / 6;
                col[q] = __ldg(cols + b0 + kb[q]);
            }
            double2 a[U][3];
#pragma unroll
            for (int q = 0; q < U; ++q) {
                const double2* vr = reinterpret_cast<const double2*>(vals + (int64_t)(b0 + kb[q]) * 36 +
                                                                     (it + 30 * q - 6 * kb[q]) * 6);
                a[q][0] = __ldg(vr);
                a[q][1] = __ldg(vr + 1);
                a[q][2] = __ldg(vr + 2);
            }
            double x[U][6];
#pragma unroll
            for (int q = 0; q < U; ++q)
#pragma unroll
                for (int k = 0; k < 6; ++k) x[q][k] = coarse_ld<CG>(v + 6 * (int64_t)col[q] + k);
#pragma unroll
            for (int q = 0; q < U; ++q)
                t += a[q][0].x * x[q][0] + a[q][0].y * x[q][1] + a[q][1].x * x[q][2] + a[q][1].y * x[q][3] +
                     a[q][2].x * x[q][4] + a[q][2].y * x[q][5];
        }
    }
    for (; it < items; it += 30) {
        const int kb = it / 6;
        const int64_t blk = b0 + kb;
        const double2* vr = reinterpret_cast<const double2*>(vals + blk * 36 + (it - 6 * kb) * 6);
        const double* xx = v + 6 * (int64_t)__ldg(cols + blk);
        const double2 a0 = __ldg(vr), a1 = __ldg(vr + 1), a2 = __ldg(vr + 2);
        t += a0.x * coarse_ld<CG>(xx) + a0.y * coarse_ld<CG>(xx + 1) + a1.x * coarse_ld<CG>(xx + 2) +
             a1.y * coarse_ld<CG>(xx + 3) + a2.x * coarse_ld<CG>(xx + 4) + a2.y * coarse_ld<CG>(xx + 5);
    }
    return t;
}

}  // namespace fx
