// Persistent multigrid-preconditioned CG: one thread-block cluster per system.
//
// The same algorithm as AmgPcg::solve (FP64 CG, one aggregation-multigrid
// V-cycle with Chebyshev smoothing per iteration, FP32 fine-level smoother
// values in mixed precision), with the launch structure turned inside out: a
// cluster of kClCtas CTAs runs the system's whole solve, every step of it a loop
// over the cluster's threads (a "virtual grid"), separated from the next step by
// a hardware cluster barrier (barrier.cluster, release / acquire at cluster
// scope). Dot products are summed per warp and per CTA in a fixed order, then
// across the cluster from each CTA's shared memory (distributed shared memory),
// so every thread holds the same totals and takes the same branches. A launch
// holds one cluster per system, so many independent decks advance in one
// launch with a per-system descriptor table (ClInst) and a small system does not
// pay ~23 launches per CG iteration.
//
// Vectors written during the kernel are read with ld.global.cg (L2), never
// through the read-only / L1 path; matrix data is read-only for the whole
// kernel. Every loop is bounded: the CG by max_iter, the phases by the row
// counts.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>

#include "amg.hpp"
#include "coarse_row.cuh"

namespace cg = cooperative_groups;

namespace fx {

namespace {

constexpr int kClThreads = 256;
constexpr int kClCtas = 8;  // CTAs per cluster (the portable maximum)
constexpr int kClWarps = kClThreads / 32;

enum : int { kOpApply = 0, kOpRUpd = 1, kOpCheb0 = 2, kOpChebK = 3 };

struct Vg {
    int t, nt;  // this thread's rank in the cluster, threads in the cluster
};

struct ClShared {
    double warp[kClWarps][2];
    double cta[2][2];  // [buffer][value]: alternating buffers, one cluster barrier per reduction
    int buf;
};

__device__ __forceinline__ double ldv(const double* p) { return __ldcg(p); }

// Fixed-order sum of NV per-thread values over the cluster; every thread gets the totals.
template <int NV>
__device__ __forceinline__ void cluster_sum(double (&v)[NV], ClShared& sh, cg::cluster_group& cl) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh.warp[w][k] = v[k];
    __syncthreads();
    const int b = sh.buf;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = 0.0;
            for (int j = 0; j < kClWarps; ++j) t += sh.warp[j][k];
            sh.cta[b][k] = t;
        }
    }
    cl.sync();
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double t = 0.0;
        for (unsigned r = 0; r < cl.num_blocks(); ++r) t += *cl.map_shared_rank(&sh.cta[b][k], r);
        v[k] = t;
    }
    __syncthreads();  // every thread has read sh.buf before thread 0 flips it
    if (threadIdx.x == 0) sh.buf = b ^ 1;
}

template <typename VT>
__device__ __forceinline__ void ld4g(const VT* p, VT o[4]);
template <>
__device__ __forceinline__ void ld4g<float>(const float* p, float o[4]) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}
template <>
__device__ __forceinline__ void ld4g<double>(const double* p, double o[4]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p));
    const double2 b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b.x;
    o[3] = b.y;
}

// Level-0 operator over the planar BSR3 (8 lanes per block row, 4 rows per warp,
// uniform trip count per warp), as the multi-kernel path's fine-level operator:
//   kOpApply  y = A v, dsum += v.y
//   kOpRUpd   r -= A v
//   kOpCheb0  r = b - A v; d = c2 D^-1 r; xo = v + d              (dot: dsum += b.xo)
//   kOpChebK  r -= A v; d = c1 v + c2 D^-1 r; xo += d             (dot: dsum += b.xo)
// G32: gathers from v4 (FP32, float4 per node) and writes the direction into d4;
// the row's own FP64 component comes from v where the mode needs the iterate (Cheb0).
template <typename VT, int MODE, bool G32>
__device__ __noinline__ void l0_op(const ClInst& I, Vg g, const VT* __restrict__ vals, const double* v, const float4* v4,
                      const double* b, double* y, double* r, double* d_out, float* d4_out, double* xo, double c1,
                      double c2, bool dot, double& dsum) {
    const int sub = g.t & 7;
    const int row0 = g.t >> 3;
    const int rows_per_grid = g.nt >> 3;
    const int nb = ((I.n + 3) / 4) * 4;
    for (int base = row0 - (row0 & 3); base < nb; base += rows_per_grid) {
        const int row = base + (row0 & 3);
        const bool valid = row < I.n;
        const int g0 = valid ? __ldg(I.goff + row) : 0;
        const int ng = valid ? __ldg(I.goff + row + 1) - g0 : 0;
        const int64_t o3 = 3 * (int64_t)row;
        const int c = sub < 3 ? sub : 0;
        const bool epi = valid && sub < 3;
        double src3[3] = {0.0, 0.0, 0.0}, Dr[3] = {0.0, 0.0, 0.0}, vc = 0.0, xoc = 0.0, bc = 0.0;
        if (epi) {
            if (MODE == kOpCheb0 || MODE == kOpChebK) {
                const double* src = MODE == kOpCheb0 ? b : r;
#pragma unroll
                for (int kk = 0; kk < 3; ++kk) {
                    src3[kk] = ldv(src + o3 + kk);
                    Dr[kk] = __ldg(I.dinv0 + 9 * (int64_t)row + 3 * c + kk);
                }
                if (G32 && MODE == kOpChebK) {
                    const float* own = reinterpret_cast<const float*>(v4 + row);
                    vc = (double)__ldcg(own + c);
                } else {
                    vc = ldv(v + o3 + c);
                }
                if (MODE == kOpChebK) xoc = ldv(xo + o3 + c);
                if (dot) bc = ldv(b + o3 + c);
            } else if (MODE == kOpApply) {
                vc = ldv(v + o3 + c);
            } else {
                src3[0] = ldv(r + o3 + c);
            }
        }
        double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 2
        for (int gg = sub; gg < ng; gg += 8) {
            const int4 cc = __ldg(reinterpret_cast<const int4*>(I.cols) + g0 + gg);
            const int cj[4] = {cc.x, cc.y, cc.z, cc.w};
            using GT = typename std::conditional<G32, float, double>::type;
            GT xv[4][3];
            if (G32) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const float4 t = __ldcg(v4 + cj[q]);
                    xv[q][0] = t.x;
                    xv[q][1] = t.y;
                    xv[q][2] = t.z;
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q)
#pragma unroll
                    for (int k = 0; k < 3; ++k) xv[q][k] = (GT)ldv(v + 3 * (int64_t)cj[q] + k);
            }
            const VT* vb = vals + ((int64_t)g0 * 9 + gg) * 4;
            const int64_t pl = (int64_t)ng * 4;
#pragma unroll
            for (int rr = 0; rr < 3; ++rr) {
                VT m0[4], m1[4], m2[4];
                ld4g<VT>(vb + (3 * rr) * pl, m0);
                ld4g<VT>(vb + (3 * rr + 1) * pl, m1);
                ld4g<VT>(vb + (3 * rr + 2) * pl, m2);
                GT t = 0;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    t += (GT)m0[q] * xv[q][0] + (GT)m1[q] * xv[q][1] + (GT)m2[q] * xv[q][2];
                acc[rr] += (double)t;
            }
        }
#pragma unroll
        for (int s = 4; s > 0; s >>= 1)
#pragma unroll
            for (int rr = 0; rr < 3; ++rr) acc[rr] += __shfl_xor_sync(0xffffffffu, acc[rr], s);
        const double axc = c == 0 ? acc[0] : (c == 1 ? acc[1] : acc[2]);
        __syncwarp();  // every lane's reads of r are ordered before any lane writes r[c]
        if (!epi) continue;
        if (MODE == kOpRUpd) {
            r[o3 + c] = src3[0] - axc;
        } else if (MODE == kOpApply) {
            y[o3 + c] = axc;
            dsum += vc * axc;
        } else {
            const double rr3[3] = {src3[0] - acc[0], src3[1] - acc[1], src3[2] - acc[2]};
            const double z = Dr[0] * rr3[0] + Dr[1] * rr3[1] + Dr[2] * rr3[2];
            r[o3 + c] = c == 0 ? rr3[0] : (c == 1 ? rr3[1] : rr3[2]);
            const double dn = (MODE == kOpCheb0 ? 0.0 : c1 * vc) + c2 * z;
            if (G32) d4_out[4 * (int64_t)row + c] = (float)dn;
            else d_out[o3 + c] = dn;
            const double xn = (MODE == kOpCheb0 ? vc : xoc) + dn;
            xo[o3 + c] = xn;
            if (dot) dsum += bc * xn;
        }
    }
}

// Coarse-level operator (6x6 blocks, warp per block row, 30 lanes over the row's
// (block, block row) items, fixed-order shuffle tree), modes as l0_op without dot.
template <int MODE>
__device__ __noinline__ void ln_op(const ClLevel& L, Vg g, const double* v, const double* b, double* r, double* d_out,
                      double* xo, double c1, double c2) {
    const int lane = g.t & 31;
    for (int row = g.t >> 5; row < L.n; row += g.nt >> 5) {
        const int64_t o6 = 6 * (int64_t)row;
        const int c = lane < 6 ? lane : 0;
        const bool epi = lane < 6;
        double src6[6] = {0, 0, 0, 0, 0, 0}, Dr[6] = {0, 0, 0, 0, 0, 0}, vc = 0.0, xoc = 0.0;
        if (epi) {
            if (MODE == kOpCheb0 || MODE == kOpChebK) {
                const double* src = MODE == kOpCheb0 ? b : r;
#pragma unroll
                for (int k = 0; k < 6; ++k) {
                    src6[k] = ldv(src + o6 + k);
                    Dr[k] = __ldg(L.dinv + 36 * (int64_t)row + 6 * c + k);
                }
                vc = ldv(v + o6 + c);
                if (MODE == kOpChebK) xoc = ldv(xo + o6 + c);
            } else {
                src6[0] = ldv(r + o6 + c);
            }
        }
        const int b0 = __ldg(L.row_ptr + row);
        double acc[6];
        coarse_row6<true>(L.cols, L.vals, v, b0, __ldg(L.row_ptr + row + 1) - b0, lane, acc);
        double axc = acc[0];
#pragma unroll
        for (int k = 1; k < 6; ++k)
            if (c == k) axc = acc[k];
        __syncwarp();
        if (!epi) continue;
        if (MODE == kOpRUpd) {
            r[o6 + c] = src6[0] - axc;
        } else {
            double z = 0.0, rc = 0.0;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const double rk = src6[k] - acc[k];
                z += Dr[k] * rk;
                if (k == c) rc = rk;
            }
            r[o6 + c] = rc;
            const double dn = (MODE == kOpCheb0 ? 0.0 : c1 * vc) + c2 * z;
            d_out[o6 + c] = dn;
            xo[o6 + c] = (MODE == kOpCheb0 ? vc : xoc) + dn;
        }
    }
}

// b_c = Q^T r_f per aggregate (warp per aggregate); with a coarse start (dinv != null)
// also the coarse level's first smoothing step from x = 0: d = xs = c2 D^-1 b_c, r = b_c.
__device__ __noinline__ void restrict_op(Vg g, int na, const int32_t* ptr, const int32_t* nodes, int bs, const double* Q,
                            const double* rf, double* bc, const double* dinv, double* cr, double* cd, double* cxs,
                            double c2) {
    const int lane = g.t & 31;
    for (int a = g.t >> 5; a < na; a += g.nt >> 5) {
        const int p0 = __ldg(ptr + a), rows = (__ldg(ptr + a + 1) - p0) * bs;
        double acc[6] = {0, 0, 0, 0, 0, 0};
        for (int r0 = lane; r0 < rows; r0 += 128) {
            double rv[4], qv[4][6];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int rr = r0 + 32 * u;
                rv[u] = 0.0;
                if (rr < rows) {
                    const int j = __ldg(nodes + p0 + rr / bs);
                    const int64_t row = (int64_t)j * bs + rr % bs;
                    rv[u] = ldv(rf + row);
#pragma unroll
                    for (int c = 0; c < 6; ++c) qv[u][c] = __ldg(Q + row * 6 + c);
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
        for (int c = 0; c < 6; ++c) t[c] = warp_sum(acc[c]);
        if (lane < 6) {
            const int64_t o = (int64_t)a * 6 + lane;
            double tk = t[0];
#pragma unroll
            for (int c = 1; c < 6; ++c)
                if (lane == c) tk = t[c];
            bc[o] = tk;
            if (dinv) {
                const double* Di = dinv + (int64_t)a * 36 + lane * 6;
                double v = 0.0;
#pragma unroll
                for (int j = 0; j < 6; ++j) v += __ldg(Di + j) * t[j];
                v *= c2;
                cd[o] = v;
                cxs[o] = v;
                cr[o] = tk;
            }
        }
    }
}

// x_f += alpha Q x_c over the fine level's dofs (bs per block row)
__device__ __noinline__ void prolong_op(Vg g, int ndof, int bs, const int32_t* agg, const double* Q, const double* xc, double* xf,
                           double alpha) {
    for (int k = g.t; k < ndof; k += g.nt) {
        const int j = k / bs;
        const double* q = Q + (int64_t)k * 6;
        const double* x = xc + (int64_t)__ldg(agg + j) * 6;
        double t = 0.0;
        for (int c = 0; c < 6; ++c) t += __ldg(q + c) * ldv(x + c);
        xf[k] += alpha * t;
    }
}

// fine level: x += alpha Q x_c and the FP32 copy of x for the smoother's gathers
__device__ __noinline__ void prolong0_op(Vg g, const ClInst& I, const double* xc, double alpha) {
    for (int i = g.t; i < I.n; i += g.nt) {
        const double* x = xc + (int64_t)__ldg(I.agg + i) * 6;
        double out[3];
        for (int k = 0; k < 3; ++k) {
            const double* q = I.Q + (3 * (int64_t)i + k) * 6;
            double t = 0.0;
            for (int c = 0; c < 6; ++c) t += __ldg(q + c) * ldv(x + c);
            out[k] = ldv(I.lx + 3 * (int64_t)i + k) + alpha * t;
            I.lx[3 * (int64_t)i + k] = out[k];
        }
        float4 q = make_float4(1.f, 1.f, 1.f, 0.f);
        if (I.sq4) q = __ldg(I.sq4 + i);  // FP16 smoother: the gathered copy is scaled by sqrt(a_ii)
        reinterpret_cast<float4*>(I.x4)[i] = make_float4((float)(out[0] * (double)q.x), (float)(out[1] * (double)q.y),
                                                         (float)(out[2] * (double)q.z), 0.0f);
    }
}

__device__ __noinline__ void dense_op(Vg g, int nd, const double* A, const double* x, double* y) {
    const int lane = g.t & 31;
    for (int row = g.t >> 5; row < nd; row += g.nt >> 5) {
        const double t = dense_row_dot<true>(A + (int64_t)row * nd, x, nd, lane);
        if (lane == 0) y[row] = t;
    }
}

// Level-0 start of the V-cycle from x = 0 with right-hand side rhs: r0 = rhs,
// x0 = d = c2 D^-1 rhs. With alpha != 0 first the CG update x += alpha p,
// r -= alpha q (rhs = r). Returns this thread's part of rhs.D^-1 rhs.
template <bool G32>
__device__ __noinline__ double start0_op(Vg g, const ClInst& I, double alpha, bool update) {
    double acc = 0.0;
    for (int i = g.t; i < I.n; i += g.nt) {
        const int64_t o3 = 3 * (int64_t)i;
        double rv[3];
        for (int c = 0; c < 3; ++c) {
            if (update) {
                I.x[o3 + c] = ldv(I.x + o3 + c) + alpha * ldv(I.p + o3 + c);
                rv[c] = ldv(I.r + o3 + c) - alpha * ldv(I.q + o3 + c);
                I.r[o3 + c] = rv[c];
            } else {
                rv[c] = ldv(I.r + o3 + c);
            }
            I.lr[o3 + c] = rv[c];
        }
        const double* D = I.dinv0 + 9 * (int64_t)i;
        double t[3];
        for (int c = 0; c < 3; ++c) {
            const double dr = __ldg(D + 3 * c) * rv[0] + __ldg(D + 3 * c + 1) * rv[1] + __ldg(D + 3 * c + 2) * rv[2];
            acc += rv[c] * dr;
            t[c] = I.c2_start * dr;
            I.lx[o3 + c] = t[c];
        }
        if (G32) reinterpret_cast<float4*>(I.d4a)[i] = make_float4((float)t[0], (float)t[1], (float)t[2], 0.0f);
        else
            for (int c = 0; c < 3; ++c) I.ld[o3 + c] = t[c];
    }
    return acc;
}

// One V-cycle for the right-hand side I.r (level-0 start already done by start0_op):
// z = cycle(r); returns this thread's part of r.z (the last post-smoothing step).
// Barriers between the phases of a cycle: the cluster's hardware barrier, or
// (for one system spread over the whole GPU) a software grid barrier whose wait
// is bounded; sync() returns false when that wait ran out.
struct ClusterBar {
    cg::cluster_group& cl;
    __device__ __forceinline__ bool sync() {
        cl.sync();
        return true;
    }
};

constexpr unsigned kGridSpinLimit = 1u << 22;  // polls of the barrier generation (~0.2-1 s) before giving up

struct GridBar {
    GridBarState* st;
    double* flag;  // set to 1 when a wait ran out
    unsigned nblocks;
    __device__ bool sync() {
        __shared__ int ok;
        __syncthreads();
        if (threadIdx.x == 0) {
            ok = 1;
            volatile unsigned* gen = &st->gen;
            const unsigned g0 = *gen;  // read before arriving: the last arrival moves it on
            __threadfence();
            if (atomicAdd(&st->count, 1u) == nblocks - 1) {
                atomicExch(&st->count, 0u);
                __threadfence();
                atomicAdd(&st->gen, 1u);
            } else {
                unsigned polls = 0;
                while (*gen == g0) {
                    if (++polls > kGridSpinLimit) {
                        ok = 0;
                        *flag = 1.0;
                        break;
                    }
                    __nanosleep(64);
                }
            }
            __threadfence();
        }
        __syncthreads();
        return ok != 0;
    }
};

// The coarse part of one V-cycle, from the level-0 residual I.lr: restriction into
// level 1 (with its first smoothing step unless it is the coarsest), the coarse
// levels down to the dense coarsest solve and back up, and the prolongation of the
// correction into the level-0 iterate (I.lx, and I.x4 with FP32 smoother vectors).
// Returns false when a barrier wait ran out (the caller stops).
template <bool G32, typename Bar>
__device__ bool coarse_cycle(const ClInst& I, Vg g, int degree, double alpha, Bar& bar) {
    // restriction into level 1 (with its first smoothing step unless it is the coarsest)
    {
        const ClLevel& c = I.lev[1];
        restrict_op(g, I.n_agg, I.agg_ptr, I.agg_nodes, 3, I.Q, I.lr, c.b, c.coarsest ? nullptr : c.dinv, c.r, c.d,
                    c.xs, c.c2_start);
        if (!bar.sync()) return false;
    }
    // coarse levels: down to the coarsest, dense solve, back up
    int m = 1;
    const int last = min(I.levels, kClMaxLevels) - 1;  // the coarsest level (setup always ends with one)
    for (; m < last && !I.lev[m].coarsest; ++m) {
        const ClLevel& l = I.lev[m];
        double* cA = l.d;
        double* cB = l.t;
        for (int st = 1; st < degree; ++st) {
            ln_op<kOpChebK>(l, g, cA, nullptr, l.r, cB, l.xs, l.c1[st], l.c2[st]);
            if (!bar.sync()) return false;
            double* t = cA;
            cA = cB;
            cB = t;
        }
        ln_op<kOpRUpd>(l, g, cA, nullptr, l.r, nullptr, nullptr, 0.0, 0.0);
        if (!bar.sync()) return false;
        const ClLevel& c = I.lev[m + 1];
        restrict_op(g, l.n_agg, l.agg_ptr, l.agg_nodes, 6, l.Q, l.r, c.b, c.coarsest ? nullptr : c.dinv, c.r, c.d,
                    c.xs, c.c2_start);
        if (!bar.sync()) return false;
    }
    {
        const ClLevel& l = I.lev[m];
        dense_op(g, 6 * l.n, l.dense_inv, l.b, l.x);
        if (!bar.sync()) return false;
    }
    for (--m; m >= 1; --m) {
        const ClLevel& l = I.lev[m];
        const ClLevel& c = I.lev[m + 1];
        prolong_op(g, 6 * l.n, 6, l.agg, l.Q, c.x, l.xs, alpha);
        if (!bar.sync()) return false;
        double* cA = l.d;
        double* cB = l.t;
        ln_op<kOpCheb0>(l, g, l.xs, l.b, l.r, cA, l.x, 0.0, l.c2_start);
        if (!bar.sync()) return false;
        for (int st = 1; st < degree; ++st) {
            ln_op<kOpChebK>(l, g, cA, nullptr, l.r, cB, l.x, l.c1[st], l.c2[st]);
            if (!bar.sync()) return false;
            double* t = cA;
            cA = cB;
            cB = t;
        }
    }
    if (G32) prolong0_op(g, I, I.lev[1].x, alpha);
    else prolong_op(g, 3 * I.n, 3, I.agg, I.Q, I.lev[1].x, I.lx, alpha);
    return bar.sync();
}

template <typename VT, bool G32>
__device__ double vcycle(const ClInst& I, Vg g, const VT* vals, int degree, double alpha, cg::cluster_group& cl) {
    double dummy = 0.0;
    // level-0 pre-smoothing: directions alternate between (ld, d4a) and (lt, d4b)
    double* dA = I.ld;
    double* dB = I.lt;
    float* dA4 = I.d4a;
    float* dB4 = I.d4b;
    for (int st = 1; st < degree; ++st) {
        l0_op<VT, kOpChebK, G32>(I, g, vals, dA, reinterpret_cast<const float4*>(dA4), nullptr, nullptr, I.lr, dB,
                                 dB4, I.lx, I.c1[st], I.c2[st], false, dummy);
        cl.sync();
        double* t = dA;
        dA = dB;
        dB = t;
        float* t4 = dA4;
        dA4 = dB4;
        dB4 = t4;
    }
    l0_op<VT, kOpRUpd, G32>(I, g, vals, dA, reinterpret_cast<const float4*>(dA4), nullptr, nullptr, I.lr, nullptr,
                            nullptr, nullptr, 0.0, 0.0, false, dummy);  // r = b - A x
    cl.sync();
    ClusterBar bar{cl};
    coarse_cycle<G32>(I, g, degree, alpha, bar);
    // post-smoothing into z (the last step reduces r.z)
    double dsum = 0.0;
    l0_op<VT, kOpCheb0, G32>(I, g, vals, I.lx, reinterpret_cast<const float4*>(I.x4), I.r, nullptr, I.lr, dA, dA4,
                             I.z, 0.0, I.c2_start, degree == 1, dsum);
    cl.sync();
    for (int st = 1; st < degree; ++st) {
        l0_op<VT, kOpChebK, G32>(I, g, vals, dA, reinterpret_cast<const float4*>(dA4), I.r, nullptr, I.lr, dB, dB4,
                                 I.z, I.c1[st], I.c2[st], st == degree - 1, dsum);
        cl.sync();
        double* t = dA;
        dA = dB;
        dB = t;
        float* t4 = dA4;
        dA4 = dB4;
        dB4 = t4;
    }
    return dsum;
}

template <typename VT, bool G32>
__global__ void __launch_bounds__(kClThreads, 2)
    k_amg_cluster(const ClInst* __restrict__ insts, ClResult* __restrict__ res, int n_inst, double rtol2,
                  int max_iter, int degree, double alpha) {
    __shared__ ClShared sh;
    cg::cluster_group cl = cg::this_cluster();
    const int inst = blockIdx.x / kClCtas;  // clusters are consecutive CTAs along x
    if (threadIdx.x == 0) sh.buf = 0;
    __syncthreads();
    if (inst >= n_inst) return;  // whole clusters only: the grid is n_inst * kClCtas
    const ClInst& I = insts[inst];
    const VT* vals = G32 ? reinterpret_cast<const VT*>(I.vals32) : reinterpret_cast<const VT*>(I.vals64);
    const Vg g{(int)cl.block_rank() * kClThreads + (int)threadIdx.x, (int)cl.num_blocks() * kClThreads};
    const int64_t nd = 3 * (int64_t)I.n;
    // x = 0, r = b
    for (int64_t i = g.t; i < nd; i += g.nt) {
        I.x[i] = 0.0;
        I.r[i] = __ldg(I.b + i);
    }
    cl.sync();
    // ||b||_D^2, z = V(b), r.z, p = z
    double v1[1] = {start0_op<G32>(g, I, 0.0, false)};
    cl.sync();
    cluster_sum<1>(v1, sh, cl);
    const double bd = v1[0];
    double rzd = bd;
    double rz1[1] = {vcycle<VT, G32>(I, g, vals, degree, alpha, cl)};
    cluster_sum<1>(rz1, sh, cl);
    double rz = rz1[0];
    for (int64_t i = g.t; i < nd; i += g.nt) I.p[i] = ldv(I.z + i);
    cl.sync();
    long long it = 0;
    int status = FX_OK;
    while (true) {
        if (!(bd > 0.0) || rzd <= rtol2 * bd) break;
        if (it >= max_iter) {
            status = FX_CONVERGENCE;
            break;
        }
        // q = A p, alpha = r.z / p.q
        double pq[1] = {0.0};
        l0_op<double, kOpApply, false>(I, g, I.vals64, I.p, nullptr, nullptr, I.q, nullptr, nullptr, nullptr,
                                       nullptr, 0.0, 0.0, false, pq[0]);
        cl.sync();
        cluster_sum<1>(pq, sh, cl);
        if (!(pq[0] > 0.0) || !isfinite(pq[0])) {
            status = FX_NUMERICAL;
            break;
        }
        const double a = rz / pq[0];
        // x += a p, r -= a q, r.D^-1 r; the V-cycle's level-0 start
        double rd[1] = {start0_op<G32>(g, I, a, true)};
        cl.sync();
        cluster_sum<1>(rd, sh, cl);
        rzd = rd[0];
        ++it;
        if (rzd <= rtol2 * bd) break;
        double rzn[1] = {vcycle<VT, G32>(I, g, vals, degree, alpha, cl)};
        cluster_sum<1>(rzn, sh, cl);
        const double beta = rz > 0.0 ? rzn[0] / rz : 0.0;
        rz = rzn[0];
        for (int64_t i = g.t; i < nd; i += g.nt) I.p[i] = ldv(I.z + i) + beta * ldv(I.p + i);
        cl.sync();
    }
    // no CTA leaves while another may still read its shared memory (the last reduction)
    cl.sync();
    if (cl.block_rank() == 0 && threadIdx.x == 0) {
        ClResult out;
        out.iterations = it;
        out.status = status;
        out.pad = 0;
        out.rzd = rzd;
        out.bd = bd;
        res[inst] = out;
    }
}

// The coarse part of the V-cycle of one large system as one cooperative launch
// (all CTAs resident), in place of a launch per coarse-level step.
template <bool G32>
__global__ void __launch_bounds__(kClThreads, 2) k_coarse_grid(const ClInst* __restrict__ inst, GridBarState* st,
                                                               double* flag, int degree, double alpha) {
    const Vg g{(int)(blockIdx.x * blockDim.x + threadIdx.x), (int)(gridDim.x * blockDim.x)};
    GridBar bar{st, flag, gridDim.x};
    coarse_cycle<G32>(*inst, g, degree, alpha, bar);
}

template <typename VT, bool G32>
void launch_t(const ClInst* insts, ClResult* res, int n, double rtol2, int max_iter, int degree, double alpha,
              cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)n * kClCtas, 1, 1);
    cfg.blockDim = dim3(kClThreads, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kClCtas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    FX_CUDA_CHECK(cudaLaunchKernelEx(&cfg, k_amg_cluster<VT, G32>, insts, res, n, rtol2, max_iter, degree, alpha));
    if (g_launch_counter) ++*g_launch_counter;
    if (debug_sync()) stream_wait(s, "k_amg_cluster", 120.0);
}

}  // namespace

void launch_amg_cluster(const ClInst* insts, ClResult* res, int n, bool fp32, double rtol, int max_iter, int degree,
                        double alpha, cudaStream_t s) {
    if (n <= 0) return;
    if (degree < 1 || degree > 8) fail(FX_INVALID_ARGUMENT, "multigrid smoother degree must be 1..8");
    const double rtol2 = rtol * rtol;
    if (fp32) launch_t<float, true>(insts, res, n, rtol2, max_iter, degree, alpha, s);
    else launch_t<double, false>(insts, res, n, rtol2, max_iter, degree, alpha, s);
}

unsigned coarse_grid_size() {
    static int cached[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 0;
    if (!cached[dev]) {
        int sms = 0, per = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_coarse_grid<true>, kClThreads, 0) != cudaSuccess) {
            cudaGetLastError();
            per = 0;
        }
        int per64 = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per64, k_coarse_grid<false>, kClThreads, 0) != cudaSuccess) {
            cudaGetLastError();
            per64 = 0;
        }
        cached[dev] = std::max(1, sms * std::min(per, per64));
    }
    return (unsigned)cached[dev];
}

void launch_coarse_grid(const ClInst* inst, GridBarState* st, double* flag, bool fp32, int degree, double alpha,
                        cudaStream_t s) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(coarse_grid_size(), 1, 1);
    cfg.blockDim = dim3(kClThreads, 1, 1);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (fp32) FX_CUDA_CHECK(cudaLaunchKernelEx(&cfg, k_coarse_grid<true>, inst, st, flag, degree, alpha));
    else FX_CUDA_CHECK(cudaLaunchKernelEx(&cfg, k_coarse_grid<false>, inst, st, flag, degree, alpha));
    if (g_launch_counter) ++*g_launch_counter;
    if (debug_sync()) stream_wait(s, "k_coarse_grid", 20.0);
}

const void* kernels_anchor_amg_cluster() { return reinterpret_cast<const void*>(&k_amg_cluster<double, false>); }

}  // namespace fx
