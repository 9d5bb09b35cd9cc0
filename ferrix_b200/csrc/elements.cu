// Element kernels for C3D4 and C3D20 (sm_100a, CUDA cores).
//
//  * stiffness: K_e = sum_gp B^T D(T_gp) B |detJ| w (element.rs:217-318) in
//    FP32 (mixed path) or FP64, written as the 3x3 node-pair blocks a <= b of
//    each element into an element buffer; also the largest single-element
//    diagonal entry |v| > 1e-12 (assembler.rs:135-143) used for the penalty.
//    C3D20: one warp per element; lanes 0..19 own a node for the Jacobian and
//    the global derivatives, then every lane accumulates up to 7 of the 210
//    node pairs with the isotropic closed form
//      K_ab[i][i] = d11 ga_i gb_i + d44 (ga.gb - ga_i gb_i)
//      K_ab[i][j] = d12 ga_i gb_j + d44 ga_j gb_i       (i != j)
//    which is B_a^T D B_b for the Voigt B of element.rs:588-606.
//    C3D4: one thread per element (one Gauss point, c3d4.rs:31-51).
//  * apply (FP64): out_e = sum_gp B^T D (cv B v - cth d_th) |detJ| w on X (+uconf).
//    cv=1, cth=1 is compute_internal_force_sdv (element.rs:352-447);
//    cv=1, cth=0 is the tangent applied to a vector (matrix-free K v);
//    cv=0, cth=-1 is compute_thermal_force (element.rs:453-520).
//    Results go to a per-element-node buffer that a node-wise gather sums in
//    a fixed order (deterministic, no atomics).
#include <cuda_runtime.h>

#include <cmath>
#include <vector>

#include "common.hpp"
#include "device.cuh"
#include "kernels.hpp"

namespace fx {

// ------------------------------------------------------------------ tables

static void c3d20_shape(double x, double y, double z, double N[20], double dN[60]) {
    // Serendipity functions in the Abaqus node order (c3d20.rs:61-84).
    static const int L[20][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1},
                                 {1, -1, 1},   {1, 1, 1},   {-1, 1, 1}, {0, -1, -1}, {1, 0, -1},
                                 {0, 1, -1},   {-1, 0, -1}, {0, -1, 1}, {1, 0, 1},   {0, 1, 1},
                                 {-1, 0, 1},   {-1, -1, 0}, {1, -1, 0}, {1, 1, 0},   {-1, 1, 0}};
    for (int a = 0; a < 20; ++a) {
        double xa = L[a][0], ya = L[a][1], za = L[a][2];
        double A = 1.0 + x * xa, B = 1.0 + y * ya, C = 1.0 + z * za;
        if (xa != 0 && ya != 0 && za != 0) {
            double s = x * xa + y * ya + z * za - 2.0;
            N[a] = A * B * C * s / 8.0;
            dN[a] = xa * B * C * (s + A) / 8.0;
            dN[20 + a] = ya * A * C * (s + B) / 8.0;
            dN[40 + a] = za * A * B * (s + C) / 8.0;
        } else if (xa == 0) {
            double q = 1.0 - x * x;
            N[a] = q * B * C / 4.0;
            dN[a] = -2.0 * x * B * C / 4.0;
            dN[20 + a] = q * ya * C / 4.0;
            dN[40 + a] = q * B * za / 4.0;
        } else if (ya == 0) {
            double q = 1.0 - y * y;
            N[a] = A * q * C / 4.0;
            dN[a] = xa * q * C / 4.0;
            dN[20 + a] = -2.0 * y * A * C / 4.0;
            dN[40 + a] = A * q * za / 4.0;
        } else {
            double q = 1.0 - z * z;
            N[a] = A * B * q / 4.0;
            dN[a] = xa * B * q / 4.0;
            dN[20 + a] = A * ya * q / 4.0;
            dN[40 + a] = -2.0 * z * A * B / 4.0;
        }
    }
}

void DeviceTables::init(cudaStream_t s) {
    // 3x3x3 Gauss rule, xi outer, zeta inner (c3d20.rs:31-51)
    const double p[3] = {-0.774596669241483, 0.0, 0.774596669241483};
    const double w[3] = {0.5555555555555556, 0.8888888888888888, 0.5555555555555556};
    std::vector<double> n(27 * 20), dn(27 * 60), wt(27);
    std::vector<float> nf(27 * 20), dnf(27 * 60);
    int g = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k, ++g) {
                c3d20_shape(p[i], p[j], p[k], &n[g * 20], &dn[g * 60]);
                wt[g] = w[i] * w[j] * w[k];
            }
    for (size_t i = 0; i < n.size(); ++i) nf[i] = (float)n[i];
    for (size_t i = 0; i < dn.size(); ++i) dnf[i] = (float)dn[i];
    std::vector<uint8_t> pairs;
    for (int a = 0; a < 20; ++a)
        for (int b = a; b < 20; ++b) {
            pairs.push_back((uint8_t)a);
            pairs.push_back((uint8_t)b);
        }
    // derivatives at the 20 node positions (local coordinates of c3d20.rs:61-84) for stress recovery
    static const double nodes20[20][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}, {-1, -1, 1},
                                          {1, -1, 1},   {1, 1, 1},   {-1, 1, 1}, {0, -1, -1}, {1, 0, -1},
                                          {0, 1, -1},   {-1, 0, -1}, {0, -1, 1}, {1, 0, 1},   {0, 1, 1},
                                          {-1, 0, 1},   {-1, -1, 0}, {1, -1, 0}, {1, 1, 0},   {-1, 1, 0}};
    std::vector<double> nn(20), dnn(20 * 60);
    for (int a = 0; a < 20; ++a) c3d20_shape(nodes20[a][0], nodes20[a][1], nodes20[a][2], nn.data(), &dnn[a * 60]);
    dn20_nodes.upload(dnn, s);
    n20_d.upload(n, s);
    dn20_d.upload(dn, s);
    n20_f.upload(nf, s);
    dn20_f.upload(dnf, s);
    w20.upload(wt, s);
    pair20.upload(pairs, s);
    FX_CUDA_CHECK(cudaStreamSynchronize(s));
}

RuleTables DeviceTables::view() const {
    return RuleTables{n20_d.ptr, dn20_d.ptr, n20_f.ptr, dn20_f.ptr, w20.ptr, pair20.ptr, dn20_nodes.ptr};
}

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ void atomic_max_pos(unsigned long long* dst, double v) {
    // non-negative doubles order like their bit patterns
    atomicMax(dst, (unsigned long long)__double_as_longlong(v));
}

template <typename T>
__device__ __forceinline__ T fmat(T a, T b, T c) {
    if constexpr (sizeof(T) == 8) return fma(a, b, c);
    else return fmaf(a, b, c);
}

// Isotropic B^T D B block of the node pair (a, b) at one Gauss point, accumulated into acc
// (row-major 3x3; g = shape-function gradients, w = weight x |J|, wdm = w (d11 - d44)):
//   K_ab[i][i] += w (d11 - d44) ga_i gb_i + w d44 (ga . gb),
//   K_ab[i][j] += w d12 ga_i gb_j + w d44 ga_j gb_i  (i != j),
// as fused multiply-adds (5 % faster than separate products for C3D20 on B200).
template <typename T>
__device__ __forceinline__ void pair_block(T acc[9], T ga0, T ga1, T ga2, T gb0, T gb1, T gb2, T wdm, T wd12,
                                           T wd44) {
    const T k0 = wd44 * ga0, k1 = wd44 * ga1, k2 = wd44 * ga2;
    const T h0 = wd12 * ga0, h1 = wd12 * ga1, h2 = wd12 * ga2;
    const T s = fmat(k2, gb2, fmat(k1, gb1, k0 * gb0));
    acc[0] = fmat(wdm * ga0, gb0, acc[0] + s);
    acc[4] = fmat(wdm * ga1, gb1, acc[4] + s);
    acc[8] = fmat(wdm * ga2, gb2, acc[8] + s);
    acc[1] = fmat(h0, gb1, fmat(k1, gb0, acc[1]));
    acc[2] = fmat(h0, gb2, fmat(k2, gb0, acc[2]));
    acc[3] = fmat(h1, gb0, fmat(k0, gb1, acc[3]));
    acc[5] = fmat(h1, gb2, fmat(k2, gb1, acc[5]));
    acc[6] = fmat(h2, gb0, fmat(k0, gb2, acc[6]));
    acc[7] = fmat(h2, gb1, fmat(k1, gb2, acc[7]));
}

// ------------------------------------------------------------------ C3D4 stiffness

template <typename T>
__global__ void __launch_bounds__(256) k_stiff4(int nelem, const int32_t* __restrict__ conn,
                                                const int32_t* __restrict__ mat, const double* __restrict__ X,
                                                const double* __restrict__ u, const double* __restrict__ Tcur,
                                                MatDev md, T* __restrict__ ebuf, unsigned long long* maxdiag,
                                                int* err) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nelem) return;
    int nd[4];
    double x[4][3], tc = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        nd[a] = conn[4 * e + a];
#pragma unroll
        for (int c = 0; c < 3; ++c) x[a][c] = X[3 * nd[a] + c] + (u ? u[3 * nd[a] + c] : 0.0);
        tc += 0.25 * Tcur[nd[a]];
    }
    Lame L;
    if (!material_d(md, mat[e], tc, &L)) {
        atomicOr(err, kErrNoMaterial);
        return;
    }
    T J[9], Ji[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        J[c] = (T)(x[1][c] - x[0][c]);
        J[3 + c] = (T)(x[2][c] - x[0][c]);
        J[6 + c] = (T)(x[3][c] - x[0][c]);
    }
    T det = inv3(J, Ji);
    if (det == T(0)) atomicOr(err, kErrSingularJ);
    T w = fabs(det) * (T)(1.0 / 6.0);
    T g[4][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        g[1][i] = Ji[3 * i + 0];
        g[2][i] = Ji[3 * i + 1];
        g[3][i] = Ji[3 * i + 2];
        g[0][i] = -Ji[3 * i + 0] - Ji[3 * i + 1] - Ji[3 * i + 2];
    }
    T wdm = w * (T)(L.d11 - L.d44), wd12 = w * (T)L.d12, wd44 = w * (T)L.d44;
    T* out = ebuf + (size_t)e * kPairs4 * 9;
    double dmax = 0.0;
    int p = 0;
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = a; b < 4; ++b, ++p) {
            T acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            pair_block(acc, g[a][0], g[a][1], g[a][2], g[b][0], g[b][1], g[b][2], wdm, wd12, wd44);
#pragma unroll
            for (int c = 0; c < 9; ++c) out[p * 9 + c] = acc[c];
            if (a == b) {
                double d0 = fabs((double)acc[0]), d1 = fabs((double)acc[4]), d2 = fabs((double)acc[8]);
                if (d0 > 1e-12) dmax = fmax(dmax, d0);
                if (d1 > 1e-12) dmax = fmax(dmax, d1);
                if (d2 > 1e-12) dmax = fmax(dmax, d2);
            }
        }
    if (dmax > 0.0) atomic_max_pos(maxdiag, dmax);
}

// ------------------------------------------------------------------ C3D20 stiffness

constexpr int kWarps20 = 8;

template <typename T>
__global__ void __launch_bounds__(256) k_stiff20(int nelem, const int32_t* __restrict__ conn,
                                                 const int32_t* __restrict__ mat, const double* __restrict__ X,
                                                 const double* __restrict__ u, const double* __restrict__ Tcur,
                                                 MatDev md, RuleTables rt, T* __restrict__ ebuf,
                                                 unsigned long long* maxdiag, int* err) {
    __shared__ T s_dn[kGp20 * 60];
    __shared__ double s_n[kGp20 * 20];
    __shared__ double s_w[kGp20];
    __shared__ uint8_t s_pair[kPairs20 * 2];
    __shared__ T s_g[kWarps20][64];
    const T* dn_src;
    if constexpr (sizeof(T) == 8) dn_src = (const T*)rt.dn20_d;
    else dn_src = (const T*)rt.dn20_f;
    for (int i = threadIdx.x; i < kGp20 * 60; i += blockDim.x) s_dn[i] = dn_src[i];
    for (int i = threadIdx.x; i < kGp20 * 20; i += blockDim.x) s_n[i] = rt.n20_d[i];
    for (int i = threadIdx.x; i < kGp20; i += blockDim.x) s_w[i] = rt.w20[i];
    for (int i = threadIdx.x; i < kPairs20 * 2; i += blockDim.x) s_pair[i] = rt.pair20[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int e = blockIdx.x * kWarps20 + warp;
    if (e >= nelem) return;
    const int k = mat[e];
    if (k < 0 || k >= md.n_mat || md.e_len[k] <= 0 || md.nu_len[k] <= 0) {
        if (lane == 0) atomicOr(err, kErrNoMaterial);
        return;
    }
    const bool t_dep = md.e_len[k] > 1 || md.nu_len[k] > 1;
    T x0 = 0, x1 = 0, x2 = 0;
    double ta = 0.0;
    if (lane < 20) {
        int nd = conn[20 * e + lane];
        double a0 = X[3 * nd], a1 = X[3 * nd + 1], a2 = X[3 * nd + 2];
        if (u) {
            a0 += u[3 * nd];
            a1 += u[3 * nd + 1];
            a2 += u[3 * nd + 2];
        }
        x0 = (T)a0;
        x1 = (T)a1;
        x2 = (T)a2;
        ta = Tcur[nd];
    }
    Lame L;
    if (!t_dep) material_d(md, k, 0.0, &L);
    T acc[7][9];
#pragma unroll
    for (int q = 0; q < 7; ++q)
#pragma unroll
        for (int c = 0; c < 9; ++c) acc[q][c] = 0;
    int bad = 0;
    for (int gp = 0; gp < kGp20; ++gp) {
        T d0 = 0, d1 = 0, d2 = 0;
        if (lane < 20) {
            d0 = s_dn[gp * 60 + lane];
            d1 = s_dn[gp * 60 + 20 + lane];
            d2 = s_dn[gp * 60 + 40 + lane];
        }
        T J[9] = {d0 * x0, d0 * x1, d0 * x2, d1 * x0, d1 * x1, d1 * x2, d2 * x0, d2 * x1, d2 * x2};
#pragma unroll
        for (int c = 0; c < 9; ++c) J[c] = warp_sum(J[c]);
        if (t_dep) {
            double tg = warp_sum(lane < 20 ? s_n[gp * 20 + lane] * ta : 0.0);
            material_d(md, k, tg, &L);
        }
        T Ji[9];
        T det = inv3(J, Ji);
        if (det == T(0)) bad = 1;
        T w = fabs(det) * (T)s_w[gp];
        if (lane < 20) {
            s_g[warp][3 * lane + 0] = Ji[0] * d0 + Ji[1] * d1 + Ji[2] * d2;
            s_g[warp][3 * lane + 1] = Ji[3] * d0 + Ji[4] * d1 + Ji[5] * d2;
            s_g[warp][3 * lane + 2] = Ji[6] * d0 + Ji[7] * d1 + Ji[8] * d2;
        }
        __syncwarp();
        T wdm = w * (T)(L.d11 - L.d44), wd12 = w * (T)L.d12, wd44 = w * (T)L.d44;
#pragma unroll
        for (int q = 0; q < 7; ++q) {
            int p = lane + 32 * q;
            if (p < kPairs20) {
                int a = s_pair[2 * p], b = s_pair[2 * p + 1];
                const T* ga = &s_g[warp][3 * a];
                const T* gb = &s_g[warp][3 * b];
                pair_block(acc[q], ga[0], ga[1], ga[2], gb[0], gb[1], gb[2], wdm, wd12, wd44);
            }
        }
        __syncwarp();
    }
    if (bad && lane == 0) atomicOr(err, kErrSingularJ);
    T* out = ebuf + (size_t)e * kPairs20 * 9;
    double dmax = 0.0;
#pragma unroll
    for (int q = 0; q < 7; ++q) {
        int p = lane + 32 * q;
        if (p < kPairs20) {
#pragma unroll
            for (int c = 0; c < 9; ++c) out[p * 9 + c] = acc[q][c];
            if (s_pair[2 * p] == s_pair[2 * p + 1]) {
                double v0 = fabs((double)acc[q][0]), v1 = fabs((double)acc[q][4]), v2 = fabs((double)acc[q][8]);
                if (v0 > 1e-12) dmax = fmax(dmax, v0);
                if (v1 > 1e-12) dmax = fmax(dmax, v1);
                if (v2 > 1e-12) dmax = fmax(dmax, v2);
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    if (lane == 0 && dmax > 0.0) atomic_max_pos(maxdiag, dmax);
}

// ------------------------------------------------------------------ FP64 apply

struct ApplyArgs {
    const double* uconf;  // coordinates X + uconf (nullable)
    const double* v;      // strain source (nullable = 0)
    const double* tinit;
    const double* tcur;
    double cv, cth;
};

__device__ __forceinline__ void stress_from(const Lame& L, const double e[6], double s[6]) {
    s[0] = L.d11 * e[0] + L.d12 * (e[1] + e[2]);
    s[1] = L.d11 * e[1] + L.d12 * (e[0] + e[2]);
    s[2] = L.d11 * e[2] + L.d12 * (e[0] + e[1]);
    s[3] = L.d44 * e[3];
    s[4] = L.d44 * e[4];
    s[5] = L.d44 * e[5];
}

__global__ void __launch_bounds__(256) k_apply4(int nelem, const int32_t* __restrict__ conn,
                                                const int32_t* __restrict__ mat, const double* __restrict__ X,
                                                ApplyArgs A, MatDev md, double* __restrict__ fe, int* err) {
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nelem) return;
    int nd[4];
    double x[4][3], v[4][3], tc = 0.0, ti = 0.0;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        nd[a] = conn[4 * e + a];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            x[a][c] = X[3 * nd[a] + c] + (A.uconf ? A.uconf[3 * nd[a] + c] : 0.0);
            v[a][c] = A.v ? A.v[3 * nd[a] + c] : 0.0;
        }
        tc += 0.25 * A.tcur[nd[a]];
        ti += 0.25 * A.tinit[nd[a]];
    }
    const int k = mat[e];
    Lame L;
    double* out = fe + (size_t)e * 12;
    if (!material_d(md, k, tc, &L)) {
        atomicOr(err, kErrNoMaterial);
        return;
    }
    double J[9], Ji[9];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        J[c] = x[1][c] - x[0][c];
        J[3 + c] = x[2][c] - x[0][c];
        J[6 + c] = x[3][c] - x[0][c];
    }
    double det = inv3(J, Ji);
    if (det == 0.0) atomicOr(err, kErrSingularJ);
    double w = fabs(det) * (1.0 / 6.0);
    double g[4][3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        g[1][i] = Ji[3 * i + 0];
        g[2][i] = Ji[3 * i + 1];
        g[3][i] = Ji[3 * i + 2];
        g[0][i] = -Ji[3 * i + 0] - Ji[3 * i + 1] - Ji[3 * i + 2];
    }
    double eps[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        eps[0] += g[a][0] * v[a][0];
        eps[1] += g[a][1] * v[a][1];
        eps[2] += g[a][2] * v[a][2];
        eps[3] += g[a][1] * v[a][0] + g[a][0] * v[a][1];
        eps[4] += g[a][2] * v[a][1] + g[a][1] * v[a][2];
        eps[5] += g[a][2] * v[a][0] + g[a][0] * v[a][2];
    }
    double dth = A.cth != 0.0 ? thermal_delta(md, k, tc, ti) : 0.0;
#pragma unroll
    for (int i = 0; i < 6; ++i) eps[i] *= A.cv;
    eps[0] -= A.cth * dth;
    eps[1] -= A.cth * dth;
    eps[2] -= A.cth * dth;
    double s[6];
    stress_from(L, eps, s);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        out[3 * a + 0] = (g[a][0] * s[0] + g[a][1] * s[3] + g[a][2] * s[5]) * w;
        out[3 * a + 1] = (g[a][1] * s[1] + g[a][0] * s[3] + g[a][2] * s[4]) * w;
        out[3 * a + 2] = (g[a][2] * s[2] + g[a][1] * s[4] + g[a][0] * s[5]) * w;
    }
}

__global__ void __launch_bounds__(256) k_apply20(int nelem, const int32_t* __restrict__ conn,
                                                 const int32_t* __restrict__ mat, const double* __restrict__ X,
                                                 ApplyArgs A, MatDev md, RuleTables rt, double* __restrict__ fe,
                                                 int* err) {
    __shared__ double s_dn[kGp20 * 60];
    __shared__ double s_n[kGp20 * 20];
    __shared__ double s_w[kGp20];
    for (int i = threadIdx.x; i < kGp20 * 60; i += blockDim.x) s_dn[i] = rt.dn20_d[i];
    for (int i = threadIdx.x; i < kGp20 * 20; i += blockDim.x) s_n[i] = rt.n20_d[i];
    for (int i = threadIdx.x; i < kGp20; i += blockDim.x) s_w[i] = rt.w20[i];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int e = blockIdx.x * kWarps20 + warp;
    if (e >= nelem) return;
    const int k = mat[e];
    if (k < 0 || k >= md.n_mat || md.e_len[k] <= 0 || md.nu_len[k] <= 0) {
        if (lane == 0) atomicOr(err, kErrNoMaterial);
        return;
    }
    const bool thermal = A.cth != 0.0 && md.a_len[k] > 0;
    const bool t_dep = md.e_len[k] > 1 || md.nu_len[k] > 1 || thermal;
    double x0 = 0, x1 = 0, x2 = 0, v0 = 0, v1 = 0, v2 = 0, tca = 0, tia = 0;
    if (lane < 20) {
        int nd = conn[20 * e + lane];
        x0 = X[3 * nd];
        x1 = X[3 * nd + 1];
        x2 = X[3 * nd + 2];
        if (A.uconf) {
            x0 += A.uconf[3 * nd];
            x1 += A.uconf[3 * nd + 1];
            x2 += A.uconf[3 * nd + 2];
        }
        if (A.v) {
            v0 = A.v[3 * nd];
            v1 = A.v[3 * nd + 1];
            v2 = A.v[3 * nd + 2];
        }
        tca = A.tcur[nd];
        tia = A.tinit[nd];
    }
    Lame L;
    if (!t_dep) material_d(md, k, 0.0, &L);
    double f0 = 0, f1 = 0, f2 = 0;
    int bad = 0;
    for (int gp = 0; gp < kGp20; ++gp) {
        double d0 = 0, d1 = 0, d2 = 0;
        if (lane < 20) {
            d0 = s_dn[gp * 60 + lane];
            d1 = s_dn[gp * 60 + 20 + lane];
            d2 = s_dn[gp * 60 + 40 + lane];
        }
        double J[9] = {d0 * x0, d0 * x1, d0 * x2, d1 * x0, d1 * x1, d1 * x2, d2 * x0, d2 * x1, d2 * x2};
#pragma unroll
        for (int c = 0; c < 9; ++c) J[c] = warp_sum(J[c]);
        double dth = 0.0;
        if (t_dep) {
            double nn = lane < 20 ? s_n[gp * 20 + lane] : 0.0;
            double tc = warp_sum(nn * tca);
            material_d(md, k, tc, &L);
            if (thermal) {
                double ti = warp_sum(nn * tia);
                dth = thermal_delta(md, k, tc, ti);
            }
        }
        double Ji[9];
        double det = inv3(J, Ji);
        if (det == 0.0) bad = 1;
        double w = fabs(det) * s_w[gp];
        double g0 = Ji[0] * d0 + Ji[1] * d1 + Ji[2] * d2;
        double g1 = Ji[3] * d0 + Ji[4] * d1 + Ji[5] * d2;
        double g2 = Ji[6] * d0 + Ji[7] * d1 + Ji[8] * d2;
        double eps[6];
        if (A.cv != 0.0) {
            eps[0] = warp_sum(g0 * v0);
            eps[1] = warp_sum(g1 * v1);
            eps[2] = warp_sum(g2 * v2);
            eps[3] = warp_sum(g1 * v0 + g0 * v1);
            eps[4] = warp_sum(g2 * v1 + g1 * v2);
            eps[5] = warp_sum(g2 * v0 + g0 * v2);
#pragma unroll
            for (int i = 0; i < 6; ++i) eps[i] *= A.cv;
        } else {
#pragma unroll
            for (int i = 0; i < 6; ++i) eps[i] = 0.0;
        }
        eps[0] -= A.cth * dth;
        eps[1] -= A.cth * dth;
        eps[2] -= A.cth * dth;
        double s[6];
        stress_from(L, eps, s);
        f0 += (g0 * s[0] + g1 * s[3] + g2 * s[5]) * w;
        f1 += (g1 * s[1] + g0 * s[3] + g2 * s[4]) * w;
        f2 += (g2 * s[2] + g1 * s[4] + g0 * s[5]) * w;
    }
    if (bad && lane == 0) atomicOr(err, kErrSingularJ);
    if (lane < 20) {
        double* out = fe + ((size_t)e * 20 + lane) * 3;
        out[0] = f0;
        out[1] = f1;
        out[2] = f2;
    }
}

// Node-wise fixed-order sum of element-node contributions: out[3i+c] = sum fe[s*3+c].
__global__ void k_node_gather(int n_nodes, const int32_t* __restrict__ ptr, const int32_t* __restrict__ slots,
                              const double* __restrict__ fe, double* __restrict__ out) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    double a0 = 0, a1 = 0, a2 = 0;
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
        const double* f = fe + (size_t)slots[k] * 3;
        a0 += f[0];
        a1 += f[1];
        a2 += f[2];
    }
    out[3 * i] = a0;
    out[3 * i + 1] = a1;
    out[3 * i + 2] = a2;
}

// ------------------------------------------------------------------ stress recovery
// StaticStep::calculate_stress_strain (static_step.rs:271-379) with
// Element::calculate_stress_strain_at_local_coords (element.rs:526-566): at every
// node of every element, strain = B(xi_node) u_e on the undeformed coordinates,
// minus the thermal strain change alpha(Tc)(Tc - Tref) - alpha(Ti)(Ti - Tref) on
// the normal components, stress = D(E(Tc), nu(Tc)) strain (update_state of the
// elastic material, material.rs:180-195). One thread per (element, node); the
// 12 values go to the element-node slot and are averaged per node in a fixed
// order (element count = slots of the node).
template <int NPE>
__global__ void __launch_bounds__(128) k_node_stress(int nelem, const int32_t* __restrict__ conn,
                                                     const int32_t* __restrict__ mat, const double* __restrict__ X,
                                                     const double* __restrict__ u, const double* __restrict__ tinit,
                                                     const double* __restrict__ tcur, MatDev md, RuleTables rt,
                                                     double* __restrict__ out, int* __restrict__ err) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nelem * NPE) return;
    const int e = (int)(t / NPE), a = (int)(t % NPE);
    const int32_t* cn = conn + (int64_t)e * NPE;
    const int k = mat[e];
    double* o = out + t * 12;
    // local derivatives at this node: C3D4 constant (c3d4.rs:31-51), C3D20 tabulated
    auto dnl = [&](int d, int b) -> double {
        if (NPE == 4) return b == 0 ? -1.0 : (b == d + 1 ? 1.0 : 0.0);
        return rt.dn20_nodes[a * 60 + d * 20 + b];
    };
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = 0; b < NPE; ++b) {
        const double* xb = X + 3 * (int64_t)cn[b];
        for (int d = 0; d < 3; ++d) {
            const double g = dnl(d, b);
            J[d * 3] += g * xb[0];
            J[d * 3 + 1] += g * xb[1];
            J[d * 3 + 2] += g * xb[2];
        }
    }
    double Ji[9];
    const double det = inv3(J, Ji);
    Lame L;
    if (det == 0.0) {
        atomicOr(err, kErrSingularJ);
        for (int c = 0; c < 12; ++c) o[c] = 0.0;
        return;
    }
    const int node = cn[a];
    const double tc = tcur[node], ti = tinit[node];
    if (k < 0 || !material_d(md, k, tc, &L)) {
        atomicOr(err, kErrNoMaterial);
        for (int c = 0; c < 12; ++c) o[c] = 0.0;
        return;
    }
    double eps[6] = {0, 0, 0, 0, 0, 0};
    for (int b = 0; b < NPE; ++b) {
        const double l0 = dnl(0, b), l1 = dnl(1, b), l2 = dnl(2, b);
        const double gx = Ji[0] * l0 + Ji[1] * l1 + Ji[2] * l2;  // dn_global = inv(J) dn_local
        const double gy = Ji[3] * l0 + Ji[4] * l1 + Ji[5] * l2;
        const double gz = Ji[6] * l0 + Ji[7] * l1 + Ji[8] * l2;
        const double* ub = u + 3 * (int64_t)cn[b];
        eps[0] += gx * ub[0];
        eps[1] += gy * ub[1];
        eps[2] += gz * ub[2];
        eps[3] += gy * ub[0] + gx * ub[1];  // engineering shear, B rows of element.rs:588-606
        eps[4] += gz * ub[1] + gy * ub[2];
        eps[5] += gz * ub[0] + gx * ub[2];
    }
    const double dth = thermal_delta(md, k, tc, ti);
    eps[0] -= dth;
    eps[1] -= dth;
    eps[2] -= dth;
    o[0] = L.d11 * eps[0] + L.d12 * (eps[1] + eps[2]);
    o[1] = L.d11 * eps[1] + L.d12 * (eps[0] + eps[2]);
    o[2] = L.d11 * eps[2] + L.d12 * (eps[0] + eps[1]);
    o[3] = L.d44 * eps[3];
    o[4] = L.d44 * eps[4];
    o[5] = L.d44 * eps[5];
    for (int c = 0; c < 6; ++c) o[6 + c] = eps[c];
}

__global__ void k_node_average12(int n_nodes, const int32_t* __restrict__ ptr, const int32_t* __restrict__ slots,
                                 const double* __restrict__ in, double* __restrict__ S, double* __restrict__ E) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_nodes) return;
    double acc[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int cnt = ptr[i + 1] - ptr[i];
    for (int k = ptr[i]; k < ptr[i + 1]; ++k) {
        const double* f = in + (size_t)slots[k] * 12;
        for (int c = 0; c < 12; ++c) acc[c] += f[c];
    }
    for (int c = 0; c < 6; ++c) {
        S[6 * (int64_t)i + c] = cnt ? acc[c] / cnt : 0.0;
        E[6 * (int64_t)i + c] = cnt ? acc[6 + c] / cnt : 0.0;
    }
}

void launch_nodal_stress(const ElemView& g4, const ElemView& g20, const double* X, const double* u,
                         const double* tinit, const double* tcur, const MatDev& md, const RuleTables& rt, int n_nodes,
                         const int32_t* node_ptr, const int32_t* node_slots, double* slot_buf, double* S, double* E,
                         int* err, cudaStream_t s) {
    if (g4.n)
        FX_LAUNCH(k_node_stress<4>, (unsigned)(((int64_t)g4.n * 4 + 127) / 128), 128, 0, s, g4.n, g4.conn, g4.mat, X,
                  u, tinit, tcur, md, rt, slot_buf, err);
    if (g20.n)
        FX_LAUNCH(k_node_stress<20>, (unsigned)(((int64_t)g20.n * 20 + 127) / 128), 128, 0, s, g20.n, g20.conn,
                  g20.mat, X, u, tinit, tcur, md, rt, slot_buf + (size_t)g4.n * 4 * 12, err);
    if (n_nodes) FX_LAUNCH(k_node_average12, (n_nodes + 255) / 256, 256, 0, s, n_nodes, node_ptr, node_slots, slot_buf, S, E);
}

// ------------------------------------------------------------------ launchers

template <typename T>
void launch_stiffness(const ElemView& g4, const ElemView& g20, const double* X, const double* u, const double* Tcur,
                      const MatDev& md, const RuleTables& rt, T* ebuf, unsigned long long* maxdiag, int* err,
                      cudaStream_t s) {
    if (g4.n) FX_LAUNCH(k_stiff4<T>, (g4.n + 255) / 256, 256, 0, s, g4.n, g4.conn, g4.mat, X, u, Tcur, md, ebuf,
                        maxdiag, err);
    if (g20.n)
        FX_LAUNCH(k_stiff20<T>, (g20.n + kWarps20 - 1) / kWarps20, 256, 0, s, g20.n, g20.conn, g20.mat, X, u, Tcur,
                  md, rt, ebuf + (size_t)g4.n * kPairs4 * 9, maxdiag, err);
}
template void launch_stiffness<float>(const ElemView&, const ElemView&, const double*, const double*, const double*,
                                      const MatDev&, const RuleTables&, float*, unsigned long long*, int*,
                                      cudaStream_t);
template void launch_stiffness<double>(const ElemView&, const ElemView&, const double*, const double*,
                                       const double*, const MatDev&, const RuleTables&, double*,
                                       unsigned long long*, int*, cudaStream_t);

void launch_apply(const ElemView& g4, const ElemView& g20, const double* X, const double* uconf, const double* v,
                  const double* tinit, const double* tcur, double cv, double cth, const MatDev& md,
                  const RuleTables& rt, double* fe, int* err, cudaStream_t s) {
    ApplyArgs A{uconf, v, tinit, tcur, cv, cth};
    if (g4.n) FX_LAUNCH(k_apply4, (g4.n + 255) / 256, 256, 0, s, g4.n, g4.conn, g4.mat, X, A, md, fe, err);
    if (g20.n)
        FX_LAUNCH(k_apply20, (g20.n + kWarps20 - 1) / kWarps20, 256, 0, s, g20.n, g20.conn, g20.mat, X, A, md, rt,
                  fe + (size_t)g4.n * 4 * 3, err);
}

void launch_node_gather(int n_nodes, const int32_t* ptr, const int32_t* slots, const double* fe, double* out,
                        cudaStream_t s) {
    if (n_nodes) FX_LAUNCH(k_node_gather, (n_nodes + 255) / 256, 256, 0, s, n_nodes, ptr, slots, fe, out);
}

// A kernel of this file's module (preload_kernels() loads all of the module's kernels).
const void* kernels_anchor_elements() { return reinterpret_cast<const void*>(&k_stiff4<double>); }

}  // namespace fx
