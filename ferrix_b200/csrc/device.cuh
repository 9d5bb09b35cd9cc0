// Device-side shared definitions: material tables, element rules, small
// helpers used by the element, assembly and solver kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fx {

constexpr int kPairs20 = 210;  // node pairs a <= b of a C3D20
constexpr int kPairs4 = 10;    // node pairs a <= b of a C3D4
constexpr int kGp20 = 27;

// Device error bits (OR-ed into one int per launch sequence).
constexpr int kErrSingularJ = 1;   // exact zero Jacobian determinant (element.rs:199-201)
constexpr int kErrNoMaterial = 2;  // element without material / elastic constants
constexpr int kErrIndex = 4;       // an index check failed (never expected)

// Material table (TemperatureDependentLUT pools, material.rs:14-69, 233-277).
struct MatDev {
    const int32_t *e_off, *e_len, *nu_off, *nu_len, *a_off, *a_len;
    const double *tref, *t, *v;
    int n_mat;
};

__device__ __forceinline__ double lut_interp(const double* t, const double* v, int n, double temp) {
    if (n == 1 || temp <= t[0]) return v[0];
    if (temp >= t[n - 1]) return v[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = lo + (hi - lo) / 2;
        if (t[mid] <= temp) lo = mid;
        else hi = mid;
    }
    double f = (temp - t[lo]) / (t[hi] - t[lo]);
    return v[lo] + (v[hi] - v[lo]) * f;
}

// Isotropic D of build_elastic_d_matrix (material.rs:202-230) as its three
// distinct entries: d11 = (1-nu) f, d12 = nu f, d44 = (1-2nu)/2 f.
struct Lame {
    double d11, d12, d44;
};

__device__ __forceinline__ bool material_d(const MatDev& m, int k, double T, Lame* out) {
    if (k < 0 || k >= m.n_mat || m.e_len[k] <= 0 || m.nu_len[k] <= 0) return false;
    double e = lut_interp(m.t + m.e_off[k], m.v + m.e_off[k], m.e_len[k], T);
    double nu = lut_interp(m.t + m.nu_off[k], m.v + m.nu_off[k], m.nu_len[k], T);
    double factor = e / ((1.0 + nu) * (1.0 - 2.0 * nu));
    out->d11 = (1.0 - nu) * factor;
    out->d12 = nu * factor;
    out->d44 = ((1.0 - 2.0 * nu) / 2.0) * factor;
    return true;
}

// eps_th(Tc) - eps_th(Ti) (element.rs:284-297); 0 when the material has no *EXPANSION.
__device__ __forceinline__ double thermal_delta(const MatDev& m, int k, double tc, double ti) {
    if (m.a_len[k] <= 0) return 0.0;
    const double* t = m.t + m.a_off[k];
    const double* v = m.v + m.a_off[k];
    int n = m.a_len[k];
    double tref = m.tref[k];
    return lut_interp(t, v, n, tc) * (tc - tref) - lut_interp(t, v, n, ti) * (ti - tref);
}

// 3x3 inverse by adjugate; returns det (exact 0 = singular, as nalgebra's try_inverse).
template <typename T>
__device__ __forceinline__ T inv3(const T J[9], T Ji[9]) {
    T c00 = J[4] * J[8] - J[5] * J[7];
    T c01 = J[5] * J[6] - J[3] * J[8];
    T c02 = J[3] * J[7] - J[4] * J[6];
    T det = J[0] * c00 + J[1] * c01 + J[2] * c02;
    T id = det != T(0) ? T(1) / det : T(0);
    Ji[0] = c00 * id;
    Ji[1] = (J[2] * J[7] - J[1] * J[8]) * id;
    Ji[2] = (J[1] * J[5] - J[2] * J[4]) * id;
    Ji[3] = c01 * id;
    Ji[4] = (J[0] * J[8] - J[2] * J[6]) * id;
    Ji[5] = (J[2] * J[3] - J[0] * J[5]) * id;
    Ji[6] = c02 * id;
    Ji[7] = (J[1] * J[6] - J[0] * J[7]) * id;
    Ji[8] = (J[0] * J[4] - J[1] * J[3]) * id;
    return det;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Element rule tables resident on the device (filled once per context).
struct RuleTables {
    const double* n20_d;   // 27 x 20
    const double* dn20_d;  // 27 x 3 x 20
    const float* n20_f;
    const float* dn20_f;
    const double* w20;     // 27
    const uint8_t* pair20; // 210 x 2 (a, b), a <= b
    const double* dn20_nodes;  // 20 x 3 x 20: shape derivatives at the element's own nodes
};

__host__ __device__ constexpr int pair_index(int npe, int a, int b) {  // a <= b
    return a * npe - (a * (a - 1)) / 2 + (b - a);
}

}  // namespace fx
