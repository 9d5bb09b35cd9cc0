/*
 * ORACLE — test infrastructure only. Not part of the product path.
 *
 * FP64 CPU restatement of the FerriX element, material and assembly loops.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * this library, and only as the checker / timed CPU baseline.
 *
 * What it restates (reference paths relative to the FerriX crate root):
 *   - TemperatureDependentLUT::interpolate        src/solver/material.rs:36-68
 *   - Material::build_elastic_d_matrix            src/solver/material.rs:202-230
 *   - Material::update_state (linear elastic)     src/solver/material.rs:180-195
 *   - C3D4 shape functions + 1-point rule         src/solver/mesh_lib/elements/c3d4.rs:31-51
 *   - C3D20 27-point rule (xi outer, zeta inner)  src/solver/mesh_lib/elements/c3d20.rs:31-51
 *   - C3D20 serendipity shape functions           src/solver/mesh_lib/elements/c3d20.rs:90-213
 *     (written here from the textbook serendipity formulas in the Abaqus
 *      node order of c3d20.rs:61-84; same functions, own derivation)
 *   - Element::compute_stiffness_sdv              src/solver/mesh_lib/elements/element.rs:217-318
 *   - Element::compute_internal_force_sdv         src/solver/mesh_lib/elements/element.rs:352-447
 *   - Element::compute_thermal_force              src/solver/mesh_lib/elements/element.rs:453-520
 *   - build_b_matrix_internal (Voigt xx,yy,zz,xy,yz,zx, engineering shear)
 *                                                 src/solver/mesh_lib/elements/element.rs:588-606
 *   - Assembler::assemble (serial loop, |v|>1e-12 filter, max single-element
 *     diagonal entry)                             src/solver/assembler.rs:37-151
 *   - Assembler::assemble_internal_force          src/solver/assembler.rs:157-241
 *   - Assembler::assemble_thermal_force           src/solver/assembler.rs:247-299
 *
 * The reference iterates a HashMap of elements; this restatement iterates
 * the caller's element order (ascending element id), which changes only the
 * rounding of the sums.
 *
 * Return codes: 0 ok, 1 singular Jacobian (NumericalError), 2 material has no
 * Young's modulus / Poisson ratio (InvalidModelState), 3 element without a
 * material (InvalidModelState).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include <stdlib.h>

#define OR_OK 0
#define OR_SINGULAR 1
#define OR_NO_ELASTIC 2
#define OR_NO_MATERIAL 3

/* ---------------------------------------------------------------- material */

/* Clamped, binary-searched linear interpolation (material.rs:36-68). */
double or_lut_interp(const double* t, const double* v, int n, double temp) {
    if (n == 1 || temp <= t[0]) return v[0];
    if (temp >= t[n - 1]) return v[n - 1];
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = lo + (hi - lo) / 2;
        if (t[mid] <= temp) lo = mid; else hi = mid;
    }
    double f = (temp - t[lo]) / (t[hi] - t[lo]);
    return v[lo] + (v[hi] - v[lo]) * f;
}

/* Material table: per material, offsets/lengths into the shared (t, v) pools
 * for E, nu and alpha (length 0 = property absent) plus the ZERO temperature. */
typedef struct {
    const int* e_off; const int* e_len;
    const int* nu_off; const int* nu_len;
    const int* a_off; const int* a_len;
    const double* tref;
    const double* lut_t; const double* lut_v;
} or_mats;

static int mat_has_alpha(const or_mats* m, int k) { return m->a_len[k] > 0; }
static double mat_alpha(const or_mats* m, int k, double T) {
    return or_lut_interp(m->lut_t + m->a_off[k], m->lut_v + m->a_off[k], m->a_len[k], T);
}

/* Isotropic D (material.rs:202-230): D = factor * [[c1 c2 c2],[c2 c1 c2],[c2 c2 c1], c3 I3]. */
static int mat_dmatrix(const or_mats* m, int k, double T, double D[36]) {
    if (m->e_len[k] <= 0 || m->nu_len[k] <= 0) return OR_NO_ELASTIC;
    double e = or_lut_interp(m->lut_t + m->e_off[k], m->lut_v + m->e_off[k], m->e_len[k], T);
    double nu = or_lut_interp(m->lut_t + m->nu_off[k], m->lut_v + m->nu_off[k], m->nu_len[k], T);
    double factor = e / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double c1 = 1.0 - nu, c2 = nu, c3 = (1.0 - 2.0 * nu) / 2.0;
    memset(D, 0, 36 * sizeof(double));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) D[i * 6 + j] = (i == j ? c1 : c2) * factor;
    for (int i = 3; i < 6; ++i) D[i * 6 + i] = c3 * factor;
    return OR_OK;
}

/* ---------------------------------------------------------------- elements */

/* Abaqus C3D20 node order in the parent cube (c3d20.rs:61-84). */
static const signed char C20_LOC[20][3] = {
    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
    {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1},
    {0, -1, -1},  {1, 0, -1},  {0, 1, -1}, {-1, 0, -1},
    {0, -1, 1},   {1, 0, 1},   {0, 1, 1},  {-1, 0, 1},
    {-1, -1, 0},  {1, -1, 0},  {1, 1, 0},  {-1, 1, 0}};

/* Serendipity shape functions and parent-space derivatives.
 *  corner:  N = (1+x xa)(1+y ya)(1+z za)(x xa + y ya + z za - 2)/8
 *  edge with xa = 0: N = (1-x^2)(1+y ya)(1+z za)/4   (and cyclic)
 * dN is row-major 3 x 20 (d/dxi, d/deta, d/dzeta). */
void or_shape_c3d20(double x, double y, double z, double N[20], double dN[60]) {
    for (int a = 0; a < 20; ++a) {
        double xa = C20_LOC[a][0], ya = C20_LOC[a][1], za = C20_LOC[a][2];
        double A = 1.0 + x * xa, B = 1.0 + y * ya, C = 1.0 + z * za;
        if (xa != 0 && ya != 0 && za != 0) {
            double s = x * xa + y * ya + z * za - 2.0;
            N[a] = A * B * C * s / 8.0;
            dN[0 * 20 + a] = xa * B * C * (s + A) / 8.0;
            dN[1 * 20 + a] = ya * A * C * (s + B) / 8.0;
            dN[2 * 20 + a] = za * A * B * (s + C) / 8.0;
        } else if (xa == 0) {
            double q = 1.0 - x * x;
            N[a] = q * B * C / 4.0;
            dN[0 * 20 + a] = -2.0 * x * B * C / 4.0;
            dN[1 * 20 + a] = q * ya * C / 4.0;
            dN[2 * 20 + a] = q * B * za / 4.0;
        } else if (ya == 0) {
            double q = 1.0 - y * y;
            N[a] = A * q * C / 4.0;
            dN[0 * 20 + a] = xa * q * C / 4.0;
            dN[1 * 20 + a] = -2.0 * y * A * C / 4.0;
            dN[2 * 20 + a] = A * q * za / 4.0;
        } else {
            double q = 1.0 - z * z;
            N[a] = A * B * q / 4.0;
            dN[0 * 20 + a] = xa * B * q / 4.0;
            dN[1 * 20 + a] = A * ya * q / 4.0;
            dN[2 * 20 + a] = -2.0 * z * A * B / 4.0;
        }
    }
}

/* Linear tet (c3d4.rs:38-51). */
void or_shape_c3d4(double x, double y, double z, double N[4], double dN[12]) {
    N[0] = 1.0 - x - y - z; N[1] = x; N[2] = y; N[3] = z;
    static const double d[12] = {-1, 1, 0, 0, -1, 0, 1, 0, -1, 0, 0, 1};
    memcpy(dN, d, sizeof(d));
}

/* Integration rules: C3D4 1 point (c3d4.rs:31-36); C3D20 3x3x3 Gauss with
 * xi outer, zeta inner (c3d20.rs:31-51). */
int or_gauss_points(int npe, double* pts /* ngp*3 */, double* wts /* ngp */) {
    if (npe == 4) {
        pts[0] = pts[1] = pts[2] = 0.25; wts[0] = 1.0 / 6.0; return 1;
    }
    const double p[3] = {-0.774596669241483, 0.0, 0.774596669241483};
    const double w[3] = {0.5555555555555556, 0.8888888888888888, 0.5555555555555556};
    int g = 0;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) {
                pts[g * 3 + 0] = p[i]; pts[g * 3 + 1] = p[j]; pts[g * 3 + 2] = p[k];
                wts[g] = w[i] * w[j] * w[k]; ++g;
            }
    return 27;
}

static void shape(int npe, const double* gp, double* N, double* dN) {
    if (npe == 4) or_shape_c3d4(gp[0], gp[1], gp[2], N, dN);
    else or_shape_c3d20(gp[0], gp[1], gp[2], N, dN);
}

/* J = dN_local (3 x n) * X^T (n x 3); det by cofactor expansion; inverse by
 * adjugate / det; exact-zero det is the singular case (nalgebra try_inverse). */
static int jacobian(int n, const double* dN, const double* xyz, double Jinv[9], double* detJ) {
    double J[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int a = 0; a < n; ++a) s += dN[i * n + a] * xyz[a * 3 + j];
            J[i * 3 + j] = s;
        }
    double c00 = J[4] * J[8] - J[5] * J[7];
    double c01 = J[5] * J[6] - J[3] * J[8];
    double c02 = J[3] * J[7] - J[4] * J[6];
    double det = J[0] * c00 + J[1] * c01 + J[2] * c02;
    *detJ = det;
    if (det == 0.0) return OR_SINGULAR;
    double id = 1.0 / det;
    Jinv[0] = c00 * id;
    Jinv[1] = (J[2] * J[7] - J[1] * J[8]) * id;
    Jinv[2] = (J[1] * J[5] - J[2] * J[4]) * id;
    Jinv[3] = c01 * id;
    Jinv[4] = (J[0] * J[8] - J[2] * J[6]) * id;
    Jinv[5] = (J[2] * J[3] - J[0] * J[5]) * id;
    Jinv[6] = c02 * id;
    Jinv[7] = (J[1] * J[6] - J[0] * J[7]) * id;
    Jinv[8] = (J[0] * J[4] - J[1] * J[3]) * id;
    return OR_OK;
}

/* B (6 x 3n, row-major) from global derivatives g (3 x n). */
static void bmatrix(int n, const double* g, double* B) {
    int m = 3 * n;
    memset(B, 0, 6 * m * sizeof(double));
    for (int a = 0; a < n; ++a) {
        int c = 3 * a;
        double dx = g[0 * n + a], dy = g[1 * n + a], dz = g[2 * n + a];
        B[0 * m + c] = dx;
        B[1 * m + c + 1] = dy;
        B[2 * m + c + 2] = dz;
        B[3 * m + c] = dy; B[3 * m + c + 1] = dx;
        B[4 * m + c + 1] = dz; B[4 * m + c + 2] = dy;
        B[5 * m + c] = dz; B[5 * m + c + 2] = dx;
    }
}

typedef struct {
    int npe, ngp;
    double pts[81], wts[27];
    double N[27][20], dN[27][60];
} rule_t;

static void make_rule(int npe, rule_t* r) {
    r->npe = npe;
    r->ngp = or_gauss_points(npe, r->pts, r->wts);
    for (int g = 0; g < r->ngp; ++g) shape(npe, r->pts + 3 * g, r->N[g], r->dN[g]);
}

/* Per Gauss point: coordinates -> (g = dN_global (3 x n), weight). */
static int gp_geometry(const rule_t* r, int g, const double* xyz, double* gl, double* weight) {
    int n = r->npe;
    double Jinv[9], det;
    int rc = jacobian(n, r->dN[g], xyz, Jinv, &det);
    if (rc) return rc;
    for (int i = 0; i < 3; ++i)
        for (int a = 0; a < n; ++a)
            gl[i * n + a] = Jinv[i * 3 + 0] * r->dN[g][0 * n + a] + Jinv[i * 3 + 1] * r->dN[g][1 * n + a] +
                            Jinv[i * 3 + 2] * r->dN[g][2 * n + a];
    *weight = fabs(det) * r->wts[g];
    return OR_OK;
}

/* Thermal strain increment eps_th(Tc) - eps_th(Ti) (element.rs:284-297). */
static double thermal_delta(const or_mats* m, int k, double tc, double ti) {
    double ac = mat_alpha(m, k, tc);
    double tref = m->tref[k];
    double ai = mat_alpha(m, k, ti);
    return ac * (tc - tref) - ai * (ti - tref);
}

static void gather_xyz(int n, const int* conn_e, const double* X, const double* u, double* xyz) {
    for (int a = 0; a < n; ++a)
        for (int d = 0; d < 3; ++d)
            xyz[a * 3 + d] = X[(int64_t)conn_e[a] * 3 + d] + (u ? u[(int64_t)conn_e[a] * 3 + d] : 0.0);
}

/* Element stiffness K_e (3n x 3n, row-major) = sum_gp B^T D(T_gp) B |detJ| w
 * (element.rs:217-318). Coordinates are X (+u when u != NULL, NLGEOM). */
int or_element_stiffness(int npe, const int* conn_e, int mat, const double* X, const double* u,
                         const double* t_cur, const or_mats* m, double* Ke) {
    rule_t r;
    make_rule(npe, &r);
    int n = npe, nd = 3 * npe;
    double xyz[60], gl[60], B[6 * 60], BtD[60 * 6], D[36], w;
    memset(Ke, 0, (size_t)nd * nd * sizeof(double));
    gather_xyz(n, conn_e, X, u, xyz);
    for (int g = 0; g < r.ngp; ++g) {
        int rc = gp_geometry(&r, g, xyz, gl, &w);
        if (rc) return rc;
        bmatrix(n, gl, B);
        double tc = 0.0;
        if (t_cur)
            for (int a = 0; a < n; ++a) tc += r.N[g][a] * t_cur[conn_e[a]];
        rc = mat_dmatrix(m, mat, tc, D);
        if (rc) return rc;
        for (int i = 0; i < nd; ++i)
            for (int k = 0; k < 6; ++k) {
                double s = 0.0;
                for (int l = 0; l < 6; ++l) s += B[l * nd + i] * D[l * 6 + k];
                BtD[i * 6 + k] = s;
            }
        for (int i = 0; i < nd; ++i)
            for (int j = 0; j < nd; ++j) {
                double s = 0.0;
                for (int k = 0; k < 6; ++k) s += BtD[i * 6 + k] * B[k * nd + j];
                Ke[i * nd + j] += s * w;
            }
    }
    return OR_OK;
}

/* Serial stiffness assembly into triplets (assembler.rs:37-151). Output
 * arrays must hold nelem*(3*npe)^2 entries; *ntrip is advanced, *maxdiag is
 * max'ed, so several element groups can append into the same arrays. */
int or_assemble(int npe, int nelem, const int* conn, const int* mats, const double* X, const double* u,
                const double* t_cur, const or_mats* m, int64_t* rows, int64_t* cols, double* vals,
                int64_t* ntrip, double* maxdiag, int* bad_elem) {
    int nd = 3 * npe;
    double* Ke = (double*)malloc((size_t)nd * nd * sizeof(double));
    int64_t t = *ntrip;
    double md = *maxdiag;
    for (int e = 0; e < nelem; ++e) {
        const int* ce = conn + (int64_t)e * npe;
        if (mats[e] < 0) { *bad_elem = e; free(Ke); return OR_NO_MATERIAL; }
        int rc = or_element_stiffness(npe, ce, mats[e], X, u, t_cur, m, Ke);
        if (rc) { *bad_elem = e; free(Ke); return rc; }
        for (int i = 0; i < npe; ++i)
            for (int j = 0; j < npe; ++j)
                for (int di = 0; di < 3; ++di)
                    for (int dj = 0; dj < 3; ++dj) {
                        double v = Ke[(i * 3 + di) * nd + j * 3 + dj];
                        if (fabs(v) > 1e-12) {
                            int64_t row = (int64_t)ce[i] * 3 + di, col = (int64_t)ce[j] * 3 + dj;
                            rows[t] = row; cols[t] = col; vals[t] = v; ++t;
                            if (row == col && fabs(v) > md) md = fabs(v);
                        }
                    }
    }
    free(Ke);
    *ntrip = t;
    *maxdiag = md;
    return OR_OK;
}

/* Internal force (element.rs:352-447 + assembler.rs:157-241): coordinates X
 * (+uconf when given), strain = B u_e - delta_th, stress = D(Tc) strain,
 * f += B^T stress |detJ| w, scattered with += into f (3N, not cleared). */
int or_internal_force(int npe, int nelem, const int* conn, const int* mats, const double* X, const double* u,
                      const double* uconf, const double* t_init, const double* t_cur, const or_mats* m,
                      double* f, int* bad_elem) {
    rule_t r;
    make_rule(npe, &r);
    int n = npe, nd = 3 * npe;
    double xyz[60], gl[60], B[6 * 60], D[36], ue[60], fe[60], w;
    for (int e = 0; e < nelem; ++e) {
        const int* ce = conn + (int64_t)e * npe;
        int k = mats[e];
        if (k < 0) { *bad_elem = e; return OR_NO_MATERIAL; }
        gather_xyz(n, ce, X, uconf, xyz);
        for (int a = 0; a < n; ++a)
            for (int d = 0; d < 3; ++d) ue[a * 3 + d] = u[(int64_t)ce[a] * 3 + d];
        memset(fe, 0, sizeof(fe));
        for (int g = 0; g < r.ngp; ++g) {
            int rc = gp_geometry(&r, g, xyz, gl, &w);
            if (rc) { *bad_elem = e; return rc; }
            bmatrix(n, gl, B);
            double tc = 0.0, ti = 0.0;
            for (int a = 0; a < n; ++a) {
                tc += r.N[g][a] * t_cur[ce[a]];
                ti += r.N[g][a] * t_init[ce[a]];
            }
            rc = mat_dmatrix(m, k, tc, D);
            if (rc) { *bad_elem = e; return rc; }
            double eps[6], sig[6];
            for (int i = 0; i < 6; ++i) {
                double s = 0.0;
                for (int j = 0; j < nd; ++j) s += B[i * nd + j] * ue[j];
                eps[i] = s;
            }
            if (mat_has_alpha(m, k)) {
                double dth = thermal_delta(m, k, tc, ti);
                eps[0] -= dth; eps[1] -= dth; eps[2] -= dth;
            }
            for (int i = 0; i < 6; ++i) {
                double s = 0.0;
                for (int j = 0; j < 6; ++j) s += D[i * 6 + j] * eps[j];
                sig[i] = s;
            }
            for (int j = 0; j < nd; ++j) {
                double s = 0.0;
                for (int i = 0; i < 6; ++i) s += B[i * nd + j] * sig[i];
                fe[j] += s * w;
            }
        }
        for (int a = 0; a < n; ++a)
            for (int d = 0; d < 3; ++d) f[(int64_t)ce[a] * 3 + d] += fe[a * 3 + d];
    }
    return OR_OK;
}

/* Thermal force (element.rs:453-520 + assembler.rs:247-299). */
int or_thermal_force(int npe, int nelem, const int* conn, const int* mats, const double* X, const double* t_init,
                     const double* t_cur, const or_mats* m, double* f, int* bad_elem) {
    rule_t r;
    make_rule(npe, &r);
    int n = npe, nd = 3 * npe;
    double xyz[60], gl[60], B[6 * 60], D[36], fe[60], w;
    for (int e = 0; e < nelem; ++e) {
        const int* ce = conn + (int64_t)e * npe;
        int k = mats[e];
        if (k < 0) { *bad_elem = e; return OR_NO_MATERIAL; }
        gather_xyz(n, ce, X, NULL, xyz);
        memset(fe, 0, sizeof(fe));
        for (int g = 0; g < r.ngp; ++g) {
            double tc = 0.0, ti = 0.0;
            for (int a = 0; a < n; ++a) {
                tc += r.N[g][a] * t_cur[ce[a]];
                ti += r.N[g][a] * t_init[ce[a]];
            }
            if (!mat_has_alpha(m, k)) continue;
            double dth = thermal_delta(m, k, tc, ti);
            int rc = mat_dmatrix(m, k, tc, D);
            if (rc) { *bad_elem = e; return rc; }
            rc = gp_geometry(&r, g, xyz, gl, &w);
            if (rc) { *bad_elem = e; return rc; }
            bmatrix(n, gl, B);
            double sig[6];
            for (int i = 0; i < 6; ++i) sig[i] = (D[i * 6 + 0] + D[i * 6 + 1] + D[i * 6 + 2]) * dth;
            for (int j = 0; j < nd; ++j) {
                double s = 0.0;
                for (int i = 0; i < 6; ++i) s += B[i * nd + j] * sig[i];
                fe[j] += s * w;
            }
        }
        for (int a = 0; a < n; ++a)
            for (int d = 0; d < 3; ++d) f[(int64_t)ce[a] * 3 + d] += fe[a * 3 + d];
    }
    return OR_OK;
}
