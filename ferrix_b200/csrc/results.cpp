// Result fields after a solve: nodal-averaged stress / strain on the GPU
// (StaticStep::calculate_stress_strain, src/solver/step/static_step.rs:271-379)
// and the legacy-VTK writer of one increment on the host
// (VtkWriter::write_increment, src/solver/io/vtk.rs:72-319).
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <string>
#include <vector>

#include "engine.hpp"

using namespace fx;

namespace {

// S, E: 6 Voigt components per node (xx, yy, zz, xy, yz, zx), node-index order.
void nodal_stress_strain(fx_model* m, std::vector<double>& S, std::vector<double>& E) {
    if (!m->state_ready) fail(FX_INVALID_ARGUMENT, "fx_state_initialize was not called");
    ensure_structure(m);
    ModelDev& d = m->dev;
    cudaStream_t s = m->ctx->stream;
    const int64_t n = m->dense.n_nodes;
    const int64_t slots = (int64_t)m->dense.g4.size() * 4 + (int64_t)m->dense.g20.size() * 20;
    DBuf<double> buf, dS, dE;
    buf.alloc((size_t)std::max<int64_t>(1, slots) * 12, s);
    dS.alloc((size_t)std::max<int64_t>(1, n) * 6, s);
    dE.alloc((size_t)std::max<int64_t>(1, n) * 6, s);
    d.err.zero(s);
    launch_nodal_stress(d.g4(), d.g20(), d.xyz.ptr, d.u.ptr, d.tinit.ptr, d.tcur.ptr, d.mats.view(),
                        m->ctx->tables.view(), (int)n, d.S.node_ptr.ptr, d.S.node_slots.ptr, buf.ptr, dS.ptr, dE.ptr,
                        d.err.ptr, s);
    check_device_errors(m, "stress recovery");
    S.resize(6 * (size_t)n);
    E.resize(6 * (size_t)n);
    dS.download(S.data(), S.size(), s);
    dE.download(E.data(), E.size(), s);
    stream_wait(s, "stress download");
}

// Eigenvalues of the symmetric 3x3 matrix [[a, d, f], [d, b, e], [f, e, c]] by the
// trigonometric solution of the characteristic cubic (O. K. Smith, Comm. ACM 4(4), 1961).
void sym3_eigenvalues(double a, double b, double c, double d, double e, double f, double ev[3]) {
    const double p1 = d * d + e * e + f * f;
    if (p1 == 0.0) {
        ev[0] = a;
        ev[1] = b;
        ev[2] = c;
        return;
    }
    const double q = (a + b + c) / 3.0;
    const double p2 = (a - q) * (a - q) + (b - q) * (b - q) + (c - q) * (c - q) + 2.0 * p1;
    const double p = std::sqrt(p2 / 6.0);
    // B = (A - qI) / p; r = det(B) / 2
    const double b11 = (a - q) / p, b22 = (b - q) / p, b33 = (c - q) / p;
    const double b12 = d / p, b23 = e / p, b13 = f / p;
    const double detB = b11 * (b22 * b33 - b23 * b23) - b12 * (b12 * b33 - b23 * b13) + b13 * (b12 * b23 - b22 * b13);
    double r = detB / 2.0;
    r = r < -1.0 ? -1.0 : (r > 1.0 ? 1.0 : r);
    const double phi = std::acos(r) / 3.0;
    const double two_pi_3 = 2.0943951023931954923;  // 2 pi / 3
    ev[0] = q + 2.0 * p * std::cos(phi);
    ev[2] = q + 2.0 * p * std::cos(phi + two_pi_3);
    ev[1] = 3.0 * q - ev[0] - ev[2];
}

void put(std::string& out, double v) {
    char buf[32];
    auto r = std::to_chars(buf, buf + sizeof(buf), v);  // shortest representation that reads back exactly
    out.append(buf, r.ptr);
}

void put(std::string& out, int64_t v) {
    char buf[24];
    auto r = std::to_chars(buf, buf + sizeof(buf), v);
    out.append(buf, r.ptr);
}

}  // namespace

extern "C" {

int fx_nodal_stress_strain(fx_model* m, double* S, double* E) {
    if (!m || !m->ctx || (!S && !E)) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        int64_t* saved = g_launch_counter;
        g_launch_counter = &m->ctx->launches;
        struct R {
            int64_t* v;
            ~R() { g_launch_counter = v; }
        } r{saved};
        std::vector<double> hs, he;
        nodal_stress_strain(m, hs, he);
        if (S) std::memcpy(S, hs.data(), hs.size() * sizeof(double));
        if (E) std::memcpy(E, he.data(), he.size() * sizeof(double));
        return FX_OK;
    });
}

int fx_write_vtk(fx_model* m, const char* path) {
    if (!m || !m->ctx || !path) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        int64_t* saved = g_launch_counter;
        g_launch_counter = &m->ctx->launches;
        struct R {
            int64_t* v;
            ~R() { g_launch_counter = v; }
        } r{saved};
        std::vector<double> S, E;
        nodal_stress_strain(m, S, E);
        const DenseModel& D = m->dense;
        const int64_t n = D.n_nodes;
        std::vector<double> u(3 * (size_t)n), tc((size_t)n);
        m->dev.u.download(u.data(), u.size(), m->ctx->stream);
        m->dev.tcur.download(tc.data(), tc.size(), m->ctx->stream);
        stream_wait(m->ctx->stream, "vtk download");
        std::vector<uint8_t> has_stress((size_t)n, 0);  // nodes of no element have no S / E entry (written as 0)
        for (const ElemGroup* g : {&D.g4, &D.g20})
            for (int32_t v : g->conn) has_stress[(size_t)v] = 1;
        std::string out;
        out.reserve((size_t)n * 200 + (size_t)(D.g4.size() * 24 + D.g20.size() * 140));
        out += "# vtk DataFile Version 3.0\nCCX-RS Analysis Results\nASCII\nDATASET UNSTRUCTURED_GRID\n";
        out += "POINTS ";
        put(out, n);
        out += " float\n";
        for (int64_t i = 0; i < n; ++i) {
            for (int c = 0; c < 3; ++c) {
                if (c) out += ' ';
                put(out, D.xyz[3 * (size_t)i + c]);
            }
            out += '\n';
        }
        const int64_t ncell = D.g4.size() + D.g20.size();
        out += "CELLS ";
        put(out, ncell);
        out += ' ';
        put(out, D.g4.size() * 5 + D.g20.size() * 21);
        out += '\n';
        for (const ElemGroup* g : {&D.g4, &D.g20})
            for (int64_t e = 0; e < g->size(); ++e) {
                put(out, (int64_t)g->npe);
                for (int a = 0; a < g->npe; ++a) {
                    out += ' ';
                    put(out, (int64_t)g->conn[(size_t)e * g->npe + a]);
                }
                out += '\n';
            }
        out += "CELL_TYPES ";
        put(out, ncell);
        out += '\n';
        for (int64_t e = 0; e < D.g4.size(); ++e) out += "10\n";   // VTK_TETRA
        for (int64_t e = 0; e < D.g20.size(); ++e) out += "25\n";  // VTK_QUADRATIC_HEXAHEDRON
        out += "POINT_DATA ";
        put(out, n);
        out += "\nVECTORS U float\n";
        for (int64_t i = 0; i < n; ++i) {
            for (int c = 0; c < 3; ++c) {
                if (c) out += ' ';
                put(out, u[3 * (size_t)i + c]);
            }
            out += '\n';
        }
        for (int field = 0; field < 2; ++field) {
            const std::vector<double>& F = field == 0 ? S : E;
            out += field == 0 ? "SCALARS S float 6\nLOOKUP_TABLE default\n" : "SCALARS E float 6\nLOOKUP_TABLE default\n";
            for (int64_t i = 0; i < n; ++i) {
                for (int c = 0; c < 6; ++c) {
                    if (c) out += ' ';
                    put(out, F[6 * (size_t)i + c]);
                }
                out += '\n';
            }
        }
        out += "SCALARS NT float 1\nLOOKUP_TABLE default\n";
        for (int64_t i = 0; i < n; ++i) {
            put(out, tc[(size_t)i]);
            out += '\n';
        }
        out += "SCALARS MISES float 1\nLOOKUP_TABLE default\n";
        for (int64_t i = 0; i < n; ++i) {
            const double* s = &S[6 * (size_t)i];
            const double v = has_stress[(size_t)i]
                                 ? std::sqrt(((s[0] - s[1]) * (s[0] - s[1]) + (s[1] - s[2]) * (s[1] - s[2]) +
                                              (s[2] - s[0]) * (s[2] - s[0]) +
                                              6.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5])) /
                                             2.0)
                                 : 0.0;
            put(out, v);
            out += '\n';
        }
        out += "SCALARS TRESCA float 1\nLOOKUP_TABLE default\n";
        for (int64_t i = 0; i < n; ++i) {
            const double* s = &S[6 * (size_t)i];
            double v = 0.0;
            if (has_stress[(size_t)i]) {
                double ev[3];
                sym3_eigenvalues(s[0], s[1], s[2], s[3], s[4], s[5], ev);
                v = std::fmax(ev[0], std::fmax(ev[1], ev[2])) - std::fmin(ev[0], std::fmin(ev[1], ev[2]));
            }
            put(out, v);
            out += '\n';
        }
        FILE* f = std::fopen(path, "wb");
        if (!f) fail(FX_GENERIC_IO, std::string("cannot open ") + path);
        const size_t w = std::fwrite(out.data(), 1, out.size(), f);
        const int c = std::fclose(f);
        if (w != out.size() || c != 0) fail(FX_GENERIC_IO, std::string("write failed: ") + path);
        return FX_OK;
    });
}

// results.vtk.series (src/solver/io/vtk.rs:46-70, 305-333), byte for byte: the header of
// init, one entry per written increment, the footer of finish.
static int series_write(const char* dir, const char* mode, const std::string& text) {
    if (!dir) return FX_INVALID_ARGUMENT;
    return guarded(nullptr, [&] {
        const std::string path = std::string(dir) + "/results.vtk.series";
        FILE* f = std::fopen(path.c_str(), mode);
        if (!f) fail(FX_GENERIC_IO, "Generic IO error: cannot open " + path);
        const size_t w = std::fwrite(text.data(), 1, text.size(), f);
        const int c = std::fclose(f);
        if (w != text.size() || c != 0) fail(FX_GENERIC_IO, "Generic IO error: write failed: " + path);
        return FX_OK;
    });
}

int fx_vtk_series_init(const char* dir) {
    if (!dir) return FX_INVALID_ARGUMENT;
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) {
        fx::thread_error().set(FX_GENERIC_IO, std::string("Generic IO error: cannot create ") + dir);
        return FX_GENERIC_IO;
    }
    return series_write(dir, "wb", "{\n          \"file-series-version\" : \"1.0\",\n          \"files\" : [\n");
}

int fx_vtk_series_add(const char* dir, const char* name, double time) {
    if (!dir || !name) return FX_INVALID_ARGUMENT;
    // the reference's "{}" of an f64: the shortest decimal that reads back to the same
    // value, never in exponent form
    char buf[512];
    const auto r = std::to_chars(buf, buf + sizeof(buf), time, std::chars_format::fixed);
    const std::string t = r.ec == std::errc() ? std::string(buf, r.ptr) : std::to_string(time);
    return series_write(dir, "ab", std::string("{ \"name\" : \"") + name + "\", \"time\" : " + t + " },\n");
}

int fx_vtk_series_finish(const char* dir) { return series_write(dir, "ab", "  ]\n}\n"); }

}  // extern "C"
