// fx_model_from_arrays: the Project that Parser::parse builds
// (src/solver/parser.rs:111-482), filled from caller arrays instead of deck
// text. It writes the same fields the parser writes (node and element
// definitions in order, material tables, amplitudes, step records, initial
// temperatures) and then resolves the mesh the same way (Mesh::build_node_mappings,
// src/solver/mesh_lib/mesh.rs:35-50), so everything downstream of the parser
// sees the same model.
#include <cstring>
#include <memory>
#include <string>

#include "engine.hpp"

using namespace fx;

namespace {

void require(bool ok, const std::string& what) {
    if (!ok) fail(FX_INVALID_ARGUMENT, "fx_model_from_arrays: " + what);
}

// TemperatureDependentLUT::push per pair (material.rs:14-35): appended, kept sorted by T.
bool fill_lut(const fx_lut_desc& d, Lut& lut, const std::string& what) {
    require(d.n >= 0, what + ": negative pair count");
    if (d.n == 0) return false;
    require(d.temperature && d.value, what + ": pairs without arrays");
    for (int64_t k = 0; k < d.n; ++k) lut.push(d.temperature[k], d.value[k]);
    return true;
}

void fill_records(int64_t n, const fx_record_desc* in, const std::vector<std::shared_ptr<const Amplitude>>& amps,
                  std::vector<Record>& out, const std::string& what) {
    require(n >= 0 && (n == 0 || in), what + ": records without an array");
    out.reserve((size_t)n);
    for (int64_t k = 0; k < n; ++k) {
        const fx_record_desc& r = in[k];
        require(r.dof >= 0 && r.dof <= 2, what + ": dof outside 0..2");
        require(r.amplitude >= -1 && r.amplitude < (int32_t)amps.size(), what + ": amplitude index out of range");
        require(r.origin_step >= 0, what + ": negative origin step");
        out.push_back(Record{r.node_id, (int)r.dof, r.value, r.amplitude >= 0 ? amps[(size_t)r.amplitude] : nullptr,
                             r.origin_step});
    }
}

void add_elements(Project& p, int64_t n, const int64_t* ids, const int64_t* nodes, const int32_t* mat, int npe,
                  int n_materials, const char* type) {
    const std::string t(type);
    require(n >= 0 && (n == 0 || (ids && nodes)), t + " elements without arrays");
    p.elem_line_off.reserve(p.elem_line_off.size() + (size_t)n);
    p.elem_line_ids.reserve(p.elem_line_ids.size() + (size_t)n);
    p.elem_line_npe.reserve(p.elem_line_npe.size() + (size_t)n);
    p.elem_line_conn.reserve(p.elem_line_conn.size() + (size_t)n * npe);
    for (int64_t e = 0; e < n; ++e) {
        p.elem_line_off.push_back((int64_t)p.elem_line_conn.size());
        p.elem_line_ids.push_back(ids[e]);
        p.elem_line_npe.push_back((uint8_t)npe);
        for (int a = 0; a < npe; ++a) p.elem_line_conn.push_back(nodes[e * npe + a]);
        const int32_t m = mat ? mat[e] : -1;
        require(m >= -1 && m < n_materials, t + " material index out of range");
        if (m >= 0) p.elem_material_lines.emplace_back(ids[e], (int)m);
    }
}

Project project_from_desc(const fx_mesh_desc& d) {
    Project p;
    require(d.n_nodes >= 0 && (d.n_nodes == 0 || (d.node_ids && d.xyz)), "nodes without arrays");
    p.node_line_ids.resize((size_t)d.n_nodes);
    p.node_line_xyz.resize((size_t)d.n_nodes);
    for (int64_t i = 0; i < d.n_nodes; ++i) {
        require(d.node_ids[i] >= 0, "negative node id");
        p.node_line_ids[(size_t)i] = d.node_ids[i];
        p.node_line_xyz[(size_t)i] = {d.xyz[3 * i], d.xyz[3 * i + 1], d.xyz[3 * i + 2]};
    }
    require(d.n_materials >= 0 && (d.n_materials == 0 || d.materials), "materials without an array");
    for (int k = 0; k < d.n_materials; ++k) {
        const fx_material_desc& md = d.materials[k];
        Material m;
        m.name = md.name ? md.name : "";
        const std::string w = "material " + std::to_string(k);
        m.has_e = fill_lut(md.youngs_modulus, m.e, w + " Young's modulus");
        m.has_nu = fill_lut(md.poisson_ratio, m.nu, w + " Poisson's ratio");
        m.has_alpha = fill_lut(md.thermal_expansion, m.alpha, w + " expansion");
        m.tref = md.reference_temperature;
        p.materials.push_back(std::move(m));
    }
    add_elements(p, d.n_c3d4, d.c3d4_ids, d.c3d4_nodes, d.c3d4_material, 4, d.n_materials, "C3D4");
    add_elements(p, d.n_c3d20, d.c3d20_ids, d.c3d20_nodes, d.c3d20_material, 20, d.n_materials, "C3D20");
    for (int64_t id : p.elem_line_ids) require(id >= 0, "negative element id");
    require(d.n_amplitudes >= 0 && (d.n_amplitudes == 0 || d.amplitudes), "amplitudes without an array");
    std::vector<std::shared_ptr<const Amplitude>> amps;
    for (int k = 0; k < d.n_amplitudes; ++k) {
        const fx_amplitude_desc& ad = d.amplitudes[k];
        require(ad.n >= 1 && ad.time && ad.value, "amplitude " + std::to_string(k) + " without pairs");
        auto a = std::make_shared<Amplitude>();
        a->total_time = ad.total_time != 0;
        a->shift_x = ad.shift_x;
        a->shift_y = ad.shift_y;
        a->t.assign(ad.time, ad.time + ad.n);
        a->v.assign(ad.value, ad.value + ad.n);
        a->has_data = true;
        p.amplitudes["#" + std::to_string(k)] = a;
        amps.push_back(a);
    }
    require(d.n_steps >= 0 && (d.n_steps == 0 || d.steps), "steps without an array");
    for (int k = 0; k < d.n_steps; ++k) {
        const fx_step_desc& sd = d.steps[k];
        StaticStep st;
        require(sd.solver >= 0 && sd.solver <= 2, "step solver outside 0..2");
        st.solver = (SolverType)sd.solver;
        st.nlgeom = sd.nlgeom != 0;
        st.inc.initial = sd.increment[0];
        st.inc.period = sd.increment[1];
        st.inc.min_inc = sd.increment[2];
        st.inc.max_inc = sd.increment[3];
        st.inc.max_increments = sd.max_increments;
        const std::string w = "step " + std::to_string(k + 1);
        fill_records(sd.n_loads, sd.loads, amps, st.loads, w + " loads");
        fill_records(sd.n_bcs, sd.bcs, amps, st.bcs, w + " boundary conditions");
        p.steps.push_back(std::move(st));
    }
    p.default_initial_temperature = d.default_temperature;
    require(d.n_initial_temperatures >= 0 &&
                (d.n_initial_temperatures == 0 || (d.initial_temperature_ids && d.initial_temperatures)),
            "initial temperatures without arrays");
    for (int64_t k = 0; k < d.n_initial_temperatures; ++k)
        p.initial_temperatures[d.initial_temperature_ids[k]] = d.initial_temperatures[k];
    p.resolve_mesh();
    return p;
}

}  // namespace

extern "C" int fx_model_from_arrays(fx_ctx* ctx, const fx_mesh_desc* desc, fx_model** out) {
    if (!out || !desc) return FX_INVALID_ARGUMENT;
    *out = nullptr;
    return guarded(ctx, [&] {
        auto m = std::make_unique<fx_model>();
        m->ctx = ctx;
        m->project = project_from_desc(*desc);
        *out = m.release();
        return FX_OK;
    });
}
