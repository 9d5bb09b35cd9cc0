// Host-side model: the Project / Mesh / Material / Step data of FerriX
// (src/solver/project.rs:32-58, src/solver/mesh_lib/mesh.rs:11-27,
// src/solver/material.rs:14-277, src/solver/step/static_step.rs:25-36)
// and its dense, index-based form that is uploaded to the GPU.
#pragma once

#include <array>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <string_view>
#include <unordered_map>
#include <utility>
#include <vector>

namespace fx {

// Allocator whose resize() leaves new elements default-initialised (not
// zeroed): bulk arrays are sized by one thread and filled by several, each
// touching its own pages first.
template <class T>
struct RawAlloc : std::allocator<T> {
    using value_type = T;
    template <class U>
    struct rebind {
        using other = RawAlloc<U>;
    };
    RawAlloc() = default;
    template <class U>
    RawAlloc(const RawAlloc<U>&) noexcept {}
    template <class U>
    void construct(U* p) noexcept {
        ::new ((void*)p) U;
    }
    template <class U, class... A>
    void construct(U* p, A&&... a) {
        ::new ((void*)p) U(std::forward<A>(a)...);
    }
};
template <class T>
using RawVec = std::vector<T, RawAlloc<T>>;

// TemperatureDependentLUT (material.rs:14-69): sorted (T, v) pairs.
struct Lut {
    std::vector<std::pair<double, double>> data;
    void push(double t, double v);  // append + stable sort by T
    double interpolate(double temp) const;
};

struct Material {
    std::string name;
    bool has_density = false, has_e = false, has_nu = false, has_alpha = false;
    Lut density, e, nu, alpha;
    double tref = 0.0;
    int64_t depvars = 0;
};

// Amplitude (amplitude.rs:9-57): tabular when has_data, else the step ramp.
struct Amplitude {
    bool total_time = false;
    double shift_x = 0.0, shift_y = 0.0;
    bool has_data = false;
    std::vector<double> t, v;
};
double amplitude_interpolate(double t, const std::vector<double>& ts, const std::vector<double>& vs,
                             double shift_x, double shift_y);

struct SolverTime {  // time.rs:8-63
    double global = 0.0, local = 0.0, local_max = 1.0;
    void new_step(double max_time) { local = 0.0; local_max = max_time; }
    void new_increment(double dt) { global += dt; local += dt; }
};

// Load / BoundaryCondition (boundary_conds.rs:9-102).
struct Record {
    int64_t node_id;
    int dof;  // 0..2
    double value;
    std::shared_ptr<const Amplitude> amp;  // null = default ramp
    int64_t origin_step;
    double eval(const SolverTime& t, int64_t current_step) const;
};

struct IncrementData {  // increment.rs:8-31
    double initial = 1.0, period = 1.0, min_inc = 1e-5, max_inc = 1.0;
    int64_t max_increments = 10000;
};

enum class SolverType { Default = 0, Direct = 1, Iterative = 2 };

struct StaticStep {
    SolverType solver = SolverType::Default;
    IncrementData inc;
    std::vector<Record> loads, bcs;
    bool nlgeom = false;
};

// Id -> position in an ascending list of unique ids: arithmetic when the ids
// are consecutive, a direct table when they are dense enough, a hash map
// otherwise. -1 when absent.
struct IdIndex {
    int64_t base = 0, count = 0;
    int mode = 0;  // 0 consecutive, 1 table, 2 map
    std::vector<int32_t> table;
    std::unordered_map<int64_t, int64_t> map;
    void build(const std::vector<int64_t>& sorted_ids);
    int64_t find(int64_t id) const {
        if (mode == 0) return id >= base && id - base < count ? id - base : -1;
        if (mode == 1) return id >= base && id - base < (int64_t)table.size() ? table[(size_t)(id - base)] : -1;
        auto it = map.find(id);
        return it == map.end() ? -1 : it->second;
    }
};

struct Project {
    // *NODE / *ELEMENT lines in deck order. A line whose id was seen before
    // replaces the earlier definition (the reference inserts into maps keyed by
    // id); resolve_mesh() applies that and sorts by id.
    RawVec<int64_t> node_line_ids;
    RawVec<std::array<double, 3>> node_line_xyz;
    RawVec<int64_t> elem_line_ids;
    RawVec<uint8_t> elem_line_npe;  // 4 (C3D4) or 20 (C3D20)
    RawVec<int64_t> elem_line_off;  // first node of the line in elem_line_conn
    RawVec<int64_t> elem_line_conn;
    // *SOLID_SECTION assignments (element id, material index) in deck order; the last one wins.
    std::vector<std::pair<int64_t, int>> elem_material_lines;
    std::unordered_map<std::string, std::vector<int64_t>> node_sets, element_sets;
    std::vector<Material> materials;
    std::vector<StaticStep> steps;
    std::vector<Record> initial_loads, initial_bcs;
    std::unordered_map<int64_t, double> initial_temperatures;
    double default_initial_temperature = 0.0;
    std::vector<std::string> nodal_output, element_output;
    std::unordered_map<std::string, std::shared_ptr<const Amplitude>> amplitudes;
    // Resolved mesh (Mesh::build_node_mappings, mesh.rs:35-50): node index =
    // rank of the node id; elements in ascending id with their defining line.
    std::vector<int64_t> index_to_node_id;
    RawVec<std::array<double, 3>> node_xyz;
    std::vector<int64_t> elem_ids, elem_line;
    IdIndex node_index;
    int64_t index_of(int64_t id) const { return node_index.find(id); }
    int64_t n_nodes() const { return (int64_t)index_to_node_id.size(); }
    int64_t n_elements() const { return (int64_t)elem_ids.size(); }
    void resolve_mesh();
};

// Preprocess + parse (parser.rs:111-147, 903-942). Throws fx::Error.
Project parse_inp(std::string_view text);

// Dense form: node index = rank of node id; one group per element type.
struct ElemGroup {
    int npe = 0;
    std::vector<int64_t> elem_ids;   // ascending
    std::vector<int32_t> conn;       // nelem * npe node indices
    std::vector<int32_t> mat;        // material index per element (-1 = none)
    int64_t size() const { return (int64_t)elem_ids.size(); }
};

struct MatTableHost {
    // per material: [off, len] for E, nu, alpha into t/v pools; tref
    std::vector<int32_t> e_off, e_len, nu_off, nu_len, a_off, a_len;
    std::vector<double> tref, t, v;
};

struct DenseModel {
    int64_t n_nodes = 0;
    std::vector<double> xyz;        // 3N
    ElemGroup g4, g20;
    MatTableHost mats;
    bool any_expansion = false;
    double volume = 0.0;              // mesh volume (tets exact, bricks from their corner hexahedron)
    std::string missing_node_error;  // NodeNotFound deferred to the first element loop
    int64_t missing_node_id = -1;
};

// Builds the dense form. Elements that reference unknown nodes are recorded
// (the reference reports NodeNotFound from the first element loop).
DenseModel build_dense(const Project& p);

}  // namespace fx
