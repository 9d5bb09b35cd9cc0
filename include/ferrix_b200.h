/*
 * ferrix_b200 — C ABI of the B200 (sm_100a) solver for FerriX's linear-static
 * and NLGEOM *STATIC path (C3D4 / C3D20 solids).
 *
 * Plain C types only: opaque handles, host pointers and sizes. The caller owns
 * every host buffer; the library owns all device memory behind the handles.
 * One context = one GPU + one CUDA stream; a context and its models must be
 * used from one thread at a time.
 *
 * Reference seams each entry point replaces (paths relative to the FerriX
 * crate root):
 *   fx_model_from_inp            Project::from_jobname / Parser::parse
 *                                (src/solver/project.rs:93-127, src/solver/parser.rs:111-147)
 *   fx_model_from_arrays         the Project that Parser::parse builds, from arrays
 *                                (src/solver/parser.rs:111-482, src/solver/mesh_lib/mesh.rs:35-50)
 *   fx_state_initialize          SolutionState::new + initialize (src/solver/state.rs:32-79)
 *                                and SolverTime::new (src/solver/time.rs:27-33)
 *   fx_step_solve                Step::solve -> StaticStep::solve
 *                                (src/solver/step/steps.rs:28-42, src/solver/step/static_step.rs:47-267)
 *   fx_assemble_csr              Assembler::assemble + TriMat::to_csr
 *                                (src/solver/assembler.rs:37-151, src/solver/step/static_step.rs:198)
 *   fx_internal_force            Assembler::assemble_internal_force (src/solver/assembler.rs:157-241)
 *   fx_thermal_force             Assembler::assemble_thermal_force (src/solver/assembler.rs:247-299)
 *   fx_solve_csr                 Solver::solve (src/solver/solvers/mod.rs:18-43), the seam behind
 *                                DirectSolver (direct.rs:19-55) and IterativeSolver (iterative.rs:26-136)
 *   fx_last_error_detail         the payload of the FerrixError variant (src/solver/error.rs:12-72)
 *   fx_batch_solve               no reference counterpart (one deck per process there): many
 *                                independent decks' first *STATIC step in one batched launch sequence
 *   fx_server_*                  no reference counterpart: continuous-batching request loop
 */
#ifndef FERRIX_B200_H
#define FERRIX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: the FerrixError variants (src/solver/error.rs:12-72) plus
 * device-side conditions. 0 is success. */
typedef enum {
    FX_OK = 0,
    FX_IO = 1,
    FX_GENERIC_IO = 2,
    FX_PARSE = 3,
    FX_UNSUPPORTED_KEYWORD = 4,
    FX_UNKNOWN_SOLVER = 5,
    FX_NODE_NOT_FOUND = 6,
    FX_ELEMENT_NOT_FOUND = 7,
    FX_MATERIAL_NOT_FOUND = 8,
    FX_ELSET_NOT_FOUND = 9,
    FX_NSET_NOT_FOUND = 10,
    FX_NUMERICAL = 11,        /* singular Jacobian, PCG breakdown, indefinite system */
    FX_CONVERGENCE = 12,      /* increment / Newton / PCG iteration limits */
    FX_INVALID_MODEL = 13,
    FX_GENERIC = 14,
    FX_CANCELLED = 15,
    FX_TIMEOUT = 16,
    FX_CUDA = 17,
    FX_INVALID_ARGUMENT = 18
} fx_status;

typedef struct fx_ctx fx_ctx;
typedef struct fx_model fx_model;
typedef struct fx_server fx_server;

/* Arithmetic of the PCG that stands in for the reference's FP64 Cholesky. */
typedef enum {
    FX_PREC_MIXED = 0, /* block-Jacobi: FP32 BSR3 SpMV and preconditioner, FP64 residual replacement and
                          accumulation; multigrid: FP64 CG, FP32 matrix values in the fine-level smoother */
    FX_PREC_FP64 = 1,  /* FP64 throughout */
    FX_PREC_FP64_CSR = 2 /* plain FP64 PCG: scalar CSR SpMV + Jacobi (the reference IterativeSolver's algorithm) */
} fx_precision;

typedef struct {
    int precision;          /* fx_precision */
    double rtol;            /* stop when ||b - A x||_M / ||b||_M <= rtol (FP64 true residual, M = block-Jacobi) */
    int max_iter;           /* PCG iteration cap per linear solve (FX_CONVERGENCE beyond) */
    int poll_interval;      /* PCG iterations per CUDA-graph replay between host checks (even) */
    double reliable_delta;  /* mixed: FP64 residual replacement once the residual fell by this factor */
    int use_graphs;         /* capture the PCG iteration block in a CUDA graph */
    int verbose;            /* print the reference's per-iteration |R| lines to stdout */
    int reference_iterative; /* SOLVER=ITERATIVE steps: reference semantics (Jacobi PCG, absolute
                                sqrt(r.z) < 1e-8, at most 1000 iterations; iterative.rs:26-136) */
    int preconditioner;     /* fx_preconditioner */
    int amg_aggregate_nodes; /* FX_PRECOND_AMG: mean nodes per fine aggregate (cell size); 0 = 40 */
    int amg_smoother_degree; /* FX_PRECOND_AMG: Chebyshev steps per pre/post smoothing, 1..8; 0 = 2 */
    int amg_cycle;           /* FX_PRECOND_AMG: 0 = V-cycle, 1 = K-cycle at the first coarse level (two
                                flexible-CG steps per coarse correction; the outer CG is then flexible) */
    int amg_smoother;        /* FX_PRECOND_AMG: 0 = Chebyshev of the first kind on [lmax/ratio, lmax],
                                1 = Chebyshev of the fourth kind (Lottes 2023) */
    double amg_overcorrect;  /* FX_PRECOND_AMG: coarse corrections are scaled by this factor, in (0, 2);
                                0 = 1.7 */
    double amg_cheb_ratio;   /* FX_PRECOND_AMG: lmax / lmin of the first-kind Chebyshev interval; 0 = 12 */
    int amg_persistent_max_dof; /* FX_PRECOND_AMG, V-cycle: systems of at most this many DOF run their
                                   whole CG in one persistent launch, one thread-block cluster per system
                                   (all such systems of a round in the same launch); 0 = default (2,000);
                                   < 0 = never (one launch per CG step and phase) */
    int amg_fused_coarse;       /* FX_PRECOND_AMG, V-cycle, systems on the multi-launch path: 1 = the coarse
                                   part of each V-cycle (restriction, coarse levels, dense coarsest solve,
                                   prolongation) as one cooperative launch over all SMs; 0 = one launch
                                   per step (default; measured faster on B200) */
    int amg_fp16_smoother;      /* FX_PRECOND_AMG with FX_PREC_MIXED, systems on the multi-launch path: the
                                   fine-level smoother reads FP16 values of the diagonally scaled matrix
                                   D^-1/2 K D^-1/2 (entries within [-1, 1]); 0 = default (FP16), 1 = FP16,
                                   -1 = FP32 values of K */
} fx_solve_opts;

/* Preconditioner of the BSR3 PCG. */
typedef enum {
    FX_PRECOND_BLOCK_JACOBI = 0, /* 3x3 block-Jacobi */
    FX_PRECOND_AMG = 1           /* aggregation multigrid V-cycle (rigid-body near-null-space), FP64 CG;
                                    with FX_PREC_MIXED the fine-level smoother reads FP32 matrix values */
} fx_preconditioner;

typedef struct {
    int increments;            /* increments attempted (converged or cut back) */
    int newton_iterations;
    int linear_solves;
    long long pcg_iterations;
    int reliable_updates;
    double last_rel_residual;  /* |R|/|F_ext| of the last converged Newton iteration */
    double last_linear_relres; /* ||b - A x||_M / ||b||_M of the last linear solve */
    double t_symbolic_ms, t_assembly_ms, t_forces_ms, t_pcg_ms, t_total_ms;  /* device event times */
    int64_t bsr_blocks;        /* 3x3 blocks of the assembled stiffness */
    int fp64_fallbacks;        /* mixed solves that stalled and were finished in FP64 */
    int amg_levels;            /* multigrid levels of the last AMG-preconditioned solve */
    double amg_setup_ms;       /* multigrid setup time, summed over the step */
} fx_step_stats;

/* Defaults: FX_PREC_MIXED, FX_PRECOND_AMG, rtol 1e-8, max_iter 50000, poll 32,
 * reliable_delta 1e-2, graphs on, 40 nodes per aggregate, Chebyshev degree 2 on
 * [lmax/12, lmax], coarse corrections scaled by 1.7.
 * fx_solve_csr has no node coordinates and always uses block-Jacobi. */
void fx_default_solve_opts(fx_solve_opts* opts);

/* ---- context ---------------------------------------------------------- */
int fx_ctx_create(int device, fx_ctx** out);
void fx_ctx_destroy(fx_ctx* ctx);
const char* fx_ctx_last_error(const fx_ctx* ctx);

/* The last failure with the payload of its FerrixError variant (src/solver/error.rs:12-72):
 *   FX_PARSE                line = deck line (0 for element-line errors, as the reference
 *                           reports them), text = the message
 *   FX_UNSUPPORTED_KEYWORD  line = deck line, text = the keyword
 *   FX_NODE_NOT_FOUND       id = the node id;   FX_ELEMENT_NOT_FOUND: id = the element id
 *   FX_UNKNOWN_SOLVER, FX_MATERIAL_NOT_FOUND, FX_ELSET_NOT_FOUND, FX_NSET_NOT_FOUND
 *                           text = the name
 *   FX_NUMERICAL, FX_CONVERGENCE, FX_INVALID_MODEL, FX_GENERIC, FX_GENERIC_IO, FX_IO
 *                           text = the variant's message (the path for FX_IO)
 * line / id are -1 where the variant has none; message = the full display text
 * (as fx_ctx_last_error). With ctx NULL: the calling thread's last failure, which
 * also covers calls made without a context (fx_model_from_inp with ctx NULL).
 * status is FX_OK when nothing has failed yet. Texts are truncated to fit. */
typedef struct {
    int status;
    int64_t line;
    int64_t id;
    char text[512];
    char message[768];
} fx_error_detail;
int fx_last_error_detail(const fx_ctx* ctx, fx_error_detail* out);
/* Number of kernel launches issued by this context so far (all entry points). */
int64_t fx_ctx_kernel_launches(const fx_ctx* ctx);
/* The context's cudaStream_t (as void*), for callers that time or order work on it. */
void* fx_ctx_stream(const fx_ctx* ctx);
/* Kernels of the library that fx_ctx_create found loaded on the context's device
 * (all of them are loaded once per device and process, so that no kernel's first
 * launch waits for other streams' work); -1 when the driver offers no way to
 * load them ahead (they then load at first launch). */
int fx_ctx_preloaded_kernels(const fx_ctx* ctx);

/* ---- model (Project) -------------------------------------------------- */
/* Preprocess + parse `.inp` text with the reference parser's semantics.
 * ctx may be NULL: the model can then be inspected but not solved. */
int fx_model_from_inp(fx_ctx* ctx, const char* text, size_t len, fx_model** out);
void fx_model_destroy(fx_model* model);

/* ---- model from arrays (binary mesh path) ---------------------------------
 * The model that Project::from_jobname / Parser::parse builds
 * (src/solver/parser.rs:111-482, src/solver/mesh_lib/mesh.rs:35-50,
 * src/solver/material.rs:14-69, src/solver/step/boundary_conds.rs:9-102,
 * src/solver/step/amplitude.rs:9-57), handed over as arrays instead of .inp
 * text, for callers that already hold the mesh in memory (a service receiving
 * binary meshes, a mesh generator): no text is formatted or parsed. Every field
 * means what it means after a deck is parsed, so the model equals the one
 * fx_model_from_inp builds from a deck that defines the same data (same node
 * index order, element groups, material tables and step records; the same
 * displacements, bit for bit). All arrays are the caller's and are copied. */
typedef struct {
    int64_t n;                  /* (temperature, value) pairs, 0 = property not defined */
    const double* temperature;  /* n; pairs are inserted in this order and kept sorted by temperature
                                   (stable), as the reference's TemperatureDependentLUT::push */
    const double* value;        /* n */
} fx_lut_desc;

typedef struct {
    const char* name;                 /* NUL-terminated; may be NULL */
    fx_lut_desc youngs_modulus;       /* *ELASTIC column 1 over column 3 */
    fx_lut_desc poisson_ratio;        /* *ELASTIC column 2 over column 3 */
    fx_lut_desc thermal_expansion;    /* *EXPANSION; n = 0 when the material has none */
    double reference_temperature;     /* *EXPANSION, ZERO= */
} fx_material_desc;

typedef struct {
    int64_t n;             /* (time, value) pairs of a tabular *AMPLITUDE, >= 1 */
    const double* time;    /* n, ascending */
    const double* value;   /* n */
    int total_time;        /* TIME=TOTAL TIME: evaluated at the total time, else at the step time */
    double shift_x, shift_y;
} fx_amplitude_desc;

typedef struct {
    int64_t node_id;
    int32_t dof;          /* 0..2 (DOFs 4-6 of a deck are dropped by the parser) */
    int32_t amplitude;    /* index into fx_mesh_desc.amplitudes; -1 = the step ramp */
    double value;
    int64_t origin_step;  /* the step the record was defined in (1-based); 0 = before the first *STEP */
} fx_record_desc;

typedef struct {
    int nlgeom;
    int solver;              /* 0 default, 1 direct, 2 iterative (*STATIC, SOLVER=) */
    double increment[4];     /* initial, period, min, max increment (the *STATIC data line) */
    int64_t max_increments;  /* *STEP, INC= (10000 when absent) */
    int64_t n_loads;         /* the step's *CLOAD records in effect (carried over ones first), in order */
    const fx_record_desc* loads;
    int64_t n_bcs;           /* the step's *BOUNDARY records in effect, in order */
    const fx_record_desc* bcs;
} fx_step_desc;

typedef struct {
    int64_t n_nodes;
    const int64_t* node_ids;      /* n_nodes ids, any order; a repeated id: the later entry wins */
    const double* xyz;            /* 3 * n_nodes */
    int64_t n_c3d4;
    const int64_t* c3d4_ids;      /* element ids, unique over both types */
    const int64_t* c3d4_nodes;    /* 4 node ids per element */
    const int32_t* c3d4_material; /* material index per element, -1 = no *SOLID SECTION (NULL: all -1) */
    int64_t n_c3d20;
    const int64_t* c3d20_ids;
    const int64_t* c3d20_nodes;   /* 20 node ids per element, Abaqus order */
    const int32_t* c3d20_material;
    int n_materials;
    const fx_material_desc* materials;
    int n_amplitudes;
    const fx_amplitude_desc* amplitudes;
    int n_steps;
    const fx_step_desc* steps;
    double default_temperature;   /* Project.default_initial_temperature */
    int64_t n_initial_temperatures; /* *INITIAL CONDITIONS, TYPE=TEMPERATURE */
    const int64_t* initial_temperature_ids;
    const double* initial_temperatures;
} fx_mesh_desc;

/* Builds a model from `desc` (ctx as in fx_model_from_inp; NULL = host only, for
 * fx_server_submit). Element nodes that are not in the mesh are reported as
 * FX_NODE_NOT_FOUND by the first solve, as for a deck. FX_INVALID_ARGUMENT for
 * inconsistent descriptions (missing arrays, dof outside 0..2, an index outside
 * its table, a table without pairs where one is required). */
int fx_model_from_arrays(fx_ctx* ctx, const fx_mesh_desc* desc, fx_model** out);
/* Counts: nodes, elements (all types), steps, materials. */
int fx_model_sizes(const fx_model* model, int64_t* n_nodes, int64_t* n_elements, int* n_steps, int* n_materials);
/* Mesh::index_to_node_id: ids[i] = node id of matrix index i (ascending ids). */
int fx_model_node_ids(const fx_model* model, int64_t* ids);
/* Mesh::get_index_for_node_id: -1 when absent. */
int64_t fx_model_node_index(const fx_model* model, int64_t node_id);
/* Project.default_initial_temperature (applied by fx_state_initialize). */
int fx_model_set_default_temperature(fx_model* model, double temperature);
/* Step description: nlgeom flag, solver (0 default, 1 direct, 2 iterative),
 * increment data (initial, period, min, max), counts of loads and BCs. */
int fx_model_step_info(const fx_model* model, int step_index, int* nlgeom, int* solver, double incr[4],
                       int64_t* n_loads, int64_t* n_bcs);

/* Dense model arrays (node index = rank of node id; elements of each type in
 * ascending id order): xyz[3N], conn[n*npe] node indices, mat[n] material
 * index (-1 = none). Pass NULL for arrays not wanted; counts always written. */
int fx_model_export(fx_model* model, double* xyz, int64_t* n4, int32_t* conn4, int32_t* mat4, int64_t* n20,
                    int32_t* conn20, int32_t* mat20);
/* Loads (is_bc = 0) or BCs (is_bc = 1) of a step in record order: node id,
 * dof (0..2), value, origin step, amplitude flag (1 = tabular amplitude). */
int fx_model_step_records(const fx_model* model, int step_index, int is_bc, int64_t* node_ids, int32_t* dofs,
                          double* values, int64_t* origin, int32_t* tabular);

/* ---- solution state (SolutionState + SolverTime) --------------------- */
int fx_state_initialize(fx_model* model);
int fx_state_get_displacements(const fx_model* model, double* u /* 3N */);
int fx_state_set_displacements(fx_model* model, const double* u /* 3N */);
int fx_state_get_temperatures(const fx_model* model, double* t_init /* N */, double* t_cur /* N */);
/* SolutionState.initial_temperatures / .temperatures are public fields in the
 * reference (src/solver/state.rs:20-24); NULL leaves a vector unchanged. */
int fx_state_set_temperatures(fx_model* model, const double* t_init /* N */, const double* t_cur /* N */);

/* ---- the static step -------------------------------------------------- */
/* Step::solve for project.steps[step_index] with step_id = step_index + 1.
 * stats may be NULL; opts NULL = fx_default_solve_opts. */
int fx_step_solve(fx_model* model, int step_index, const fx_solve_opts* opts, fx_step_stats* stats);

/* Called on the host after every converged increment of fx_step_solve_cb, where the
 * reference hands the increment's result to ResultWriter::write_increment
 * (src/solver/step/static_step.rs:219-248, src/solver/io/writer.rs:7-34): step_id (1-based),
 * inc_id (the step's increment counter, failed attempts included, as the reference counts
 * them) and global_time (SolverTime::global_time, src/solver/time.rs:51-55). While it runs,
 * the model's displacements and temperatures are that increment's, so the callback may
 * read them (fx_state_get_displacements, fx_nodal_stress_strain, fx_write_vtk, ...); it must
 * not solve on the same model. A nonzero return ends the step with FX_GENERIC_IO. */
typedef int (*fx_increment_cb)(void* user, fx_model* model, int step_id, int inc_id, double global_time);
/* fx_step_solve with cb called after every converged increment (cb NULL: fx_step_solve). */
int fx_step_solve_cb(fx_model* model, int step_index, const fx_solve_opts* opts, fx_step_stats* stats,
                     fx_increment_cb cb, void* user);

/* ---- lower-level seams (parity tests, Rust shims) -------------------- */
/* Stiffness on X (+u when u != NULL) with the current temperatures, as the
 * expanded CSR of the 3x3 block structure (explicit zeros kept), FP64 values
 * of the `precision` assembly. Call with indptr/indices/data NULL to get *nnz. */
int fx_assemble_csr(fx_model* model, const double* u_or_null, int precision, int64_t* nnz, int64_t* indptr,
                    int64_t* indices, double* data, double* maxdiag);
/* f_int(u) on X (+uconf when != NULL), current temperatures; f is 3N. */
int fx_internal_force(fx_model* model, const double* u, const double* uconf_or_null, double* f);
int fx_thermal_force(fx_model* model, double* f);
/* Solver::solve seam: solve K x = b for a host CSR matrix (square, symmetric
 * positive definite, n rows, int64 row offsets and columns) on the GPU.
 * Solver::solve(k, f, precond, tol, max_iter) maps onto `opts`:
 *   IterativeSolver (iterative.rs:26-136): reference_iterative = 1, rtol = tol,
 *     max_iter = max_iter -> Jacobi PCG on the matrix as given, stopping when the
 *     ABSOLUTE sqrt(r.z) < tol (z = D^-1 r), FX_CONVERGENCE after max_iter
 *     iterations, as the reference (the static step passes tol 1e-8, 1000);
 *   DirectSolver (direct.rs:19-55, which ignores tol and max_iter): leave
 *     reference_iterative 0 and keep the library's rtol (1e-8) and max_iter;
 *     the matrix is regrouped into 3x3 blocks and solved by block-Jacobi PCG
 *     (FX_PREC_MIXED: FP32 with FP64 residual replacement and a 100x tighter
 *     FP64 target, finished in FP64 if FP32 stalls; FX_PREC_FP64), stopping on
 *     the RELATIVE ||b - K x||_M / ||b||_M <= rtol, M = 3x3 block-Jacobi;
 *     FX_PREC_FP64_CSR: scalar-CSR Jacobi PCG with the relative test.
 * The matrix carries no node coordinates, so the multigrid preconditioner of
 * fx_step_solve is not available here. */
int fx_solve_csr(fx_ctx* ctx, int64_t n, const int64_t* indptr, const int64_t* indices, const double* data,
                 const double* b, double* x, const fx_solve_opts* opts, fx_step_stats* stats);

/* Drops the cached sparsity pattern and assembled matrices of a model; the
 * next solve rebuilds them (the symbolic phase then counts in its time). */
int fx_model_drop_cache(fx_model* model);
/* Measurement: assembles K (precision, X only, penalty applied) and times
 * `reps` standalone launches of the PCG SpMV kernel with CUDA events on the
 * context stream; *ms = mean duration of one launch, *bytes = algorithmic
 * bytes of one launch (matrix values + column indices + row offsets + the
 * two gathered vectors + the two written vectors, padding excluded). */
int fx_profile_spmv(fx_model* model, int precision, int reps, double* ms, double* bytes);

/* Same measurement for the multigrid preconditioner's fine-level operator: one
 * fused Chebyshev smoothing step (BSR3 SpMV with FP64 vectors, then the
 * row-local residual / 3x3 block-Jacobi / direction / iterate update), FP32
 * matrix values when precision is FX_PREC_MIXED (FP16 values of the scaled
 * matrix when fp16 != 0, as amg_fp16_smoother), FP64 otherwise; *bytes =
 * compulsory traffic (values + column indices once, row offsets, 216 B per node
 * of vector and block-inverse traffic). No reference counterpart: measurement
 * support for the FX_PRECOND_AMG path. */
int fx_profile_smoother(fx_model* model, int precision, int fp16, int reps, double* ms, double* bytes);

/* Same measurement for the assembly (Assembler::assemble, src/solver/assembler.rs:37-151):
 * `reps` standalone launches of the element stiffness kernels (precision
 * FX_PREC_MIXED: FP32 element matrices, else FP64) on X with the current
 * temperatures, then of the gather of the element-pair blocks into the BSR3
 * values. *stiff_flops = declared FLOPs of one launch (354,780 per C3D20, 900
 * per C3D4 element: D B and the symmetric upper B^T (D B) per Gauss point),
 * *gather_bytes = compulsory traffic of one gather (element-pair blocks read
 * once, slot list, segment offsets, blocks written once). Measurement support,
 * no counterpart in the reference. */
int fx_profile_assembly(fx_model* model, int precision, int reps, double* stiff_ms, double* stiff_flops,
                        double* gather_ms, double* gather_bytes);

/* ---- result fields ---------------------------------------------------- */
/* StaticStep::calculate_stress_strain (src/solver/step/static_step.rs:271-379):
 * nodal-averaged stress and mechanical strain of the current state, 6 Voigt
 * components per node (xx, yy, zz, xy, yz, zx; engineering shear strains), in
 * node-index order; strain = B at each element's nodes on the undeformed mesh
 * minus the thermal strain change, stress = D(E(T), nu(T)) at the node's current
 * temperature; nodes of no element get zeros. S or E may be NULL. */
int fx_nodal_stress_strain(fx_model* model, double* S, double* E);
/* VtkWriter::write_increment (src/solver/io/vtk.rs:72-319) for the current
 * state: legacy ASCII VTK unstructured grid with POINTS, CELLS (C3D4 as
 * VTK_TETRA, C3D20 as VTK_QUADRATIC_HEXAHEDRON), U, S, E, NT, MISES, TRESCA.
 * Cells are written per element type in ascending element id (the reference
 * follows its hash-map order). The series file and directory layout stay
 * with the caller. */
int fx_write_vtk(fx_model* model, const char* path);
/* The ParaView time series of the reference's VtkWriter (src/solver/io/vtk.rs:46-70,
 * 305-333): fx_vtk_series_init creates `dir` (and its parents) and writes the header of
 * dir/results.vtk.series; fx_vtk_series_add appends { "name" : name, "time" : time } (the
 * reference writes step_<step_id>_<inc_id>.vtk beside it, with fx_write_vtk here);
 * fx_vtk_series_finish closes the list. The bytes match the reference's file, including the
 * comma after the last entry. FX_GENERIC_IO when a file cannot be created or written. */
int fx_vtk_series_init(const char* dir);
int fx_vtk_series_add(const char* dir, const char* name, double time);
int fx_vtk_series_finish(const char* dir);

/* ---- batched decks ---------------------------------------------------- */
/* Runs the first step of every model (each fx_state_initialize'd) with all
 * linear solves of the batch advanced together; per-model status in status[]. */
int fx_batch_solve(fx_ctx* ctx, fx_model* const* models, int n, const fx_solve_opts* opts, int* status,
                   fx_step_stats* stats);

/* ---- request loop (continuous batching) ---------------------------------
 * No reference counterpart (FerriX solves one deck per process, src/main.rs:49-64).
 * The server runs `slots` worker threads on one GPU, each with its own context
 * and stream. Submitted models wait in a FIFO queue; a free slot admits the head
 * request when the summed device-footprint estimate of the running requests
 * plus its own fits the HBM budget (a request larger than the budget runs
 * alone). An admitted model is bound to the slot's context, its first *STATIC
 * step is solved (fx_step_solve semantics, the server's solve options), the
 * displacements are copied to host memory and all of its device memory is
 * released again. Requests on different slots overlap on the device; each
 * result is the same as when the model is solved alone. */
typedef struct {
    int device;
    int slots;               /* concurrent requests (worker threads, one stream each), 1..64 */
    double hbm_budget_bytes; /* admission budget for the summed footprint estimates; 0 = 70% of free memory.
                                fx_server_create reserves it in the device's memory pool (kept by the
                                process until it exits) */
    fx_solve_opts opts;      /* solve options of every request */
} fx_server_opts;

typedef struct {
    int status;             /* fx_status of the request */
    int slot;               /* worker that ran it */
    double queue_ms;        /* submit -> admission */
    double service_ms;      /* admission -> displacements on the host */
    double latency_ms;      /* submit -> displacements on the host */
    double footprint_bytes; /* admission estimate */
    double admit_at_ms;     /* admission time, ms since fx_server_create */
    double done_at_ms;      /* completion time, ms since fx_server_create */
    fx_step_stats stats;    /* of the solved step */
    char error[256];        /* message when status != FX_OK */
    double setup_ms;        /* service_ms split: state initialisation and model upload, */
    double solve_ms;        /* the step solve (host wall time; stats.t_total_ms is its device time), */
    double finish_ms;       /* displacement download and release of the model's device memory */
} fx_request_result;

void fx_default_server_opts(fx_server_opts* opts);
int fx_server_create(const fx_server_opts* opts, fx_server** out);
/* `model` must come from fx_model_from_inp with ctx NULL and must stay alive,
 * unused by the caller, until fx_server_wait has returned its result. */
int fx_server_submit(fx_server* server, fx_model* model, int64_t* ticket);
/* Waits up to timeout_s (< 0: no limit) for the request; FX_TIMEOUT if it is
 * not done yet (the ticket stays valid). Otherwise copies the displacements
 * (3 * nodes doubles, node-id order; u may be NULL), fills *result, releases
 * the ticket and returns the request's status. */
int fx_server_wait(fx_server* server, int64_t ticket, double timeout_s, double* u, fx_request_result* result);
/* Finishes the running requests, cancels the queued ones, joins the workers. */
/* What the server set up: slots with a context, kernels found loaded on the device
 * by the slot contexts (fx_ctx_preloaded_kernels, least over slots), the admission
 * budget, the bytes the device's memory pool held after the budget was reserved,
 * and the reservation's outcome (1 the pool grew, 0 it held enough already, -1
 * it could not grow in one piece and grows on demand, which stalls the streams
 * running at that moment). */
typedef struct {
    int slots;
    int preloaded_kernels;
    double budget_bytes;
    double pool_reserved_bytes;
    int reservation;
} fx_server_info;
int fx_server_get_info(fx_server* server, fx_server_info* out);
void fx_server_destroy(fx_server* server);

/* ---- allocation-free SpMV with fused dot -------------------------------
 * No counterpart in the reference. y = A x and *dot = x . y for an FP64 CSR
 * matrix of n rows, all pointers on `device`, work queued on `stream`
 * (cudaStream_t as void*, NULL = default stream); results are ready when the
 * stream reaches them. For callers that may not allocate device memory (a
 * loop being captured into a CUDA graph, a layer that only sees memory owned
 * by the host application's own allocator, a real-time path): it calls no
 * cudaMalloc / cudaFree and uses only a fixed ~513 KiB scratch array compiled
 * into the library, held by every GPU that loads it until exit. Limit: at most
 * 524,288 rows (FX_INVALID_ARGUMENT beyond). The first call on a device looks
 * up the scratch address — make it before any stream capture. Calls share the
 * scratch: calls that overlap on the GPU race and must be ordered. y must not
 * overlap x (FX_INVALID_ARGUMENT). A CUDA error already pending in the calling
 * thread when the call starts is returned as FX_CUDA and left pending. */
int fx_spmv_dot_noalloc(int device, int64_t n, const int64_t* indptr, const int64_t* indices, const double* data,
                        const double* x, double* y, double* dot, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* FERRIX_B200_H */
