// Device-resident static step driver: StaticStep::solve
// (src/solver/step/static_step.rs:47-267) with every vector on the GPU.
//
// Per Newton iteration: f_ext from the loads (host evaluates the amplitudes,
// :102-108), thermal force (:111-118), FP64 internal force on X or X+u
// (:120-136), R = f_ext + f_th - f_int, BC-masked norms and the 1e-3 test
// (:139-171), tangent stiffness on X or X+u (:174-181), penalty
// 1e6 x max element diagonal per BC record (:184-195), PCG for du (:197-204),
// u += du (:207-209). Increments are clipped to the step period and halved
// on failure; the timer advances at the start of every attempt (:80-84,
// :251-259), as in the reference.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <thread>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>

#include "engine.hpp"
#include "pcg_csr.hpp"
#include "amg.hpp"

namespace fx {

thread_local int64_t* g_launch_counter = nullptr;

bool debug_sync() {
    static const bool on = std::getenv("FX_DEBUG_SYNC") != nullptr;
    return on;
}

#ifndef FX_WAIT_SPIN_US
#define FX_WAIT_SPIN_US 5000
#endif
constexpr double kWaitSpinS = FX_WAIT_SPIN_US * 1e-6;

void stream_wait(cudaStream_t s, const char* what, double timeout_s) {
    auto t0 = std::chrono::steady_clock::now();
    while (true) {
        cudaError_t e = cudaStreamQuery(s);
        if (e == cudaSuccess) break;
        if (e != cudaErrorNotReady) fail(FX_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
        double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (dt > timeout_s) fail(FX_TIMEOUT, std::string("device work did not finish in time: ") + what);
        // The first kWaitSpinS of a wait poll without sleeping: a short sleep lasts the kernel's
        // timer slack (~50 us on Linux), which the GPU spent idle after every CG replay (~2 ms
        // of work) before the host could launch the next; longer waits sleep between polls.
        if (dt >= kWaitSpinS) std::this_thread::sleep_for(std::chrono::microseconds(dt < 0.05 ? 20 : 200));
    }
    if (debug_sync()) std::fprintf(stderr, "[sync] %s ok\n", what);
}

void ensure_dense(fx_model* m) {
    if (m->dense_built) return;
    m->dense = build_dense(m->project);
    m->dense_built = true;
}

static void upload_mats(const MatTableHost& h, MatTableDev& d, cudaStream_t s) {
    d.e_off.upload(h.e_off, s);
    d.e_len.upload(h.e_len, s);
    d.nu_off.upload(h.nu_off, s);
    d.nu_len.upload(h.nu_len, s);
    d.a_off.upload(h.a_off, s);
    d.a_len.upload(h.a_len, s);
    d.tref.upload(h.tref, s);
    d.t.upload(h.t, s);
    d.v.upload(h.v, s);
    d.n_mat = (int)h.tref.size();
}

// Element pair buffers and the symbolic sort per element, BSR3 values (FP64 +
// FP32), column indices and the slot map per block, vectors and the multigrid
// hierarchy per node. Blocks per element: 240 for C3D20 and 2.8 for C3D4
// bricks-of-tets meshes (node pairs shared by neighbouring elements counted once).
double model_footprint(const DenseModel& D) {
    const double e20 = (double)D.g20.size(), e4 = (double)D.g4.size(), n = (double)D.n_nodes;
    const double blocks = 240.0 * e20 + 2.8 * e4;
    // per 3x3 block: FP64, FP32 and FP16 values (126 B), column ids and group padding
    return e20 * 32.0e3 + e4 * 1.6e3 + blocks * 136.0 + n * 1.0e3 + 64.0e6;
}

// Spare pool memory to hold before a model's work is queued: 50 % over the
// footprint estimate plus 256 MB, which absorbs the fragmentation that
// otherwise made each new model grow the pool by a few tens of MB.
double model_slack(const DenseModel& D) { return 1.5 * model_footprint(D) + 256.0e6; }

// The pool is grown here, up front and with slack, because growing it goes to
// the driver's physical allocator, which on shared B200 hosts stalled for up to
// 0.5 s at times (even for 40 MB), and a pool that grows while kernels of other
// streams are in flight stalls those too (requests of 7k DOF took 0.3-0.5 s
// instead of 10 ms in a four-slot request loop). One allocation before any work
// is queued cost about 12 ms per GB.
int reserve_pool(int device, cudaStream_t s, double bytes) {
    if (!(bytes > 0.0)) return 0;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    uint64_t keep = UINT64_MAX, reserved = 0, used = 0;  // the pool keeps freed memory (fx_ctx_create sets the same)
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    const double spare = (double)reserved - (double)used;
    if (spare >= bytes) return 0;
    const size_t granule = (size_t)2 << 20;
    const size_t want = ((size_t)(bytes - spare) + granule - 1) / granule * granule;
    void* p = nullptr;
    if (cudaMallocAsync(&p, want, s) != cudaSuccess) {
        cudaGetLastError();  // not enough memory in one piece: the pool grows on demand instead
        return -1;
    }
    cudaFreeAsync(p, s);
    return 1;
}

double pool_reserved_bytes(int device) {
    cudaMemPool_t pool;
    uint64_t reserved = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, device) != cudaSuccess ||
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess) {
        cudaGetLastError();
        return -1.0;
    }
    return (double)reserved;
}

void upload_model(fx_model* m) {
    ensure_dense(m);
    ModelDev& d = m->dev;
    if (d.uploaded) return;
    cudaStream_t s = m->ctx->stream;
    const DenseModel& D = m->dense;
    reserve_pool(m->ctx->device, s, model_slack(D));
    d.xyz.upload(D.xyz, s);
    d.conn4.upload(D.g4.conn, s);
    d.mat4.upload(D.g4.mat, s);
    d.conn20.upload(D.g20.conn, s);
    d.mat20.upload(D.g20.mat, s);
    upload_mats(D.mats, d.mats, s);
    const size_t n3 = 3 * (size_t)D.n_nodes;
    d.tinit.upload(m->t_init, s);
    d.tcur.upload(m->t_cur, s);
    for (DBuf<double>* b : {&d.u, &d.ustart, &d.du, &d.fext, &d.ftmp, &d.fint, &d.R, &d.r64, &d.ax}) {
        b->alloc(n3, s);
        b->zero(s);
    }
    d.fe.alloc(((size_t)D.g4.size() * 4 + (size_t)D.g20.size() * 20) * 3 + 3, s);
    d.maxdiag.alloc(1, s);
    d.err.alloc(1, s);
    d.err.zero(s);
    d.norm_part.alloc(2 * 296, s);
    d.norm_out.alloc(2, s);
    d.uploaded = true;
}

void ensure_structure(fx_model* m) {
    upload_model(m);
    ModelDev& d = m->dev;
    if (d.have_structure) return;
    build_bsr_structure(d.g4(), d.g20(), (int)m->dense.n_nodes, d.S, m->ctx->stream);
    d.have_structure = true;
}

void state_initialize(fx_model* m) {
    // SolutionState::new + initialize (state.rs:32-79) and SolverTime::new
    Project& p = m->project;
    ensure_dense(m);
    for (size_t k = 0; k < m->dense.g4.mat.size(); ++k)
        if (m->dense.g4.mat[k] < 0) fail(FX_INVALID_MODEL, "Element has no material assigned");
    for (size_t k = 0; k < m->dense.g20.mat.size(); ++k)
        if (m->dense.g20.mat[k] < 0) fail(FX_INVALID_MODEL, "Element has no material assigned");
    const int64_t n = m->dense.n_nodes;
    m->t_init.assign(n, p.default_initial_temperature);
    for (auto& kv : p.initial_temperatures) {
        int64_t idx = p.index_of(kv.first);
        if (idx >= 0) m->t_init[idx] = kv.second;
    }
    m->t_cur = m->t_init;
    m->timer = SolverTime();
    if (m->dev.uploaded) {
        cudaStream_t s = m->ctx->stream;
        m->dev.tinit.upload(m->t_init, s);
        m->dev.tcur.upload(m->t_cur, s);
        m->dev.u.zero(s);
    } else {
        upload_model(m);
    }
    m->dev.u_zero = true;
    m->state_ready = true;
}

void check_device_errors(fx_model* m, const char* where) {
    int e = 0;
    FX_CUDA_CHECK(cudaMemcpyAsync(&e, m->dev.err.ptr, sizeof(int), cudaMemcpyDeviceToHost, m->ctx->stream));
    FX_CUDA_CHECK(cudaStreamSynchronize(m->ctx->stream));
    if (e & kErrSingularJ) fail(FX_NUMERICAL, std::string("Mathematical error: Singular Jacobian (") + where + ")");
    if (e & kErrNoMaterial)
        fail(FX_INVALID_MODEL, std::string("Invalid model state: material without elastic constants (") + where + ")");
    if (e) fail(FX_GENERIC, std::string("device error flag ") + std::to_string(e) + " in " + where);
}

static void precheck(fx_model* m) {
    ensure_dense(m);
    const DenseModel& D = m->dense;
    if (D.missing_node_id >= 0) fail_detail(FX_NODE_NOT_FOUND, D.missing_node_error, -1, D.missing_node_id, "");
    for (const ElemGroup* g : {&D.g4, &D.g20})
        for (int64_t k = 0; k < g->size(); ++k) {
            int mi = g->mat[k];
            if (mi < 0)
                fail(FX_INVALID_MODEL, "Invalid model state: Element " + std::to_string(g->elem_ids[k]) +
                                           " has no material assigned.");
            const Material& mat = m->project.materials[mi];
            if (!mat.has_e)
                fail(FX_INVALID_MODEL, "Invalid model state: No Young's Modulus definition found for material '" +
                                           mat.name + "'!");
            if (!mat.has_nu)
                fail(FX_INVALID_MODEL, "Invalid model state: No Poisson's Ratio definition found for material '" +
                                           mat.name + "'!");
        }
}

static void apply_elements(fx_model* m, const double* d_uconf, const double* d_v, double cv, double cth,
                           double* d_out) {
    ModelDev& d = m->dev;
    cudaStream_t s = m->ctx->stream;
    launch_apply(d.g4(), d.g20(), d.xyz.ptr, d_uconf, d_v, d.tinit.ptr, d.tcur.ptr, cv, cth, d.mats.view(),
                 m->ctx->tables.view(), d.fe.ptr, d.err.ptr, s);
    launch_node_gather((int)m->dense.n_nodes, d.S.node_ptr.ptr, d.S.node_slots.ptr, d.fe.ptr, d_out, s);
}

void compute_internal_force(fx_model* m, const double* d_u, const double* d_uconf, double* d_out) {
    ensure_structure(m);
    apply_elements(m, d_uconf, d_u, 1.0, 1.0, d_out);
}

void compute_thermal_force(fx_model* m, double* d_out) {
    ensure_structure(m);
    apply_elements(m, nullptr, nullptr, 0.0, -1.0, d_out);
}

double assemble(fx_model* m, const double* d_u, bool fp64) {
    ensure_structure(m);
    ModelDev& d = m->dev;
    cudaStream_t s = m->ctx->stream;
    const size_t slots = (size_t)d.g4().n * kPairs4 + (size_t)d.g20().n * kPairs20;
    d.maxdiag.zero(s);
    if (fp64) {
        d.ebuf64.alloc(slots * 9 + 9, s);
        d.vals64.alloc((size_t)d.S.n_groups * 36, s);
        launch_stiffness<double>(d.g4(), d.g20(), d.xyz.ptr, d_u, d.tcur.ptr, d.mats.view(), m->ctx->tables.view(),
                                 d.ebuf64.ptr, d.maxdiag.ptr, d.err.ptr, s);
        launch_bsr_gather<double>(d.S, d.ebuf64.ptr, d.vals64.ptr, s);
    } else {
        d.ebuf32.alloc(slots * 9 + 9, s);
        d.vals32.alloc((size_t)d.S.n_groups * 36, s);
        launch_stiffness<float>(d.g4(), d.g20(), d.xyz.ptr, d_u, d.tcur.ptr, d.mats.view(), m->ctx->tables.view(),
                                d.ebuf32.ptr, d.maxdiag.ptr, d.err.ptr, s);
        launch_bsr_gather<float>(d.S, d.ebuf32.ptr, d.vals32.ptr, s);
    }
    unsigned long long bits = 0;
    FX_CUDA_CHECK(cudaMemcpyAsync(&bits, d.maxdiag.ptr, sizeof(bits), cudaMemcpyDeviceToHost, s));
    check_device_errors(m, "stiffness");
    double md;
    std::memcpy(&md, &bits, sizeof(md));
    return md;
}

// ------------------------------------------------------------------ step runner

// One model's StaticStep::solve as a state machine advanced in rounds; each
// round evaluates at most one Newton residual and prepares at most one linear
// system, so many models can share one batched PCG per round.
struct StepRunner {
    fx_model* m = nullptr;
    int k = 0;
    const StaticStep* step = nullptr;
    int64_t step_id = 0;
    fx_solve_opts o{};
    bool fp64 = false;
    StepBc bc;
    BcView bcv{};
    std::vector<int32_t> ldof;
    std::vector<std::vector<int>> lrecs;
    std::vector<double> lval, usum;
    DBuf<double> ucur;
    double cur = 0.0, dt = 0.0;
    int64_t n_inc = 0;
    int it = 0;
    bool ustart_zero = false;  // no increment has converged yet and the step started from u = 0
    enum { kNewInc, kIter, kDone } state = kNewInc;
    bool need_solve = false;
    // host callback after every converged increment (fx_step_solve_cb), else null
    fx_increment_cb inc_cb = nullptr;
    void* inc_user = nullptr;
    fx_step_stats S{};
    double nrm[2] = {0, 0};
    int err_flag = 0;
    PcgSystem<float> sys32;
    PcgSystem<double> sys64;
    // scalar-CSR FP64 Jacobi PCG (FX_PREC_FP64_CSR, or SOLVER=ITERATIVE with reference semantics)
    bool csr = false, csr_reference = false;
    CsrSystem csr_sys;
    int csr_status = FX_OK;
    long long csr_iters = 0;
    double csr_relres = 0.0;
    // aggregation-multigrid preconditioned FP64 CG (FX_PRECOND_AMG)
    bool amg = false;
    double amg_cell = 0.0;
    DBuf<double> amg_xyz;

    void begin(fx_model* mm, int kk, const fx_solve_opts& oo) {
        m = mm;
        k = kk;
        o = oo;
        Project& p = m->project;
        if (k < 0 || k >= (int)p.steps.size()) fail(FX_INVALID_ARGUMENT, "step index out of range");
        if (!m->state_ready) fail(FX_INVALID_ARGUMENT, "fx_state_initialize was not called");
        precheck(m);
        ensure_structure(m);
        step = &p.steps[k];
        step_id = k + 1;
        csr_reference = o.reference_iterative && step->solver == SolverType::Iterative;
        csr = o.precision == FX_PREC_FP64_CSR || csr_reference;
        amg = !csr && o.preconditioner == FX_PRECOND_AMG;
        fp64 = o.precision == FX_PREC_FP64 || csr || amg;
        if (amg) {  // aggregate cells holding amg_aggregate_nodes nodes on average
            const double vol = m->dense.volume > 0.0 ? m->dense.volume : 1.0;
            const double per = o.amg_aggregate_nodes > 0 ? (double)o.amg_aggregate_nodes : 40.0;
            amg_cell = std::cbrt(per * vol / (double)std::max<int64_t>(1, m->dense.n_nodes));
        }
        cudaStream_t s = m->ctx->stream;
        ModelDev& d = m->dev;
        const size_t n3 = 3 * (size_t)m->dense.n_nodes;
        m->timer.new_step(step->inc.period);  // Step::solve (steps.rs:34)
        std::map<int32_t, int> slot;
        for (size_t r = 0; r < step->bcs.size(); ++r) {
            int64_t idx = p.index_of(step->bcs[r].node_id);
            if (idx < 0) continue;
            int32_t dof = (int32_t)(3 * idx + step->bcs[r].dof);
            auto ins = slot.emplace(dof, (int)bc.dof.size());
            if (ins.second) {
                bc.dof.push_back(dof);
                bc.cnt.push_back(0.0);
                bc.recs.emplace_back();
            }
            bc.cnt[ins.first->second] += 1.0;
            bc.recs[ins.first->second].push_back((int)r);
        }
        bc.d_dof.upload(bc.dof, s);
        bc.d_cnt.upload(bc.cnt, s);
        bc.d_usum.alloc(bc.dof.size() + 1, s);
        std::vector<uint8_t> mask(n3, 0);
        for (int32_t dd : bc.dof) mask[dd] = 1;
        bc.d_mask.upload(mask, s);
        bcv = BcView{(int)bc.dof.size(), bc.d_dof.ptr, bc.d_cnt.ptr, bc.d_usum.ptr};
        slot.clear();
        for (size_t r = 0; r < step->loads.size(); ++r) {
            int64_t idx = p.index_of(step->loads[r].node_id);
            if (idx < 0) continue;
            int32_t dof = (int32_t)(3 * idx + step->loads[r].dof);
            auto ins = slot.emplace(dof, (int)ldof.size());
            if (ins.second) {
                ldof.push_back(dof);
                lrecs.emplace_back();
            }
            lrecs[ins.first->second].push_back((int)r);
        }
        d.load_dof.upload(ldof, s);
        d.load_val.alloc(ldof.size() + 1, s);
        lval.resize(ldof.size());
        usum.resize(bc.dof.size());
        ucur.alloc(n3, s);
        cur = 0.0;
        n_inc = 0;
        dt = step->inc.initial;
        FX_CUDA_CHECK(cudaMemcpyAsync(d.ustart.ptr, d.u.ptr, n3 * sizeof(double), cudaMemcpyDeviceToDevice, s));
        ustart_zero = d.u_zero;
        state = kNewInc;
    }

    // increment bookkeeping (static_step.rs:71-98); returns false when the step is done
    bool start_increment_if_needed() {
        if (state == kDone) return false;
        if (state != kNewInc) return true;
        if (!(cur < step->inc.period)) {
            finish();
            return false;
        }
        ++n_inc;
        if (n_inc > step->inc.max_increments)
            fail(FX_CONVERGENCE, "Solver failed to converge: Maximum increment count of " +
                                     std::to_string(step->inc.max_increments) + " exceeded.");
        if (cur + dt > step->inc.period) dt = step->inc.period - cur;
        m->timer.new_increment(dt);
        S.increments++;
        if (o.verbose)
            std::printf("Increment %lld | Step Time: %.4e | Increment Size: %.4e\n", (long long)n_inc,
                        m->timer.local, dt);
        const size_t n3 = 3 * (size_t)m->dense.n_nodes;
        FX_CUDA_CHECK(cudaMemcpyAsync(ucur.ptr, m->dev.ustart.ptr, n3 * sizeof(double), cudaMemcpyDeviceToDevice,
                                      m->ctx->stream));
        it = 0;
        state = kIter;
        return true;
    }

    // f_ext + f_th - f_int and the masked norms, queued without a host sync
    void launch_residual() {
        ModelDev& d = m->dev;
        cudaStream_t s = m->ctx->stream;
        const size_t n3 = 3 * (size_t)m->dense.n_nodes;
        S.newton_iterations++;
        for (size_t j = 0; j < ldof.size(); ++j) {
            double acc = 0.0;
            for (int r : lrecs[j]) acc += step->loads[r].eval(m->timer, step_id);
            lval[j] = acc;
        }
        d.load_val.upload(lval.data(), lval.size(), s);
        d.fext.zero(s);
        launch_scatter_set((int)ldof.size(), d.load_dof.ptr, d.load_val.ptr, d.fext.ptr, s);
        if (m->dense.any_expansion) {
            compute_thermal_force(m, d.ftmp.ptr);
            launch_axpby((int64_t)n3, 1.0, d.fext.ptr, 1.0, d.ftmp.ptr, d.fext.ptr, s);
        }
        if (it == 0 && ustart_zero && !step->nlgeom && !m->dense.any_expansion) {
            // ucur is a copy of the all-zero ustart and no strain is thermal: every term of
            // f_int = sum B^T D (B u - eps_th) is a zero, so the element pass is skipped (R =
            // f_ext - f_int has the same bits for either sign of those zeros)
            d.fint.zero(s);
        } else {
            compute_internal_force(m, ucur.ptr, step->nlgeom ? ucur.ptr : nullptr, d.fint.ptr);
        }
        launch_axpby((int64_t)n3, 1.0, d.fext.ptr, -1.0, d.fint.ptr, d.R.ptr, s);
        launch_masked_norms((int64_t)n3, d.R.ptr, d.fext.ptr, bc.d_mask.ptr, d.norm_part.ptr, d.norm_out.ptr, s);
        FX_CUDA_CHECK(cudaMemcpyAsync(nrm, d.norm_out.ptr, sizeof(nrm), cudaMemcpyDeviceToHost, s));
        FX_CUDA_CHECK(cudaMemcpyAsync(&err_flag, d.err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    }

    // after the host sync: the 1e-3 test (static_step.rs:145-171)
    void decide() {
        if (err_flag) check_device_errors(m, "internal force");
        double rn = std::sqrt(nrm[0]), fn = std::sqrt(nrm[1]);
        double rel = fn > 1e-6 ? rn / fn : rn;
        if (o.verbose) std::printf("  Iteration %d: |R| = %.3e, |R|/|F_ext| = %.3e\n", it, rn, rel);
        if (rel < 1e-3) {
            S.last_rel_residual = rel;
            cur += dt;
            const size_t n3 = 3 * (size_t)m->dense.n_nodes;
            FX_CUDA_CHECK(cudaMemcpyAsync(m->dev.ustart.ptr, ucur.ptr, n3 * sizeof(double), cudaMemcpyDeviceToDevice,
                                          m->ctx->stream));
            ustart_zero = false;
            state = kNewInc;
            need_solve = false;
            if (inc_cb) {  // the converged increment's result (static_step.rs:219-248: write_increment)
                FX_CUDA_CHECK(cudaMemcpyAsync(m->dev.u.ptr, m->dev.ustart.ptr, n3 * sizeof(double),
                                              cudaMemcpyDeviceToDevice, m->ctx->stream));
                m->dev.u_zero = false;
                stream_wait(m->ctx->stream, "increment result");
                const int rc = inc_cb(inc_user, m, step_id, (int)n_inc, m->timer.global);
                if (rc != 0) fail(FX_GENERIC_IO, "Generic IO error: increment callback returned " + std::to_string(rc));
            }
        } else {
            need_solve = true;
        }
    }

    // tangent, penalty, block-Jacobi (static_step.rs:173-199)
    void prepare_solve() {
        ModelDev& d = m->dev;
        cudaStream_t s = m->ctx->stream;
        EventTimer ph;
        ph.start(s);
        assemble(m, step->nlgeom ? ucur.ptr : nullptr, fp64);
        for (size_t j = 0; j < bc.dof.size(); ++j) {
            double acc = 0.0;
            for (int r : bc.recs[j]) acc += step->bcs[r].eval(m->timer, step_id);
            usum[j] = acc;
        }
        bc.d_usum.upload(usum.data(), usum.size(), s);
        const int64_t nn = m->dense.n_nodes;
        if (csr) {
            launch_penalty<double>(d.S, d.vals64.ptr, bcv, d.maxdiag.ptr, d.R.ptr, ucur.ptr, s);
            csr_sys.from_bsr(d.S, d.vals64.ptr, s);
        } else if (amg) {
            launch_penalty<double>(d.S, d.vals64.ptr, bcv, d.maxdiag.ptr, d.R.ptr, ucur.ptr, s);
            d.minv64.alloc((size_t)nn * 9, s);
            launch_block_jacobi<double>(d.S, d.vals64.ptr, d.minv64.ptr, s);
            amg_xyz.alloc(3 * (size_t)nn, s);
            // aggregation and rigid-body modes on the configuration the tangent is taken at
            launch_axpby(3 * nn, 1.0, d.xyz.ptr, step->nlgeom ? 1.0 : 0.0, step->nlgeom ? ucur.ptr : nullptr,
                         amg_xyz.ptr, s);
        } else if (fp64) {
            launch_penalty<double>(d.S, d.vals64.ptr, bcv, d.maxdiag.ptr, d.R.ptr, ucur.ptr, s);
            d.minv64.alloc((size_t)nn * 9, s);
            launch_block_jacobi<double>(d.S, d.vals64.ptr, d.minv64.ptr, s);
        } else {
            launch_penalty<float>(d.S, d.vals32.ptr, bcv, d.maxdiag.ptr, d.R.ptr, ucur.ptr, s);
            d.minv32.alloc((size_t)nn * 9, s);
            launch_block_jacobi<float>(d.S, d.vals32.ptr, d.minv32.ptr, s);
        }
        S.t_assembly_ms += ph.stop_ms(s);
        const double* uconf = step->nlgeom ? ucur.ptr : nullptr;
        fx_model* mm = m;
        BcView bv = bcv;
        auto residual64 = [mm, uconf, bv](const double* x, const double* b, double* r64, cudaStream_t ss) {
            ModelDev& dd = mm->dev;
            launch_apply(dd.g4(), dd.g20(), dd.xyz.ptr, uconf, x, dd.tinit.ptr, dd.tcur.ptr, 1.0, 0.0,
                         dd.mats.view(), mm->ctx->tables.view(), dd.fe.ptr, dd.err.ptr, ss);
            launch_node_gather((int)mm->dense.n_nodes, dd.S.node_ptr.ptr, dd.S.node_slots.ptr, dd.fe.ptr, dd.r64.ptr,
                               ss);
            launch_axpby((int64_t)3 * mm->dense.n_nodes, 1.0, b, -1.0, dd.r64.ptr, r64, ss);
            launch_penalty_apply(bv, dd.maxdiag.ptr, x, r64, ss);
        };
        if (fp64) {
            sys64 = PcgSystem<double>();
            sys64.S = &d.S;
            sys64.vals = d.vals64.ptr;
            sys64.minv = d.minv64.ptr;
            sys64.b = d.R.ptr;
            sys64.x = d.du.ptr;
            sys64.residual64 = residual64;
        } else {
            sys32 = PcgSystem<float>();
            sys32.S = &d.S;
            sys32.vals = d.vals32.ptr;
            sys32.minv = d.minv32.ptr;
            sys32.b = d.R.ptr;
            sys32.x = d.du.ptr;
            sys32.residual64 = residual64;
        }
    }

    // Mixed precision stalled (FP32 stiffness too coarse for this system's
    // conditioning): assemble the FP64 tangent with the same penalty value and
    // continue in FP64 from the mixed iterate.
    bool fallback = false;
    void prepare_fp64_fallback() {
        ModelDev& d = m->dev;
        cudaStream_t s = m->ctx->stream;
        S.pcg_iterations += sys32.iterations;
        S.reliable_updates += sys32.replacements;
        DBuf<unsigned long long> keep;
        keep.alloc(1, s);
        FX_CUDA_CHECK(cudaMemcpyAsync(keep.ptr, d.maxdiag.ptr, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s));
        assemble(m, step->nlgeom ? ucur.ptr : nullptr, true);
        FX_CUDA_CHECK(cudaMemcpyAsync(d.maxdiag.ptr, keep.ptr, sizeof(unsigned long long), cudaMemcpyDeviceToDevice, s));
        launch_penalty<double>(d.S, d.vals64.ptr, bcv, d.maxdiag.ptr, nullptr, nullptr, s);
        d.minv64.alloc((size_t)m->dense.n_nodes * 9, s);
        launch_block_jacobi<double>(d.S, d.vals64.ptr, d.minv64.ptr, s);
        sys64 = PcgSystem<double>();
        sys64.S = &d.S;
        sys64.vals = d.vals64.ptr;
        sys64.minv = d.minv64.ptr;
        sys64.b = d.R.ptr;
        sys64.x = d.du.ptr;
        sys64.residual64 = sys32.residual64;
        sys64.warm_start = true;
        sys64.bnorm2 = sys32.bnorm2_seen;  // the tolerance stays relative to the step's right-hand side
        fallback = true;
        S.fp64_fallbacks++;
    }

    // u += du (static_step.rs:207-209); cut-back after 15 solves (:251-259)
    void after_solve() {
        const bool use64 = fp64 || fallback;
        const bool scalar = csr || amg;  // solved outside the batched BSR3 PCG
        long long iters = scalar ? csr_iters : use64 ? sys64.iterations : sys32.iterations;
        int st = scalar ? csr_status : use64 ? sys64.status : sys32.status;
        fallback = false;
        S.linear_solves++;
        S.pcg_iterations += iters;
        S.reliable_updates += scalar ? 0 : use64 ? sys64.replacements : sys32.replacements;
        S.last_linear_relres = scalar ? csr_relres : use64 ? sys64.relres : sys32.relres;
        if (st == FX_NUMERICAL)
            fail(FX_NUMERICAL,
                 "Mathematical error: PCG breakdown (system not positive definite). Check for rigid body modes!");
        if (st == FX_CONVERGENCE)
            fail(FX_CONVERGENCE,
                 "Solver failed to converge: PCG did not converge after " + std::to_string(iters) + " iterations");
        if (st != FX_OK) fail(st, "linear solve failed");
        const size_t n3 = 3 * (size_t)m->dense.n_nodes;
        launch_axpby((int64_t)n3, 1.0, ucur.ptr, 1.0, m->dev.du.ptr, ucur.ptr, m->ctx->stream);
        need_solve = false;
        if (++it >= 15) {
            if (o.verbose) std::printf("Increment failed to converge. Retrying with smaller increment.\n");
            dt /= 2.0;
            if (dt < step->inc.min_inc)
                fail(FX_CONVERGENCE, "Solver failed to converge: Minimum time increment reached. Convergence failed.");
            state = kNewInc;
        }
    }

    void finish() {
        const size_t n3 = 3 * (size_t)m->dense.n_nodes;
        FX_CUDA_CHECK(cudaMemcpyAsync(m->dev.u.ptr, m->dev.ustart.ptr, n3 * sizeof(double),
                                      cudaMemcpyDeviceToDevice, m->ctx->stream));
        m->dev.u_zero = false;
        S.bsr_blocks = m->dev.S.n_blocks;
        state = kDone;
    }
};

// Advances all runners in lockstep rounds; runners share the context stream.
// Returns per-runner status (FX_OK or the error that stopped that model).
static void run_rounds(fx_ctx* ctx, std::vector<StepRunner*>& rs, std::vector<int>& status,
                       std::vector<std::string>& msgs) {
    cudaStream_t s = ctx->stream;
    const size_t n = rs.size();
    status.assign(n, FX_OK);
    msgs.assign(n, std::string());
    std::vector<char> alive(n, 1);
    auto guard = [&](size_t i, auto&& f) {
        if (!alive[i]) return;
        try {
            f();
        } catch (const Error& e) {
            status[i] = e.status;
            msgs[i] = e.what();
            alive[i] = 0;
        }
    };
    PcgOptions po;
    if (!rs.empty()) {
        po.rtol = rs[0]->o.rtol;
        po.max_iter = rs[0]->o.max_iter;
        po.poll = rs[0]->o.poll_interval;
        po.reliable_delta = rs[0]->o.reliable_delta;
        po.graphs = rs[0]->o.use_graphs != 0;
        po.amg_degree = rs[0]->o.amg_smoother_degree > 0 ? rs[0]->o.amg_smoother_degree : 2;
        po.amg_fp32 = rs[0]->o.precision == FX_PREC_MIXED;
        po.amg_kcycle = rs[0]->o.amg_cycle == 1;
        po.amg_cheb_kind = rs[0]->o.amg_smoother == 1 ? 1 : 0;
        const double oc = rs[0]->o.amg_overcorrect;
        po.amg_overcorrect = oc > 0.0 && oc < 2.0 ? oc : kAmgOvercorrect;
        po.amg_cheb_ratio = rs[0]->o.amg_cheb_ratio > 1.0 ? rs[0]->o.amg_cheb_ratio : kAmgChebRatio;
        po.amg_fused_coarse = rs[0]->o.amg_fused_coarse == 1;
        po.amg_fp16 = rs[0]->o.amg_fp16_smoother >= 0;
        // persistent cluster solve for tiny systems (a cluster's few SMs are latency-bound
        // where the multi-launch path uses the whole GPU); all of a round's in one launch
        const int pm = rs[0]->o.amg_persistent_max_dof;
        po.amg_persistent_max_dof = pm != 0 ? pm : kClDefaultMaxDof;
    }
    while (true) {
        bool any = false;
        for (size_t i = 0; i < n; ++i)
            guard(i, [&] {
                if (rs[i]->start_increment_if_needed()) {
                    rs[i]->launch_residual();
                    any = true;
                } else {
                    alive[i] = 0;
                }
            });
        if (!any) break;
        stream_wait(s, "stream");
        std::vector<size_t> solve;
        for (size_t i = 0; i < n; ++i)
            guard(i, [&] {
                rs[i]->decide();
                if (rs[i]->need_solve) {
                    rs[i]->prepare_solve();
                    solve.push_back(i);
                }
            });
        if (solve.empty()) continue;
        EventTimer ph;
        ph.start(s);
        std::vector<size_t> csr_ids, bsr_ids, cluster_ids;
        for (size_t i : solve) (rs[i]->csr || rs[i]->amg ? csr_ids : bsr_ids).push_back(i);
        for (size_t i : csr_ids) {
            StepRunner& r = *rs[i];
            if (r.amg) {
                AmgStats ast;
                // NLGEOM: the Newton iterations after the first of an increment keep the
                // hierarchy built at the increment's first tangent (aggregates and
                // rigid-body prolongators of that configuration) and refresh its values
                const bool reuse = r.step->nlgeom && r.it > 0;
                ModelDev& d = r.m->dev;
                if (!d.amg) d.amg = std::make_unique<AmgPcg>();
                const int64_t ndof = 3 * r.m->dense.n_nodes;
                if (!po.amg_kcycle && po.amg_persistent_max_dof > 0 && ndof <= po.amg_persistent_max_dof) {
                    // small system: hierarchy now, its whole CG in the round's persistent launch below
                    guard(i, [&] {
                        d.amg->prepare(d.S, d.vals64.ptr, d.minv64.ptr, r.amg_xyz.ptr, r.amg_cell, po, s, &ast,
                                       reuse, true);
                        r.S.amg_levels = ast.levels;
                        r.S.amg_setup_ms += ast.setup_ms;
                        cluster_ids.push_back(i);
                    });
                    continue;
                }
                r.csr_status = d.amg->solve(d.S, d.vals64.ptr, d.minv64.ptr, r.amg_xyz.ptr, r.amg_cell, d.R.ptr,
                                            d.du.ptr, po, s, &ctx->launches, &r.csr_iters, &r.csr_relres, &ast, reuse);
                r.S.amg_levels = ast.levels;
                r.S.amg_setup_ms += ast.setup_ms;
                continue;
            }
            PcgOptions pc = po;
            if (r.csr_reference) {  // iterative.rs:26-122 called with tol 1e-8, max_iter 1000 (static_step.rs:204)
                pc.rtol = 1e-8;
                pc.max_iter = 1000;
            }
            r.csr_status = ctx->pcgcsr.solve(r.csr_sys, r.m->dev.R.ptr, r.m->dev.du.ptr, pc, r.csr_reference, s,
                                             &ctx->launches, &r.csr_iters, &r.csr_relres);
        }
        if (!cluster_ids.empty()) {
            // every small multigrid system of the round in one persistent launch (a cluster each)
            std::vector<ClInst> desc;
            for (size_t i : cluster_ids) desc.push_back(rs[i]->m->dev.amg->describe(rs[i]->m->dev.R.ptr,
                                                                                    rs[i]->m->dev.du.ptr));
            DBuf<ClInst> d_desc;
            DBuf<ClResult> d_res;
            d_desc.upload(desc, s);
            d_res.alloc(desc.size(), s);
            const AmgPcg& a0 = *rs[cluster_ids[0]]->m->dev.amg;
            launch_amg_cluster(d_desc.ptr, d_res.ptr, (int)desc.size(), po.amg_fp32, po.rtol, po.max_iter,
                               a0.amg.degree(), a0.amg.overcorrect(), s);
            std::vector<ClResult> res(desc.size());
            d_res.download(res.data(), res.size(), s);
            stream_wait(s, "persistent multigrid CG");
            for (size_t k = 0; k < cluster_ids.size(); ++k) {
                StepRunner& r = *rs[cluster_ids[k]];
                r.csr_status = res[k].status;
                r.csr_iters = res[k].iterations;
                guard(cluster_ids[k], [&] {
                    r.csr_relres = r.m->dev.amg->true_relres(r.m->dev.R.ptr, r.m->dev.du.ptr, s);
                });
            }
        }
        {
            std::vector<PcgSystem<double>*> v64;
            std::vector<PcgSystem<float>*> v32;
            for (size_t i : bsr_ids) {
                if (rs[i]->fp64) v64.push_back(&rs[i]->sys64);
                else v32.push_back(&rs[i]->sys32);
            }
            if (!v64.empty()) ctx->pcg64.solve(v64, po, s, &ctx->launches);
            if (!v32.empty()) {
                PcgOptions p32 = po;  // mixed: the tightened residual target, also for its FP64 finish
                p32.rtol = po.rtol * kMixedBjResidualFactor;
                p32.accept_rtol = po.rtol;
                ctx->pcg32.solve(v32, p32, s, &ctx->launches);
                std::vector<PcgSystem<double>*> fb;
                for (size_t i : bsr_ids)
                    if (!rs[i]->fp64 && rs[i]->sys32.stagnated)
                        guard(i, [&] {
                            rs[i]->prepare_fp64_fallback();
                            fb.push_back(&rs[i]->sys64);
                        });
                if (!fb.empty()) ctx->pcg64.solve(fb, p32, s, &ctx->launches);
            }
        }
        solve.swap(bsr_ids);
        double ms = ph.stop_ms(s);
        solve.insert(solve.end(), csr_ids.begin(), csr_ids.end());
        for (size_t i : solve) {
            rs[i]->S.t_pcg_ms += ms;
            guard(i, [&] {
                check_device_errors(rs[i]->m, "linear solve");
                rs[i]->after_solve();
            });
        }
    }
    stream_wait(s, "stream");
}

int step_solve(fx_model* m, int k, const fx_solve_opts& o, fx_step_stats* st, fx_increment_cb cb, void* user) {
    fx_ctx* ctx = m->ctx;
    int64_t* saved = g_launch_counter;
    g_launch_counter = &ctx->launches;
    struct Restore {
        int64_t* v;
        ~Restore() { g_launch_counter = v; }
    } restore{saved};
    ensure_dense(m);
    reserve_pool(ctx->device, ctx->stream, model_slack(m->dense));
    EventTimer tot;
    tot.start(ctx->stream);
    StepRunner r;
    r.begin(m, k, o);
    r.inc_cb = cb;
    r.inc_user = user;
    std::vector<StepRunner*> rs{&r};
    std::vector<int> status;
    std::vector<std::string> msgs;
    run_rounds(ctx, rs, status, msgs);
    r.S.t_total_ms = tot.stop_ms(ctx->stream);
    if (st) *st = r.S;
    if (status[0] != FX_OK) fail(status[0], msgs[0]);
    return FX_OK;
}

// The batch on one context: every model's step advanced in lockstep rounds on its stream.
static int batch_solve_on(fx_ctx* ctx, fx_model* const* models, int n, const fx_solve_opts& o, int* status_out,
                          fx_step_stats* stats) {
    int64_t* saved = g_launch_counter;
    g_launch_counter = &ctx->launches;
    struct Restore {
        int64_t* v;
        ~Restore() { g_launch_counter = v; }
    } restore{saved};
    EventTimer tot;
    tot.start(ctx->stream);
    std::vector<StepRunner> runners(n);
    std::vector<StepRunner*> rs;
    std::vector<int> pre(n, FX_OK);
    std::string first_msg;
    for (int i = 0; i < n; ++i) {
        try {
            if (!models[i] || models[i]->ctx != ctx) fail(FX_INVALID_ARGUMENT, "model not bound to this context");
            runners[i].begin(models[i], 0, o);
            rs.push_back(&runners[i]);
        } catch (const Error& e) {
            pre[i] = e.status;
            if (first_msg.empty()) first_msg = e.what();
        }
    }
    std::vector<int> status;
    std::vector<std::string> msgs;
    run_rounds(ctx, rs, status, msgs);
    double ms = tot.stop_ms(ctx->stream);
    int rc = FX_OK;
    size_t j = 0;
    for (int i = 0; i < n; ++i) {
        int st = pre[i];
        if (st == FX_OK) {
            st = status[j];
            if (st != FX_OK && first_msg.empty()) first_msg = msgs[j];
            if (stats) {
                stats[i] = runners[i].S;
                stats[i].t_total_ms = ms;
            }
            ++j;
        }
        if (status_out) status_out[i] = st;
        if (st != FX_OK && rc == FX_OK) rc = st;
    }
    if (rc != FX_OK) ctx->last_error = first_msg;
    return rc;
}

// A batch of several models is spread over kBatchWorkers worker contexts of the
// caller's context (own streams and host threads; balanced by DOF, largest first):
// each worker runs its models' rounds (assembly, multigrid setup with its host round
// trips, the multi-launch CG of each system, one persistent launch for its tiny ones)
// while the others do theirs, so the kernels of up to kBatchWorkers systems share the
// GPU. A model takes the same path whichever worker it lands on.
#ifndef FX_BATCH_WORKERS
#define FX_BATCH_WORKERS 4
#endif
constexpr int kBatchWorkers = FX_BATCH_WORKERS;

int batch_solve(fx_ctx* ctx, fx_model* const* models, int n, const fx_solve_opts& o_in, int* status_out,
                fx_step_stats* stats) {
    const fx_solve_opts& o = o_in;
    const int K = std::min(kBatchWorkers, n);
    if (K <= 1) return batch_solve_on(ctx, models, n, o, status_out, stats);
    for (int i = 0; i < n; ++i)
        if (!models[i] || models[i]->ctx != ctx) {
            ctx->last_error = "model not bound to this context";
            return FX_INVALID_ARGUMENT;
        }
    while ((int)ctx->workers.size() < K) {
        fx_ctx* w = nullptr;
        const int rc = fx_ctx_create(ctx->device, &w);
        if (rc != FX_OK) fail(rc, "batch worker context creation failed");
        ctx->workers.push_back(w);
    }
    FX_CUDA_CHECK(cudaStreamSynchronize(ctx->stream));  // the models' uploads on this stream are done
    std::vector<int> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        ensure_dense(models[a]);
        ensure_dense(models[b]);
        return models[a]->dense.n_nodes > models[b]->dense.n_nodes;
    });
    std::vector<std::vector<int>> part(K);
    std::vector<int64_t> load(K, 0);
    for (int i : order) {
        const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        part[k].push_back(i);
        load[k] += models[i]->dense.n_nodes;
    }
    std::vector<int> rcs(K, FX_OK);
    std::vector<std::string> errs(K);
    std::vector<int64_t> launches0(K);
    std::vector<std::thread> threads;
    for (int k = 0; k < K; ++k) {
        threads.emplace_back([&, k] {
            fx_ctx* w = ctx->workers[k];
            launches0[k] = w->launches;
            cudaSetDevice(w->device);
            std::vector<fx_model*> ms;
            for (int i : part[k]) {
                models[i]->ctx = w;
                ms.push_back(models[i]);
            }
            std::vector<int> st(ms.size(), FX_OK);
            std::vector<fx_step_stats> ss(ms.size());
            rcs[k] = guarded(w, [&] {
                return batch_solve_on(w, ms.data(), (int)ms.size(), o, st.data(), ss.data());
            });
            if (rcs[k] != FX_OK) errs[k] = w->last_error;
            cudaStreamSynchronize(w->stream);
            for (size_t j = 0; j < ms.size(); ++j) {
                ms[j]->ctx = ctx;
                if (status_out) status_out[part[k][j]] = st[j];
                if (stats) stats[part[k][j]] = ss[j];
            }
        });
    }
    for (auto& t : threads) t.join();
    int rc = FX_OK;
    for (int k = 0; k < K; ++k) {
        ctx->launches += ctx->workers[k]->launches - launches0[k];
        if (rc == FX_OK && rcs[k] != FX_OK) {
            rc = rcs[k];
            ctx->last_error = errs[k];
        }
    }
    return rc;
}

}  // namespace fx
