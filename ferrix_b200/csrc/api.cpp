// extern "C" boundary (include/ferrix_b200.h). Every entry point converts
// fx::Error / CUDA failures into an fx_status and keeps the message for
// fx_ctx_last_error.
#include <cuda.h>

#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <map>
#include <vector>

#include "engine.hpp"

using namespace fx;


namespace {
template <typename T>
static double profile_t(fx_model* m, int reps, double* bytes) {
    ModelDev& d = m->dev;
    cudaStream_t s = m->ctx->stream;
    const bool is64 = sizeof(T) == 8;
    assemble(m, nullptr, is64);
    const int64_t nn = m->dense.n_nodes;
    DBuf<T> minv;
    minv.alloc((size_t)nn * 9, s);
    const T* vals = is64 ? (const T*)d.vals64.ptr : (const T*)d.vals32.ptr;
    launch_block_jacobi<T>(d.S, vals, minv.ptr, s);
    std::vector<double> ones(3 * (size_t)nn, 1.0);
    d.R.upload(ones, s);
    PcgSystem<T> sys;
    sys.S = &d.S;
    sys.vals = vals;
    sys.minv = minv.ptr;
    sys.b = d.R.ptr;
    sys.x = d.du.ptr;
    PcgBatch<T> batch;
    double ms = batch.profile_spmv(sys, reps, s);
    // compulsory bytes of one k_pcg_spmv launch: every block's 9 values and column id, the
    // row offsets, the direction p read once (3 components per node; the fourth, padding
    // lane of its node-aligned layout excluded) and q written once
    const double nb = (double)d.S.n_blocks, n3 = 3.0 * (double)nn;
    *bytes = nb * (9.0 * sizeof(T) + 4.0) + 4.0 * (nn + 1) + 2.0 * sizeof(T) * n3;
    return ms;
}

}  // namespace

namespace fx {

ErrorRecord& thread_error() {
    static thread_local ErrorRecord rec;
    return rec;
}

// The display prefixes of FerrixError (src/solver/error.rs:12-72) whose variant
// carries only a message string: the payload is the text after the prefix.
static std::string strip_variant_prefix(const std::string& m) {
    for (const char* p : {"Mathematical error: ", "Solver failed to converge: ", "Invalid model state: ",
                          "Generic error: ", "Generic IO error: "})
        if (m.rfind(p, 0) == 0) return m.substr(std::strlen(p));
    return m;
}

void ErrorRecord::set(const Error& e) {
    status = e.status;
    line = e.line;
    id = e.id;
    message = e.what();
    text = e.text.empty() ? strip_variant_prefix(message) : e.text;
}

void ErrorRecord::set(int st, const std::string& msg) { set(Error(st, msg)); }

// Loads every kernel of the library's modules on `device` (CUDA 12.4 driver
// entry points, looked up at run time; without them, or on any error, kernels
// load at their first launch as before). Returns the number of kernels the
// first call on this device loaded (later calls return the same count), -1
// when the driver entry points are missing.
int preload_kernels(int device) {
    static std::mutex mu;
    static std::map<int, int> done;
    std::lock_guard<std::mutex> g(mu);
    auto it = done.find(device);
    if (it != done.end()) return it->second;
    int loaded = -1;
    using GetModule = CUresult (*)(CUmodule*, CUfunction);
    using Count = CUresult (*)(unsigned int*, CUmodule);
    using Enumerate = CUresult (*)(CUfunction*, unsigned int, CUmodule);
    using Load = CUresult (*)(CUfunction);
    void *p_get = nullptr, *p_count = nullptr, *p_enum = nullptr, *p_load = nullptr;
    cudaDriverEntryPointQueryResult q;
    const bool ok = cudaGetDriverEntryPointByVersion("cuFuncGetModule", &p_get, 12040, cudaEnableDefault, &q) ==
                        cudaSuccess && p_get &&
                    cudaGetDriverEntryPointByVersion("cuModuleGetFunctionCount", &p_count, 12040, cudaEnableDefault,
                                                     &q) == cudaSuccess && p_count &&
                    cudaGetDriverEntryPointByVersion("cuModuleEnumerateFunctions", &p_enum, 12040, cudaEnableDefault,
                                                     &q) == cudaSuccess && p_enum &&
                    cudaGetDriverEntryPointByVersion("cuFuncLoad", &p_load, 12040, cudaEnableDefault, &q) ==
                        cudaSuccess && p_load;
    if (ok) {
        loaded = 0;
        for (const void* anchor : {kernels_anchor_amg(), kernels_anchor_amg_cluster(), kernels_anchor_assembly(),
                                   kernels_anchor_csr_solve(),
                                   kernels_anchor_elements(), kernels_anchor_noalloc(), kernels_anchor_pcg(),
                                   kernels_anchor_pcg_csr(), kernels_anchor_vectors()}) {
            cudaFunction_t f = nullptr;
            if (cudaGetFuncBySymbol(&f, anchor) != cudaSuccess || !f) continue;
            CUmodule mod = nullptr;
            unsigned int n = 0;
            if (reinterpret_cast<GetModule>(p_get)(&mod, reinterpret_cast<CUfunction>(f)) != CUDA_SUCCESS ||
                reinterpret_cast<Count>(p_count)(&n, mod) != CUDA_SUCCESS)
                continue;
            std::vector<CUfunction> fns(n);
            if (n == 0 || reinterpret_cast<Enumerate>(p_enum)(fns.data(), n, mod) != CUDA_SUCCESS) continue;
            for (CUfunction fn : fns)
                if (reinterpret_cast<Load>(p_load)(fn) == CUDA_SUCCESS) ++loaded;
        }
    }
    cudaGetLastError();
    done[device] = loaded;
    return loaded;
}

}  // namespace fx

extern "C" {

void fx_default_solve_opts(fx_solve_opts* o) {
    if (!o) return;
    o->precision = FX_PREC_MIXED;
    o->rtol = 1e-8;
    o->max_iter = 50000;
    o->poll_interval = 32;
    o->reliable_delta = 1e-2;
    o->use_graphs = 1;
    o->verbose = 0;
    o->reference_iterative = 0;
    o->preconditioner = FX_PRECOND_AMG;
    o->amg_aggregate_nodes = 40;
    o->amg_smoother_degree = 2;
    o->amg_cycle = 0;  // V-cycle
    o->amg_smoother = 0;
    o->amg_overcorrect = 0.0;
    o->amg_cheb_ratio = 0.0;
    o->amg_persistent_max_dof = 0;
    o->amg_fused_coarse = 0;
    o->amg_fp16_smoother = 0;
}

int fx_ctx_create(int device, fx_ctx** out) {
    if (!out) return FX_INVALID_ARGUMENT;
    *out = nullptr;
    fx_ctx* c = new (std::nothrow) fx_ctx();
    if (!c) return FX_GENERIC;
    int rc = guarded(c, [&] {
        int n = 0;
        FX_CUDA_CHECK(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) fail(FX_INVALID_ARGUMENT, "no such CUDA device");
        c->device = device;
        FX_CUDA_CHECK(cudaSetDevice(device));
        FX_CUDA_CHECK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->preload_functions = preload_kernels(device);
        // keep freed stream-ordered allocations in this process's pool between solves
        // instead of returning them to the driver at every synchronisation
        cudaMemPool_t pool;
        FX_CUDA_CHECK(cudaDeviceGetDefaultMemPool(&pool, device));
        uint64_t keep = UINT64_MAX;
        FX_CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
        // an allocation never takes memory whose free is still queued behind another
        // stream's work: with that reuse, a request of one request-loop slot waited for the
        // queued solve of another (set-up stalls of up to 0.7 s in the four-slot loop); the
        // pool holds the memory reserved ahead, so allocations do not need it
        int no = 0;
        FX_CUDA_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no));
        c->tables.init(c->stream);
        return FX_OK;
    });
    if (rc != FX_OK) {
        fx_ctx_destroy(c);
        return rc;
    }
    *out = c;
    return FX_OK;
}

void fx_ctx_destroy(fx_ctx* ctx) {
    if (!ctx) return;
    for (fx_ctx* w : ctx->workers) fx_ctx_destroy(w);
    ctx->workers.clear();
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaStream_t s = ctx->stream;
    ctx->stream = nullptr;
    delete ctx;  // buffers free on their own streams
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
}

const char* fx_ctx_last_error(const fx_ctx* ctx) { return ctx ? ctx->last_error.c_str() : "null context"; }

int fx_last_error_detail(const fx_ctx* ctx, fx_error_detail* out) {
    if (!out) return FX_INVALID_ARGUMENT;
    const ErrorRecord& r = ctx ? ctx->last_detail : thread_error();
    out->status = r.status;
    out->line = r.line;
    out->id = r.id;
    std::snprintf(out->text, sizeof(out->text), "%s", r.text.c_str());
    std::snprintf(out->message, sizeof(out->message), "%s", r.message.c_str());
    return FX_OK;
}

int fx_ctx_preloaded_kernels(const fx_ctx* ctx) { return ctx ? ctx->preload_functions : -1; }

int64_t fx_ctx_kernel_launches(const fx_ctx* ctx) { return ctx ? ctx->launches : 0; }

void* fx_ctx_stream(const fx_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int fx_model_from_inp(fx_ctx* ctx, const char* text, size_t len, fx_model** out) {
    if (!out || (!text && len)) return FX_INVALID_ARGUMENT;
    *out = nullptr;
    return guarded(ctx, [&] {
        fx_model* m = new fx_model();
        m->ctx = ctx;
        try {
            m->project = parse_inp(std::string_view(text ? text : "", len));
        } catch (...) {
            delete m;
            throw;
        }
        *out = m;
        return FX_OK;
    });
}

int fx_model_export(fx_model* m, double* xyz, int64_t* n4, int32_t* conn4, int32_t* mat4, int64_t* n20,
                    int32_t* conn20, int32_t* mat20) {
    if (!m) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        ensure_dense(m);
        const DenseModel& D = m->dense;
        if (xyz) std::memcpy(xyz, D.xyz.data(), D.xyz.size() * sizeof(double));
        if (n4) *n4 = D.g4.size();
        if (n20) *n20 = D.g20.size();
        if (conn4) std::memcpy(conn4, D.g4.conn.data(), D.g4.conn.size() * sizeof(int32_t));
        if (mat4) std::memcpy(mat4, D.g4.mat.data(), D.g4.mat.size() * sizeof(int32_t));
        if (conn20) std::memcpy(conn20, D.g20.conn.data(), D.g20.conn.size() * sizeof(int32_t));
        if (mat20) std::memcpy(mat20, D.g20.mat.data(), D.g20.mat.size() * sizeof(int32_t));
        return FX_OK;
    });
}

int fx_model_step_records(const fx_model* m, int k, int is_bc, int64_t* ids, int32_t* dofs, double* vals,
                          int64_t* origin, int32_t* tab) {
    if (!m || k < 0 || k >= (int)m->project.steps.size()) return FX_INVALID_ARGUMENT;
    const auto& recs = is_bc ? m->project.steps[k].bcs : m->project.steps[k].loads;
    for (size_t i = 0; i < recs.size(); ++i) {
        if (ids) ids[i] = recs[i].node_id;
        if (dofs) dofs[i] = recs[i].dof;
        if (vals) vals[i] = recs[i].value;
        if (origin) origin[i] = recs[i].origin_step;
        if (tab) tab[i] = recs[i].amp && recs[i].amp->has_data ? 1 : 0;
    }
    return FX_OK;
}

void fx_model_destroy(fx_model* m) {
    if (!m) return;
    if (m->ctx) {
        cudaSetDevice(m->ctx->device);
        cudaStreamSynchronize(m->ctx->stream);
    }
    delete m;
}

int fx_model_sizes(const fx_model* m, int64_t* nn, int64_t* ne, int* ns, int* nm) {
    if (!m) return FX_INVALID_ARGUMENT;
    if (nn) *nn = m->project.n_nodes();
    if (ne) *ne = m->project.n_elements();
    if (ns) *ns = (int)m->project.steps.size();
    if (nm) *nm = (int)m->project.materials.size();
    return FX_OK;
}

int fx_model_node_ids(const fx_model* m, int64_t* ids) {
    if (!m || !ids) return FX_INVALID_ARGUMENT;
    std::memcpy(ids, m->project.index_to_node_id.data(), m->project.index_to_node_id.size() * sizeof(int64_t));
    return FX_OK;
}

int64_t fx_model_node_index(const fx_model* m, int64_t id) { return m ? m->project.index_of(id) : -1; }

int fx_model_set_default_temperature(fx_model* m, double t) {
    if (!m) return FX_INVALID_ARGUMENT;
    m->project.default_initial_temperature = t;
    return FX_OK;
}

int fx_model_step_info(const fx_model* m, int k, int* nlgeom, int* solver, double incr[4], int64_t* nl,
                       int64_t* nb) {
    if (!m || k < 0 || k >= (int)m->project.steps.size()) return FX_INVALID_ARGUMENT;
    const StaticStep& s = m->project.steps[k];
    if (nlgeom) *nlgeom = s.nlgeom ? 1 : 0;
    if (solver) *solver = (int)s.solver;
    if (incr) {
        incr[0] = s.inc.initial;
        incr[1] = s.inc.period;
        incr[2] = s.inc.min_inc;
        incr[3] = s.inc.max_inc;
    }
    if (nl) *nl = (int64_t)s.loads.size();
    if (nb) *nb = (int64_t)s.bcs.size();
    return FX_OK;
}

int fx_state_initialize(fx_model* m) {
    if (!m || !m->ctx) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        state_initialize(m);
        return FX_OK;
    });
}

int fx_state_get_displacements(const fx_model* m, double* u) {
    if (!m || !u) return FX_INVALID_ARGUMENT;
    if (!m->state_ready) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        m->dev.u.download(u, 3 * (size_t)m->dense.n_nodes, m->ctx->stream);
        FX_CUDA_CHECK(cudaStreamSynchronize(m->ctx->stream));
        return FX_OK;
    });
}

int fx_state_set_displacements(fx_model* m, const double* u) {
    if (!m || !u || !m->state_ready) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        m->dev.u_zero = false;
        FX_CUDA_CHECK(cudaMemcpyAsync(m->dev.u.ptr, u, 3 * (size_t)m->dense.n_nodes * sizeof(double),
                                      cudaMemcpyHostToDevice, m->ctx->stream));
        FX_CUDA_CHECK(cudaStreamSynchronize(m->ctx->stream));
        return FX_OK;
    });
}

int fx_state_get_temperatures(const fx_model* m, double* ti, double* tc) {
    if (!m || !m->state_ready) return FX_INVALID_ARGUMENT;
    if (ti) std::memcpy(ti, m->t_init.data(), m->t_init.size() * sizeof(double));
    if (tc) std::memcpy(tc, m->t_cur.data(), m->t_cur.size() * sizeof(double));
    return FX_OK;
}

int fx_state_set_temperatures(fx_model* m, const double* ti, const double* tc) {
    if (!m || !m->state_ready) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        const size_t n = (size_t)m->dense.n_nodes;
        if (ti) m->t_init.assign(ti, ti + n);
        if (tc) m->t_cur.assign(tc, tc + n);
        m->dev.tinit.upload(m->t_init, m->ctx->stream);
        m->dev.tcur.upload(m->t_cur, m->ctx->stream);
        FX_CUDA_CHECK(cudaStreamSynchronize(m->ctx->stream));
        return FX_OK;
    });
}

int fx_step_solve(fx_model* m, int k, const fx_solve_opts* opts, fx_step_stats* st) {
    if (!m || !m->ctx) return FX_INVALID_ARGUMENT;
    fx_solve_opts o;
    if (opts) o = *opts;
    else fx_default_solve_opts(&o);
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        return step_solve(m, k, o, st);
    });
}

int fx_step_solve_cb(fx_model* m, int k, const fx_solve_opts* opts, fx_step_stats* st, fx_increment_cb cb,
                     void* user) {
    if (!m || !m->ctx) return FX_INVALID_ARGUMENT;
    fx_solve_opts o;
    if (opts) o = *opts;
    else fx_default_solve_opts(&o);
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        return step_solve(m, k, o, st, cb, user);
    });
}

int fx_assemble_csr(fx_model* m, const double* u, int precision, int64_t* nnz, int64_t* indptr, int64_t* indices,
                    double* data, double* maxdiag) {
    if (!m || !nnz) return FX_INVALID_ARGUMENT;
    if (!m->state_ready) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        fx_ctx* ctx = m->ctx;
        int64_t* saved = g_launch_counter;
        g_launch_counter = &ctx->launches;
        struct R {
            int64_t* v;
            ~R() { g_launch_counter = v; }
        } r{saved};
        ensure_dense(m);
        if (m->dense.missing_node_id >= 0) fail_detail(FX_NODE_NOT_FOUND, m->dense.missing_node_error, -1, m->dense.missing_node_id, "");
        ensure_structure(m);
        ModelDev& d = m->dev;
        cudaStream_t s = ctx->stream;
        const int64_t nn = m->dense.n_nodes;
        std::vector<int32_t> rp(nn + 1);
        d.S.row_ptr.download(rp.data(), nn + 1, s);
        FX_CUDA_CHECK(cudaStreamSynchronize(s));
        std::vector<int64_t> ip(3 * nn + 1, 0);
        for (int64_t i = 0; i < nn; ++i)
            for (int rr = 0; rr < 3; ++rr) ip[3 * i + rr + 1] = ip[3 * i + rr] + 3 * (int64_t)(rp[i + 1] - rp[i]);
        *nnz = ip[3 * nn];
        if (!indptr || !indices || !data) return FX_OK;
        DBuf<double> du;
        const double* dptr = nullptr;
        if (u) {
            du.upload(u, 3 * (size_t)nn, s);
            dptr = du.ptr;
        }
        double md = assemble(m, dptr, precision == FX_PREC_FP64);
        if (maxdiag) *maxdiag = md;
        DBuf<int64_t> dip, dind;
        DBuf<double> ddat;
        dip.upload(ip, s);
        dind.alloc(*nnz, s);
        ddat.alloc(*nnz, s);
        if (precision == FX_PREC_FP64) launch_bsr_to_csr<double>(d.S, d.vals64.ptr, dip.ptr, dind.ptr, ddat.ptr, s);
        else launch_bsr_to_csr<float>(d.S, d.vals32.ptr, dip.ptr, dind.ptr, ddat.ptr, s);
        std::memcpy(indptr, ip.data(), ip.size() * sizeof(int64_t));
        dind.download(indices, *nnz, s);
        ddat.download(data, *nnz, s);
        FX_CUDA_CHECK(cudaStreamSynchronize(s));
        return FX_OK;
    });
}

static int force_common(fx_model* m, const double* u, const double* uconf, double* f, bool thermal) {
    if (!m || !f || (!thermal && !u) || !m->state_ready) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        fx_ctx* ctx = m->ctx;
        int64_t* saved = g_launch_counter;
        g_launch_counter = &ctx->launches;
        struct R {
            int64_t* v;
            ~R() { g_launch_counter = v; }
        } r{saved};
        ensure_dense(m);
        if (m->dense.missing_node_id >= 0) fail_detail(FX_NODE_NOT_FOUND, m->dense.missing_node_error, -1, m->dense.missing_node_id, "");
        ensure_structure(m);
        cudaStream_t s = ctx->stream;
        const size_t n3 = 3 * (size_t)m->dense.n_nodes;
        DBuf<double> du, duc, out;
        out.alloc(n3, s);
        if (thermal) {
            compute_thermal_force(m, out.ptr);
        } else {
            du.upload(u, n3, s);
            if (uconf) duc.upload(uconf, n3, s);
            compute_internal_force(m, du.ptr, uconf ? duc.ptr : nullptr, out.ptr);
        }
        check_device_errors(m, thermal ? "thermal force" : "internal force");
        out.download(f, n3, s);
        FX_CUDA_CHECK(cudaStreamSynchronize(s));
        return FX_OK;
    });
}

int fx_internal_force(fx_model* m, const double* u, const double* uconf, double* f) {
    return force_common(m, u, uconf, f, false);
}

int fx_thermal_force(fx_model* m, double* f) { return force_common(m, nullptr, nullptr, f, true); }

int fx_model_drop_cache(fx_model* m) {
    if (!m || !m->ctx) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        ModelDev& d = m->dev;
        d.have_structure = false;
        d.S = BsrStructure();
        d.ebuf32.release();
        d.vals32.release();
        d.minv32.release();
        d.ebuf64.release();
        d.vals64.release();
        d.minv64.release();
        stream_wait(m->ctx->stream, "drop cache");
        return FX_OK;
    });
}

int fx_profile_spmv(fx_model* m, int precision, int reps, double* ms, double* bytes) {
    if (!m || !m->ctx || !ms || !bytes || reps <= 0 || !m->state_ready) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        int64_t* saved = g_launch_counter;
        g_launch_counter = &m->ctx->launches;
        struct R {
            int64_t* v;
            ~R() { g_launch_counter = v; }
        } r{saved};
        ensure_dense(m);
        if (m->dense.missing_node_id >= 0) fail_detail(FX_NODE_NOT_FOUND, m->dense.missing_node_error, -1, m->dense.missing_node_id, "");
        ensure_structure(m);
        *ms = precision == FX_PREC_MIXED ? profile_t<float>(m, reps, bytes) : profile_t<double>(m, reps, bytes);
        return FX_OK;
    });
}

int fx_profile_assembly(fx_model* m, int precision, int reps, double* stiff_ms, double* stiff_flops,
                        double* gather_ms, double* gather_bytes) {
    if (!m || !m->ctx || !stiff_ms || !stiff_flops || !gather_ms || !gather_bytes || reps <= 0 || !m->state_ready)
        return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        int64_t* saved = g_launch_counter;
        g_launch_counter = &m->ctx->launches;
        struct R {
            int64_t* v;
            ~R() { g_launch_counter = v; }
        } r{saved};
        ensure_dense(m);
        if (m->dense.missing_node_id >= 0)
            fail_detail(FX_NODE_NOT_FOUND, m->dense.missing_node_error, -1, m->dense.missing_node_id, "");
        ensure_structure(m);
        ModelDev& d = m->dev;
        cudaStream_t s = m->ctx->stream;
        const bool fp64 = precision != FX_PREC_MIXED;
        const size_t slots = (size_t)d.g4().n * kPairs4 + (size_t)d.g20().n * kPairs20;
        const size_t tsz = fp64 ? sizeof(double) : sizeof(float);
        auto stiff = [&] {
            if (fp64)
                launch_stiffness<double>(d.g4(), d.g20(), d.xyz.ptr, nullptr, d.tcur.ptr, d.mats.view(),
                                         m->ctx->tables.view(), d.ebuf64.ptr, d.maxdiag.ptr, d.err.ptr, s);
            else
                launch_stiffness<float>(d.g4(), d.g20(), d.xyz.ptr, nullptr, d.tcur.ptr, d.mats.view(),
                                        m->ctx->tables.view(), d.ebuf32.ptr, d.maxdiag.ptr, d.err.ptr, s);
        };
        auto gather = [&] {
            if (fp64) launch_bsr_gather<double>(d.S, d.ebuf64.ptr, d.vals64.ptr, s);
            else launch_bsr_gather<float>(d.S, d.ebuf32.ptr, d.vals32.ptr, s);
        };
        if (fp64) {
            d.ebuf64.alloc(slots * 9 + 9, s);
            d.vals64.alloc((size_t)d.S.n_groups * 36, s);
        } else {
            d.ebuf32.alloc(slots * 9 + 9, s);
            d.vals32.alloc((size_t)d.S.n_groups * 36, s);
        }
        d.maxdiag.zero(s);
        for (int k = 0; k < 2; ++k) {  // warm-up
            stiff();
            gather();
        }
        check_device_errors(m, "stiffness");
        EventTimer t;
        t.start(s);
        for (int k = 0; k < reps; ++k) stiff();
        *stiff_ms = t.stop_ms(s) / reps;
        t.start(s);
        for (int k = 0; k < reps; ++k) gather();
        *gather_ms = t.stop_ms(s) / reps;
        // declared FLOPs: 13,140 per Gauss point x 27 for C3D20 (D.B plus the symmetric upper
        // B^T (D B)), 900 per C3D4 element
        *stiff_flops = 354780.0 * d.g20().n + 900.0 * d.g4().n;
        // compulsory bytes of the gather: every element-pair block read once, the sorted slot
        // list (both orientations of every off-diagonal pair), the per-block segment offsets
        // and every 3x3 block written once
        *gather_bytes = (double)slots * 9.0 * tsz + 4.0 * (double)d.S.n_pairs +
                        (double)d.S.n_blocks * (8.0 + 9.0 * tsz);
        return FX_OK;
    });
}

int fx_profile_smoother(fx_model* m, int precision, int fp16, int reps, double* ms, double* bytes) {
    if (!m || !m->ctx || !ms || !bytes || reps <= 0 || !m->state_ready) return FX_INVALID_ARGUMENT;
    return guarded(m->ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(m->ctx->device));
        int64_t* saved = g_launch_counter;
        g_launch_counter = &m->ctx->launches;
        struct R {
            int64_t* v;
            ~R() { g_launch_counter = v; }
        } r{saved};
        ensure_dense(m);
        if (m->dense.missing_node_id >= 0) fail_detail(FX_NODE_NOT_FOUND, m->dense.missing_node_error, -1, m->dense.missing_node_id, "");
        ensure_structure(m);
        ModelDev& d = m->dev;
        cudaStream_t s = m->ctx->stream;
        assemble(m, nullptr, true);
        DBuf<double> minv;
        minv.alloc((size_t)m->dense.n_nodes * 9, s);
        launch_block_jacobi<double>(d.S, d.vals64.ptr, minv.ptr, s);
        *ms = profile_smoother_op(d.S, d.vals64.ptr, minv.ptr, precision == FX_PREC_MIXED, fp16 != 0, reps, s, bytes);
        return FX_OK;
    });
}

int fx_batch_solve(fx_ctx* ctx, fx_model* const* models, int n, const fx_solve_opts* opts, int* status,
                   fx_step_stats* stats) {
    if (!ctx || (!models && n)) return FX_INVALID_ARGUMENT;
    fx_solve_opts o;
    if (opts) o = *opts;
    else fx_default_solve_opts(&o);
    return guarded(ctx, [&] {
        FX_CUDA_CHECK(cudaSetDevice(ctx->device));
        return batch_solve(ctx, models, n, o, status, stats);
    });
}

}  // extern "C"
