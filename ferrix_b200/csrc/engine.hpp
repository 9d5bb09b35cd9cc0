// Context / model objects behind the C ABI and the device-resident static
// step driver.
#pragma once

#include <memory>
#include <new>
#include <string>
#include <vector>

#include "kernels.hpp"
#include "model.hpp"
#include "pcg.hpp"
#include "pcg_csr.hpp"
#include "amg.hpp"

struct fx_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    fx::DeviceTables tables;
    std::string last_error;
    fx::ErrorRecord last_detail;
    int preload_functions = -1;  // kernels loaded by fx_ctx_create on this device (-1: entry points missing)
    int64_t launches = 0;
    fx::PcgBatch<float> pcg32;
    fx::PcgBatch<double> pcg64;
    fx::CsrPcg pcgcsr;
    // fx_batch_solve's worker contexts on the same device (own streams; created at the first
    // batch, destroyed with this context, after its models)
    std::vector<fx_ctx*> workers;
};

namespace fx {

struct MatTableDev {
    DBuf<int32_t> e_off, e_len, nu_off, nu_len, a_off, a_len;
    DBuf<double> tref, t, v;
    int n_mat = 0;
    MatDev view() const {
        return MatDev{e_off.ptr, e_len.ptr, nu_off.ptr, nu_len.ptr, a_off.ptr, a_len.ptr, tref.ptr, t.ptr, v.ptr,
                      n_mat};
    }
};

// Penalty / mask / load data of one step, merged per DOF on the host.
struct StepBc {
    std::vector<int32_t> dof;            // unique constrained DOFs, ascending
    std::vector<double> cnt;             // records per DOF
    std::vector<std::vector<int>> recs;  // record indices per DOF (for target sums)
    DBuf<int32_t> d_dof;
    DBuf<double> d_cnt, d_usum;
    DBuf<uint8_t> d_mask;
};

struct ModelDev {
    bool uploaded = false;
    DBuf<double> xyz, tinit, tcur;
    DBuf<int32_t> conn4, conn20, mat4, mat20;
    MatTableDev mats;
    bool have_structure = false;
    BsrStructure S;
    DBuf<float> ebuf32, vals32, minv32;
    DBuf<double> ebuf64, vals64, minv64;
    DBuf<double> fe, u, ustart, du, fext, ftmp, fint, R, r64, ax;
    bool u_zero = false;  // u is all zeros: set by the state reset, cleared by every other write of u
    DBuf<unsigned long long> maxdiag;
    DBuf<int> err;
    DBuf<double> norm_part, norm_out;
    DBuf<int32_t> load_dof;
    DBuf<double> load_val;
    // the model's multigrid hierarchy and CG workspace (kept between Newton iterations,
    // whose values are refreshed on it, and across steps until the structure changes)
    std::unique_ptr<AmgPcg> amg;
    ElemView g4() const { return ElemView{(int)conn4.n / 4, conn4.ptr, mat4.ptr}; }
    ElemView g20() const { return ElemView{(int)conn20.n / 20, conn20.ptr, mat20.ptr}; }
};

}  // namespace fx

struct fx_model {
    fx_ctx* ctx = nullptr;
    fx::Project project;
    fx::DenseModel dense;
    bool dense_built = false;
    bool state_ready = false;
    std::vector<double> t_init, t_cur;  // SolutionState temperatures
    fx::SolverTime timer;
    fx::ModelDev dev;
};

namespace fx {
// The calling thread's last failure (entry points called without a context,
// e.g. fx_model_from_inp with ctx NULL, report here only).
ErrorRecord& thread_error();
}  // namespace fx

// Runs an entry point's body: fx::Error and standard exceptions become status
// codes, with the message stored as the context's last error and the message
// and payload as the context's and the thread's last error detail.
template <typename F>
inline int guarded(fx_ctx* ctx, F&& f) {
    auto record = [&](const fx::Error& e) {
        fx::thread_error().set(e);
        if (ctx) {
            ctx->last_error = e.what();
            ctx->last_detail.set(e);
        }
        return e.status;
    };
    try {
        return f();
    } catch (const fx::Error& e) {
        return record(e);
    } catch (const std::bad_alloc&) {
        return record(fx::Error(FX_GENERIC, "Generic error: host allocation failed"));
    } catch (const std::exception& e) {
        return record(fx::Error(FX_GENERIC, e.what()));
    }
}

namespace fx {

void ensure_dense(fx_model* m);
// One kernel of each source file's module, and the loading of every kernel of
// those modules on the current device (once per device and process): with lazy
// module loading, a kernel's first launch would otherwise wait for the kernels
// running on other streams.
const void* kernels_anchor_amg();
const void* kernels_anchor_amg_cluster();
const void* kernels_anchor_assembly();
const void* kernels_anchor_csr_solve();
const void* kernels_anchor_elements();
const void* kernels_anchor_noalloc();
const void* kernels_anchor_pcg();
const void* kernels_anchor_pcg_csr();
const void* kernels_anchor_vectors();
int preload_kernels(int device);
// Device bytes of one model while it is solved (an upper estimate), and the
// spare pool memory held for it (with slack for fragmentation).
double model_footprint(const DenseModel& D);
double model_slack(const DenseModel& D);
// Grows the device's stream-ordered memory pool (which keeps what it holds) so
// that it has `bytes` more than it has in use, by one allocation queued on `s`
// and freed again, before the caller queues any work. Best effort: a failed
// allocation leaves the pool as it was. Returns 1 when the pool grew, 0 when it
// already held enough, -1 when it could not grow (it then grows on demand).
int reserve_pool(int device, cudaStream_t s, double bytes);
// Bytes the device's memory pool holds (reserved), -1 when it cannot be read.
double pool_reserved_bytes(int device);
void upload_model(fx_model* m);
void ensure_structure(fx_model* m);
void state_initialize(fx_model* m);
// element loops
void compute_internal_force(fx_model* m, const double* d_u, const double* d_uconf, double* d_out);
void compute_thermal_force(fx_model* m, double* d_out);
// assembles K (precision) at X (+d_u) into dev.vals32/vals64; returns maxdiag (host copy)
double assemble(fx_model* m, const double* d_u, bool fp64);
void check_device_errors(fx_model* m, const char* where);
int step_solve(fx_model* m, int step_index, const fx_solve_opts& opts, fx_step_stats* stats,
               fx_increment_cb cb = nullptr, void* user = nullptr);
int batch_solve(fx_ctx* ctx, fx_model* const* models, int n, const fx_solve_opts& opts, int* status,
                fx_step_stats* stats);

}  // namespace fx
