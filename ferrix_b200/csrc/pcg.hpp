// Batched preconditioned conjugate gradient over BSR(3x3) systems.
//
// Stands in for the reference's DirectSolver (src/solver/solvers/direct.rs:19-55,
// an FP64 sparse Cholesky) and IterativeSolver (src/solver/solvers/iterative.rs:26-136,
// a Jacobi-PCG): both solve K du = R; this solver returns du to a stated
// tolerance on the FP64 true residual.
//
// Mixed precision (T = float): the SpMV, the 3x3 block-Jacobi and the vector
// recurrences run in FP32 while the solution is accumulated in FP64 and the
// residual is periodically replaced by the FP64 true residual b - A x
// (residual replacement / "reliable updates", van der Vorst & Ye 2000),
// computed by a caller-supplied FP64 operator. This is the FP64
// iterative-refinement loop around the FP32 Krylov iteration, without
// discarding the search direction at each refinement.
// FP64 (T = double): the same kernels on FP64 data; the true residual is
// checked once at the end.
//
// Per iteration three kernels run per batch: (C) p = z + beta p, (A) q = K p with
// the p.q partial sum (one gathered vector, four values per node), (B)
// x += alpha p, r -= alpha q, z = M r and the r.z partial sum. Scalars are
// reduced by the last CTA of each system in a fixed order (deterministic).
// A block of `poll_interval` iterations is captured in a CUDA graph and
// replayed between host checks.
#pragma once

#include <algorithm>
#include <functional>
#include <vector>

#include "kernels.hpp"

namespace fx {

enum PcgStatus : int { kRun = 0, kConv = 1, kBreak = 2, kIdle = 3 };

// scalars per system
enum PcgScal : int {
    kRz = 0, kPq = 1, kAlpha = 2, kBeta = 3, kRzOld = 4, kRr = 5, kRzRef = 6, kIters = 7, kThresh = 8,
    kRz64 = 9, kBnorm = 10, kNScal = 16
};

template <typename T>
struct InstDev {
    int n_rows;
    int chunk0, nchunks;
    const int32_t* goff;
    const int32_t* cols;
    const T* vals;
    const T* minv;
    T *r, *q;          // three per node
    T *z, *p0;         // four per node (the fourth is padding): one vector load per gathered node
    double* x;
    const double* r64;
    double* scal;
    int* status;
    int* counter;
    double* part;
};

struct ChunkDev {
    int inst, row0, row1, pad;
};

// One linear system of a batch.
template <typename T>
struct PcgSystem {
    const BsrStructure* S = nullptr;
    const T* vals = nullptr;
    const T* minv = nullptr;
    const double* b = nullptr;  // FP64 right-hand side (device)
    double* x = nullptr;        // FP64 solution (device), overwritten
    // r64 = b - A x in FP64 (device pointers); the FP64 operator of this system
    std::function<void(const double* x, const double* b, double* r64, cudaStream_t)> residual64;
    bool warm_start = false;    // start from the given x (r0 = b - A x by residual64) instead of x = 0
    double bnorm2 = 0.0;        // warm start: ||b||_M^2 that rtol refers to (0: the starting residual's)
    // outputs
    int status = 0;
    bool stagnated = false;     // mixed: FP64 residual stopped improving across replacements
    long long iterations = 0;
    int replacements = 0;
    double relres = 0.0;  // final ||b - A x||_M / ||b||_M
    double bnorm2_seen = 0.0;  // the ||.||_M^2 this solve measured its residual against
};

// Multigrid defaults, from a sweep on the 417k-DOF C3D20 box (136 -> 100 CG
// iterations) and a population of C3D4 / C3D20 boxes (13 % less time):
// coarse corrections scaled by 1.7 (aggregation without prolongator smoothing
// under-corrects), first-kind Chebyshev on [lmax / 12, lmax].
constexpr double kAmgOvercorrect = 1.7;
constexpr double kAmgChebRatio = 12.0;

// Mixed block-Jacobi PCG: FP64 true-residual target as a fraction of the
// caller's rtol. Its FP32 Krylov recurrence leaves a residual whose smooth
// (low-eigenvalue) components are larger than those FP64 CG leaves at the same
// residual norm, so its displacement error at rtol = 1e-8 reached 2e-9 on the
// 417k-DOF C3D20 box and exceeded 1e-8 on thin random boxes, where FP64 PCG
// stays below; a residual 100x smaller keeps the mixed displacement error within
// the rtol that the caller asked for.
constexpr double kMixedBjResidualFactor = 1e-2;

struct PcgOptions {
    double rtol = 1e-10;
    int max_iter = 20000;
    int poll = 32;
    double reliable_delta = 1e-2;
    bool graphs = true;
    int stall_limit = 4;  // replacements without halving the best FP64 residual before giving up (mixed)
    int replace_every = 512;  // mixed: FP64 residual replacement at least this often (iterations)
    int stall_iters = 2048;   // mixed: give up on FP32 when the FP64 residual has not halved for this long
    // FP64 finish of a mixed solve: rtol is the tightened target; once the FP64 true residual
    // stops improving (stall_limit replacements without halving) at or below accept_rtol (the
    // caller's own tolerance), the solve ends converged (0: no such acceptance)
    double accept_rtol = 0.0;
    // multigrid preconditioner
    int amg_degree = 2;       // Chebyshev smoothing steps per pre/post smoothing
    bool amg_fp32 = false;    // FP32 fine-matrix values in the level-0 smoother
    bool amg_kcycle = false;  // K-cycle at the first coarse level (flexible outer CG)
    int amg_cheb_kind = 0;    // 0: Chebyshev of the first kind on [lmax/ratio, lmax], 1: fourth kind
    double amg_overcorrect = kAmgOvercorrect;  // scale of every coarse correction
    double amg_cheb_ratio = kAmgChebRatio;  // lmax / lmin of the first-kind Chebyshev interval
    int64_t amg_persistent_max_dof = 0;     // systems up to this size: one persistent cluster launch (< 0: never)
    bool amg_fused_coarse = true;           // coarse part of each V-cycle as one cooperative launch
    bool amg_fp16 = false;                  // level-0 smoothing with FP16 values of the scaled matrix
};

template <typename T>
class PcgBatch {
   public:
    // Solves all systems; returns FX_OK or the first failing status (per-system status in sys[i].status).
    int solve(std::vector<PcgSystem<T>*>& sys, const PcgOptions& opt, cudaStream_t s, int64_t* launches);
    // Mean duration (ms) of one standalone launch of the fused SpMV kernel on this system.
    double profile_spmv(PcgSystem<T>& sys, int reps, cudaStream_t s);

   private:
    void prepare(std::vector<PcgSystem<T>*>& sys, cudaStream_t s, std::vector<ChunkDev>& chunks,
                 std::vector<int>& chunk0, std::vector<int>& nch);
    int64_t spmv_resident();
    unsigned spmv_grid(size_t nchunks) { return (unsigned)std::min<int64_t>((int64_t)nchunks, spmv_resident()); }
    int64_t resident_ = 0;
    struct Work {
        DBuf<T> r, z, p0, q;
        DBuf<double> r64;
    };
    std::vector<Work> work_;
    DBuf<InstDev<T>> d_inst_;
    DBuf<ChunkDev> d_chunks_;
    DBuf<double> d_scal_, d_part_;
    DBuf<int> d_status_, d_counter_;
};

}  // namespace fx
