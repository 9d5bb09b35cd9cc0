// Aggregation multigrid preconditioner for the stiffness systems (3 DOF per
// node), used inside PCG in place of the 3x3 block-Jacobi preconditioner.
//
// Hierarchy (setup, all on the GPU, deterministic):
//   * aggregation by spatial binning of the level's points (nodes, then
//     aggregate centroids) into cubic cells;
//   * tentative prolongator from the six rigid-body modes (three translations,
//     three rotations about the aggregate centroid): per aggregate a QR of the
//     stacked near-null-space rows (one warp per aggregate, modified
//     Gram-Schmidt applied twice); Q gives the prolongator rows, R the next
//     level's near-null-space (Vanek, Mandel & Brezina 1996, without the
//     prolongator smoothing step);
//   * Galerkin coarse matrix A_c = Q^T A Q: fine blocks are sorted by their
//     (aggregate, aggregate) key and every coarse 6x6 block sums Q_i^T A_ij Q_j
//     over its fine blocks in a fixed order (no atomics);
//   * Chebyshev smoothing of degree 2 on D^-1 A (D = block diagonal) with the
//     largest eigenvalue from power iteration; dense inverse at the coarsest
//     level.
// Application: one V-cycle per PCG iteration.
#pragma once

#include <cuda_fp16.h>

#include <vector>

#include "kernels.hpp"
#include "pcg.hpp"

namespace fx {

// State of the software grid barrier of the cooperative coarse-cycle launch (zeroed
// before a solve; a wait that ran out leaves it inconsistent until then).
struct GridBarState {
    unsigned int count, gen;
};

struct ClInst;

struct AmgLevel {
    int n = 0;   // block rows (nodes at level 0, aggregates above)
    int bs = 3;  // block size
    // level 0 matrix: the planar BSR3 of the fine system
    const BsrStructure* S0 = nullptr;
    const double* vals0 = nullptr;
    const double* dinv0 = nullptr;  // 3x3 block inverses of the fine diagonal (block-Jacobi)
    // coarse levels: row-major block CSR, blocks of bs x bs
    DBuf<int32_t> row_ptr, cols;
    DBuf<double> vals, dinv;
    int64_t nblocks = 0;
    double lmax = 0.0;
    // transfer to the next level
    DBuf<int32_t> agg;                 // aggregate of each block row
    DBuf<double> Q;                    // n * bs * 6 prolongator rows
    DBuf<int32_t> agg_ptr, agg_nodes;  // members of each aggregate
    int n_agg = 0;
    // work vectors (n * bs); xs: pre-smoothed iterate of the coarse-level cycle
    DBuf<double> x, b, r, d, t, xs;
    // fine level with FP32 smoother values: directions and the iterate as float4 per node
    DBuf<float> d4a, d4b, x4;
    // coarsest level: dense inverse (n*bs)^2
    bool coarsest = false;
    DBuf<double> dense_inv;
    // K-cycle work vectors (first coarse level): z1, v1, r, z2, v2 and scalars
    DBuf<double> kc[5], kcs;
    // Galerkin map to the next level (kept for refresh): the fine blocks sorted by
    // coarse block, each coarse block's segment of them, and (levels > 0) the row
    // of every fine block
    DBuf<int64_t> gal_seg, gal_blk;
    DBuf<int32_t> gal_rows;
    // last power-iteration vector of the eigenvalue estimate (start of the next refresh's)
    DBuf<double> ev;
    const double* dinv_ptr() const { return S0 ? dinv0 : dinv.ptr; }
};

struct AmgStats {
    int levels = 0;
    std::vector<int> sizes;   // DOF per level
    double setup_ms = 0.0;
};

// First smoothing step of a coarse level, done by the restriction kernel into it.
struct CoarseStart {
    const double* dinv;  // 6x6 block inverses of the coarse level
    double *r, *d, *xs;
    double c2;
};

class Amg {
   public:
    // xyz: FP64 node coordinates (device, 3 per node); dinv0: fine 3x3 block inverses.
    void setup(const BsrStructure& S0, const double* vals0, const double* dinv0, const double* xyz, int n_nodes,
               double cell0, cudaStream_t s, AmgStats* st);
    // New matrix values on the structure of the last setup: aggregates, prolongators
    // and coarse patterns are kept; coarse values, block inverses, eigenvalue
    // estimates and the coarsest inverse are recomputed.
    void refresh(const double* vals0, const double* dinv0, cudaStream_t s, AmgStats* st);
    uint64_t built_for = 0;  // BsrStructure::id of the last setup (0: none)
    // Smoother settings: Chebyshev degree (1..8) and, when vals_f32 is not null,
    // FP32 values of the fine matrix for the level-0 smoothing (FP64 vectors).
    void set_smoother(int degree, const float* vals_f32) {
        degree_ = degree;
        vals0_f32_ = vals_f32;
        vals0_f16_ = nullptr;
        sq4_ = nullptr;
    }
    // FP16 values of the scaled fine matrix S A S (S = diag(a_ii)^-1/2) and sqrt(a_ii) per
    // node for the level-0 smoothing steps, in place of FP32 values (null: off)
    void set_smoother_f16(const __half* vals16, const float4* sq4) {
        vals0_f16_ = vals16;
        sq4_ = sq4;
    }
    // FP16 smoother directions: where the V-cycle started from x = 0 finds r.D^-1 r of its
    // right-hand side (rdr) and the two floats where each V-cycle publishes its power-of-two
    // scale of the stored directions (hs); null: unscaled
    void set_smoother_scale(const double* rdr, float* hs) {
        rdr_ = rdr;
        hs_ = hs;
    }
    // K-cycle at the first coarse level (true) or V-cycles throughout.
    void set_cycle(bool kcycle) { kcycle_ = kcycle; }
    // Chebyshev smoother: 0 = first kind on [lmax/30, lmax], 1 = fourth kind
    void set_smoother_kind(int kind) { cheb_kind_ = kind; }
    // coarse corrections x += alpha P e; first-kind Chebyshev interval [lmax / ratio, lmax]
    void set_overcorrect(double alpha) { alpha_ = alpha; }
    void set_cheb_ratio(double ratio) { cheb_ratio_ = ratio; }
    bool kcycle() const { return kcycle_; }
    // z = cycle(r), FP64 vectors of 3 * n_nodes. With S != null the last
    // smoothing step also reduces r.z (and r.zold when zold != null, for the
    // flexible CG) into the outer CG scalars (S[0], S[4]).
    // started: the level-0 start (r0 = b, x = d = c2 D^-1 b) was done by the caller, into start0()
    void apply(const double* r, double* z, double* S, double* part, int* counter, const double* zold,
               cudaStream_t s, bool started = false);
    // slots of the `part` buffer apply() reduces into (two per CTA of the reducing launch)
    void set_part_slots(int64_t n) { part_slots_ = n; }
    // where the level-0 start writes: the smoother's residual, iterate and first direction
    // (FP32 float4 per node when the smoother is FP32, else FP64), and its coefficient
    struct Start0 {
        double *r, *x, *d;
        float4* d4;
        double c2;
        const float4* sq4;  // FP16 smoother: the float4 direction is written scaled by sqrt(a_ii)
        float* hs;          // FP16 directions: where the start publishes the V-cycle's scale (else null)
    };
    Start0 start0() const;
    // the hierarchy, smoother coefficients and work vectors, for the persistent solve
    void describe(ClInst& out) const;
    // The coarse part of each V-cycle as one cooperative launch (on: after every setup /
    // refresh the hierarchy's descriptor is uploaded; flag = where a barrier timeout is
    // reported) or as one launch per coarse-level step (off).
    void set_fused_coarse(bool on, double* flag) {
        fused_coarse_ = on;
        gflag_ = flag;
    }
    void upload_descriptor(cudaStream_t s);
    int degree() const { return degree_; }
    double overcorrect() const { return alpha_; }
    std::vector<AmgLevel> L;

   private:
    // started: the restriction into this level already did the first smoothing step
    void cycle(int l, const double* b, double* x, cudaStream_t s, bool started = false);
    // the start that the restriction into level m does (dinv null: none)
    CoarseStart coarse_start(int m) const;
    void coarse(int m, cudaStream_t s);
    void coarsest_inverse(AmgLevel& l, cudaStream_t s);
    template <typename VT>
    void vcycle0(const VT* vals, const double* b, double* z, double* S, double* part, int* counter,
                 const double* zold, cudaStream_t s, bool started);
    bool kcycle_ = false;
    int64_t part_slots_ = 0;
    int cheb_kind_ = 0;
    double alpha_ = 1.0, cheb_ratio_ = 30.0;
    int degree_ = 2;
    const float* vals0_f32_ = nullptr;
    const __half* vals0_f16_ = nullptr;
    const float4* sq4_ = nullptr;
    const double* rdr_ = nullptr;
    float* hs_ = nullptr;
    float* h16_scale_slot() const;
    bool fused_coarse_ = false;
    double* gflag_ = nullptr;
    DBuf<ClInst> desc_;
    DBuf<GridBarState> gbar_;
    DBuf<uint8_t> tmp_;
    DBuf<double> red_;  // reduction scratch
};

// ---- persistent solve of small systems (amg_cluster.cu)
// The whole multigrid-preconditioned CG of one system runs inside one thread-block
// cluster: every CG step and V-cycle phase is a loop over the cluster's threads,
// phases are separated by hardware cluster barriers, dot products are summed per
// CTA and across the cluster through distributed shared memory in a fixed order.
// One launch advances any number of systems (one cluster each); a system's
// arithmetic does not depend on the others, so it is the same alone and in a batch.
constexpr int kClMaxLevels = 8;

struct ClLevel {  // coarse level m >= 1 (6x6 blocks) and its transfer to level m + 1
    int n = 0, coarsest = 0, n_agg = 0;
    const int32_t *row_ptr = nullptr, *cols = nullptr;
    const double *vals = nullptr, *dinv = nullptr, *dense_inv = nullptr;
    const int32_t *agg = nullptr, *agg_ptr = nullptr, *agg_nodes = nullptr;
    const double* Q = nullptr;
    double *x = nullptr, *b = nullptr, *r = nullptr, *d = nullptr, *t = nullptr, *xs = nullptr;
    double c2_start = 0.0, c1[8] = {}, c2[8] = {};
};

struct ClInst {
    int n = 0, levels = 0;
    // level 0: planar BSR3 (FP64 values; FP32 copy for the smoother or null), 3x3 block inverses
    const int32_t *goff = nullptr, *cols = nullptr;
    const double* vals64 = nullptr;
    const float* vals32 = nullptr;
    const double* dinv0 = nullptr;
    const float4* sq4 = nullptr;  // FP16 smoother: the FP32 iterate copy is scaled by sqrt(a_ii)
    const int32_t *agg = nullptr, *agg_ptr = nullptr, *agg_nodes = nullptr;
    const double* Q = nullptr;
    int n_agg = 0;
    double *lr = nullptr, *lx = nullptr, *ld = nullptr, *lt = nullptr;
    float *d4a = nullptr, *d4b = nullptr, *x4 = nullptr;
    double c2_start = 0.0, c1[8] = {}, c2[8] = {};
    // the CG: right-hand side, iterate and work vectors (3n each)
    const double* b = nullptr;
    double *x = nullptr, *r = nullptr, *z = nullptr, *p = nullptr, *q = nullptr;
    ClLevel lev[kClMaxLevels];
};

struct ClResult {
    long long iterations;
    int status;  // FX_OK, FX_NUMERICAL (breakdown), FX_CONVERGENCE (max_iter)
    int pad;
    double rzd, bd;  // r.D^-1 r at the end and b.D^-1 b
};

// Launches the persistent solve of `n` systems (descriptors and results in device
// memory); fp32: level-0 smoothing with the FP32 values. Smoother degree 1..8,
// coarse corrections scaled by alpha.
void launch_amg_cluster(const ClInst* insts, ClResult* res, int n, bool fp32, double rtol, int max_iter, int degree,
                        double alpha, cudaStream_t s);
// The coarse part of one V-cycle (restriction from the level-0 residual, coarse
// levels, prolongation into the level-0 iterate) of the system `inst` describes,
// as one cooperative launch over all SMs; *flag = 1 when a barrier wait ran out.
void launch_coarse_grid(const ClInst* inst, GridBarState* st, double* flag, bool fp32, int degree, double alpha,
                        cudaStream_t s);
// Systems of at most this many DOF are solved by the persistent launch by default, alone
// or in a batch. Alone, a cluster is slower than the multi-launch path from about 3,600 DOF
// on (3.9 ms against 3.3 ms there, 17 ms against 7 ms at 15k DOF); in a batch of 64 C3D4
// decks of 2k-60k DOF spread over four worker streams, one persistent launch per worker
// took 243-324 ms against 183 ms for the multi-launch path on every stream (B200).
constexpr int64_t kClDefaultMaxDof = 2000;

// CG on the FP64 BSR3 system preconditioned by one V-cycle per iteration.
// CUDA-event time (ms per launch) of the fused fine-level Chebyshev step (SpMV +
// smoother update) on the given FP64 system, with FP32 values when fp32; bytes =
// compulsory traffic of one launch.
double profile_smoother_op(const BsrStructure& S, const double* vals64, const double* dinv64, bool fp32, bool fp16,
                           int reps,
                           cudaStream_t s, double* bytes);

class AmgPcg {
   public:
    // For the persistent solve: set up (or refresh) the hierarchy for the system and
    // allocate the CG vectors, without iterating; then describe it for the kernel.
    void prepare(const BsrStructure& S, const double* vals64, const double* dinv64, const double* xyz, double cell0,
                 const PcgOptions& opt, cudaStream_t s, AmgStats* st, bool reuse, bool persistent = false);
    ClInst describe(const double* b, double* x) const;
    // ||b - A x||_D / ||b||_D of the assembled FP64 system after a persistent solve
    double true_relres(const double* b, const double* x, cudaStream_t s);
    // reuse: keep the hierarchy's aggregates, prolongators and coarse patterns when
    // the last setup was on the same structure S (only the values are refreshed)
    int solve(const BsrStructure& S, const double* vals64, const double* dinv64, const double* xyz, double cell0,
              const double* b, double* x, const PcgOptions& opt, cudaStream_t s, int64_t* launches, long long* iters,
              double* relres, AmgStats* st, bool reuse = false);
    Amg amg;

   private:
    const BsrStructure* S_ = nullptr;
    const double* vals64_ = nullptr;
    const double* dinv64_ = nullptr;
    DBuf<double> r_, z_, z2_, p_, q_, part_, sc_;
    DBuf<float> vals32_;
    DBuf<__half> vals16_;
    DBuf<float4> sq4_;
    DBuf<float> hs_;  // FP16 smoother directions: the current V-cycle's {2^k, 2^-k}
    DBuf<int> counter_;
};

}  // namespace fx
