// Batched BSR3 PCG kernels and host loop (see pcg.hpp).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "pcg.hpp"

namespace fx {

constexpr int kChunkRows = 256;   // rows per CTA work item
constexpr int kSpmvThreads = 256; // 32 rows per pass, 8 lanes per row
constexpr int kUpdThreads = 256;  // one row per thread

__device__ __forceinline__ void ld4(const float* p, int64_t i4, float o[4]) {
    float4 v = __ldcs(reinterpret_cast<const float4*>(p) + i4);
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
}
__device__ __forceinline__ void ld4(const double* p, int64_t i4, double o[4]) {
    const double2* q = reinterpret_cast<const double2*>(p) + 2 * i4;
    double2 a = __ldcs(q), b = __ldcs(q + 1);
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b.x;
    o[3] = b.y;
}

// The three components of node j of a vector stored four per node (the fourth is
// padding), in one 16-byte load (FP32) or two (FP64).
__device__ __forceinline__ void ld_node(const float* v, int64_t j, float o[3]) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(v) + j);
    o[0] = t.x;
    o[1] = t.y;
    o[2] = t.z;
}
__device__ __forceinline__ void ld_node(const double* v, int64_t j, double o[3]) {
    const double2 a = __ldg(reinterpret_cast<const double2*>(v) + 2 * j);
    const double b = __ldg(v + 4 * j + 2);
    o[0] = a.x;
    o[1] = a.y;
    o[2] = b;
}

// Fixed-order block reduction of NV doubles; result valid in thread 0.
template <int NV>
__device__ __forceinline__ void block_sum(double v[NV], double* sh /* [NV][32] */) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (l == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k * 32 + w] = v[k];
    __syncthreads();
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double t = 0.0;
            for (int j = 0; j < nw; ++j) t += sh[k * 32 + j];
            v[k] = t;
        }
}

// Publish this CTA's partials; returns true in every thread of the CTA that
// completes the system (then `tot` holds the fixed-order totals in thread 0).
template <int NV>
__device__ __forceinline__ bool last_cta_reduce(double v[NV], double* part, int chunk_id, int chunk0, int nchunks,
                                                int* counter, double* sh, double tot[NV]) {
    __shared__ int s_last;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) part[(int64_t)chunk_id * 4 + k] = v[k];
        __threadfence();
        int t = atomicAdd(counter, 1);
        s_last = (t == nchunks - 1);
    }
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    for (int c = threadIdx.x; c < nchunks; c += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) acc[k] += __ldcg(part + (int64_t)(chunk0 + c) * 4 + k);
    __syncthreads();
    block_sum<NV>(acc, sh);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) tot[k] = acc[k];
        *counter = 0;
    }
    return true;
}

// Status read once per CTA and broadcast, so every thread of a CTA takes the same path.
__device__ __forceinline__ bool cta_running(const int* status) {
    __shared__ int s_st;
    if (threadIdx.x == 0) s_st = *(volatile const int*)status;
    __syncthreads();
    return s_st == kRun;
}

// (C) p = z + beta p (four per node), a light pass before the SpMV so that the SpMV
// gathers one vector.
template <typename T>
__global__ void __launch_bounds__(kUpdThreads) k_pcg_dir(const ChunkDev* __restrict__ chunks,
                                                         const InstDev<T>* __restrict__ insts) {
    const ChunkDev ck = chunks[blockIdx.x];
    const InstDev<T> I = insts[ck.inst];
    if (!cta_running(I.status)) return;
    const T beta = (T)I.scal[kBeta];
    for (int row = ck.row0 + threadIdx.x; row < ck.row1; row += blockDim.x)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int64_t at = 4 * (int64_t)row + c;
            I.p0[at] = I.z[at] + beta * I.p0[at];
        }
}

// (A) q = K p, partial p . q, alpha = r.z / p.q.
// Persistent CTAs walk the chunk list (chunk c, c + gridDim.x, ...); in a chunk,
// 8 lanes share a block row (32 rows per pass) and each lane keeps two column
// groups in flight, gathering one 16-byte (FP32) node vector per column; with FP32
// values each 4-block group is summed in FP32 and added to the FP64 row sums.
// 256-thread CTAs, two per SM (at most 128 registers).
template <typename T>
__global__ void __launch_bounds__(kSpmvThreads, 2) k_pcg_spmv(const ChunkDev* __restrict__ chunks, int nchunks,
                                                             const InstDev<T>* __restrict__ insts) {
    __shared__ double sh[4 * 32];
    const int sub = threadIdx.x & 7, grp = threadIdx.x >> 3;
    for (int ci = blockIdx.x; ci < nchunks; ci += gridDim.x) {
        const ChunkDev ck = chunks[ci];
        const InstDev<T> I = insts[ck.inst];
        if (!cta_running(I.status)) continue;  // CTA-uniform
        const T* __restrict__ p = I.p0;
        double dot = 0.0;
        const int nrows = ck.row1 - ck.row0;
        // The trip count is uniform across the CTA so that every lane reaches the
        // full-warp shuffles below; lanes past the chunk end carry zeros.
        for (int base = 0; base < nrows; base += kSpmvThreads / 8) {
            const bool valid = base + grp < nrows;
            const int row = ck.row0 + (valid ? base + grp : 0);
            const int g0 = valid ? I.goff[row] : 0;
            const int ng = valid ? I.goff[row + 1] - g0 : 0;
            const int c = sub < 3 ? sub : 0;
            T pc = 0;
            if (valid && sub < 3) pc = __ldg(p + 4 * (int64_t)row + c);  // ahead of the gathers
            double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll 2
            for (int g = sub; g < ng; g += 8) {
                const int4 cc = __ldg(reinterpret_cast<const int4*>(I.cols) + g0 + g);
                const int cj[4] = {cc.x, cc.y, cc.z, cc.w};
                T xv[4][3];
#pragma unroll
                for (int q = 0; q < 4; ++q) ld_node(p, cj[q], xv[q]);
                const int64_t pl = (int64_t)ng;
                const int64_t vb = (int64_t)g0 * 9 + g;
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    T m0[4], m1[4], m2[4];
                    ld4(I.vals, vb + (3 * r) * pl, m0);
                    ld4(I.vals, vb + (3 * r + 1) * pl, m1);
                    ld4(I.vals, vb + (3 * r + 2) * pl, m2);
                    T t = 0;
#pragma unroll
                    for (int q = 0; q < 4; ++q) t += m0[q] * xv[q][0] + m1[q] * xv[q][1] + m2[q] * xv[q][2];
                    acc[r] += (double)t;
                }
            }
#pragma unroll
            for (int o = 4; o > 0; o >>= 1)
#pragma unroll
                for (int r = 0; r < 3; ++r) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
            if (valid && sub < 3) {
                const T qc = (T)(c == 0 ? acc[0] : (c == 1 ? acc[1] : acc[2]));
                I.q[3 * (int64_t)row + c] = qc;
                dot += (double)pc * (double)qc;
            }
        }
        double v[1] = {dot}, tot[1];
        block_sum<1>(v, sh);
        __syncthreads();
        if (last_cta_reduce<1>(v, I.part, ck.pad, I.chunk0, I.nchunks, I.counter, sh, tot) && threadIdx.x == 0) {
            double pq = tot[0];
            I.scal[kPq] = pq;
            if (!(pq > 0.0) || !isfinite(pq)) {
                *I.status = kBreak;
                I.scal[kAlpha] = 0.0;
            } else {
                I.scal[kAlpha] = I.scal[kRz] / pq;
            }
        }
        __syncthreads();  // shared partials and s_last are reused by the next chunk
    }
}

// (B) x += alpha p, r -= alpha q, z = M r, partial r.z and r.r
template <typename T>
__global__ void __launch_bounds__(kUpdThreads) k_pcg_update(const ChunkDev* __restrict__ chunks,
                                                            const InstDev<T>* __restrict__ insts) {
    __shared__ double sh[4 * 32];
    const ChunkDev ck = chunks[blockIdx.x];
    const InstDev<T> I = insts[ck.inst];
    if (!cta_running(I.status)) return;
    const double alpha = I.scal[kAlpha];
    const T* __restrict__ p = I.p0;
    double rz = 0.0, rr = 0.0;
    for (int row = ck.row0 + threadIdx.x; row < ck.row1; row += blockDim.x) {
        const int r3 = 3 * row;
        T r[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T pc = p[4 * (int64_t)row + c];
            I.x[r3 + c] += alpha * (double)pc;
            r[c] = I.r[r3 + c] - (T)alpha * I.q[r3 + c];
            I.r[r3 + c] = r[c];
        }
        const T* m = I.minv + 9 * (int64_t)row;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T zc = m[3 * c] * r[0] + m[3 * c + 1] * r[1] + m[3 * c + 2] * r[2];
            I.z[4 * (int64_t)row + c] = zc;
            rz += (double)r[c] * (double)zc;
            rr += (double)r[c] * (double)r[c];
        }
    }
    double v[2] = {rz, rr}, tot[2];
    block_sum<2>(v, sh);
    __syncthreads();
    if (last_cta_reduce<2>(v, I.part, ck.pad, I.chunk0, I.nchunks, I.counter + 1, sh, tot) && threadIdx.x == 0) {
        double rzn = tot[0];
        double rzo = I.scal[kRz];
        I.scal[kRzOld] = rzo;
        I.scal[kRz] = rzn;
        I.scal[kRr] = tot[1];
        I.scal[kBeta] = rzo > 0.0 ? rzn / rzo : 0.0;
        I.scal[kIters] += 1.0;
        if (!isfinite(rzn) || rzn < 0.0) *I.status = kBreak;
        else if (rzn <= I.scal[kThresh]) *I.status = kConv;
    }
}

// Residual (re)placement: r = (T) r64, z = M r, r.z; FP64 r64 . M r64.
// first != 0: start of a solve (beta = 0, ||b||_M^2 and the stop threshold recorded).
template <typename T>
__global__ void __launch_bounds__(kUpdThreads) k_pcg_replace(const ChunkDev* __restrict__ chunks,
                                                             const InstDev<T>* __restrict__ insts, int first,
                                                             double rtol2) {
    __shared__ double sh[4 * 32];
    const ChunkDev ck = chunks[blockIdx.x];
    const InstDev<T> I = insts[ck.inst];
    double rz = 0.0, rz64 = 0.0;
    for (int row = ck.row0 + threadIdx.x; row < ck.row1; row += blockDim.x) {
        const int r3 = 3 * row;
        double r64[3];
        T r[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            r64[c] = I.r64[r3 + c];
            r[c] = (T)r64[c];
            I.r[r3 + c] = r[c];
        }
        const T* m = I.minv + 9 * (int64_t)row;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            T zc = m[3 * c] * r[0] + m[3 * c + 1] * r[1] + m[3 * c + 2] * r[2];
            I.z[4 * (int64_t)row + c] = zc;
            rz += (double)r[c] * (double)zc;
            double z64 = (double)m[3 * c] * r64[0] + (double)m[3 * c + 1] * r64[1] + (double)m[3 * c + 2] * r64[2];
            rz64 += r64[c] * z64;
        }
    }
    double v[2] = {rz, rz64}, tot[2];
    block_sum<2>(v, sh);
    __syncthreads();
    if (last_cta_reduce<2>(v, I.part, ck.pad, I.chunk0, I.nchunks, I.counter + 2, sh, tot) && threadIdx.x == 0) {
        double rzn = tot[0];
        I.scal[kRz64] = tot[1];
        if (first) {
            I.scal[kBnorm] = tot[1];
            I.scal[kThresh] = rtol2 * tot[1];
            I.scal[kBeta] = 0.0;
            I.scal[kIters] = 0.0;
        } else {
            double rzo = I.scal[kRzOld];
            I.scal[kBeta] = rzo > 0.0 ? rzn / rzo : 0.0;
        }
        I.scal[kRz] = rzn;
        I.scal[kRzRef] = rzn;
        *I.status = kRun;
    }
}

// ------------------------------------------------------------------ host loop

// Resident CTAs of the SpMV kernel on the current device (its persistent grid).
template <typename T>
int64_t PcgBatch<T>::spmv_resident() {
    if (resident_ > 0) return resident_;
    int dev = 0, sms = 148, per_sm = 2;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pcg_spmv<T>, kSpmvThreads, 0) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    resident_ = (int64_t)sms * per_sm;
    return resident_;
}

template <typename T>
void PcgBatch<T>::prepare(std::vector<PcgSystem<T>*>& sys, cudaStream_t s, std::vector<ChunkDev>& all_chunks,
                          std::vector<int>& chunk0, std::vector<int>& nch) {
    const int n = (int)sys.size();
    work_.resize(n);
    std::vector<InstDev<T>> hi(n);
    all_chunks.clear();
    d_scal_.alloc((size_t)n * kNScal, s);
    d_scal_.zero(s);
    d_status_.alloc(n, s);
    d_status_.zero(s);
    d_counter_.alloc((size_t)n * 4, s);
    d_counter_.zero(s);
    chunk0.assign(n, 0);
    nch.assign(n, 0);
    // Chunks of 64..kChunkRows rows. A system's chunks depend on its own row count only
    // (its partial sums, and so its results, are the same alone and in a batch); a large
    // system gets a whole number of equal chunks per resident SpMV CTA.
    const int64_t res = spmv_resident();
    for (int i = 0; i < n; ++i) {
        const int rows = sys[i]->S->n_rows;
        const int64_t per_cta = std::max<int64_t>(1, (rows + res * kChunkRows - 1) / (res * kChunkRows));
        const int64_t target = std::min<int64_t>(kChunkRows, std::max<int64_t>(
                                   64, (rows + res * per_cta - 1) / (res * per_cta)));
        chunk0[i] = (int)all_chunks.size();
        const int64_t k = std::max<int64_t>(1, (rows + target - 1) / target);
        for (int64_t j = 0; j < k; ++j) {
            const int r0 = (int)(rows * j / k), r1 = (int)(rows * (j + 1) / k);
            all_chunks.push_back(ChunkDev{i, r0, r1, (int)all_chunks.size()});
        }
        nch[i] = (int)all_chunks.size() - chunk0[i];
    }
    d_part_.alloc(all_chunks.size() * 4 + 4, s);
    for (int i = 0; i < n; ++i) {
        PcgSystem<T>& S = *sys[i];
        Work& w = work_[i];
        const size_t m = 3 * (size_t)S.S->n_rows;
        w.r.alloc(m, s);
        const size_t m4 = 4 * (size_t)S.S->n_rows;  // z and the directions: four per node (one padding)
        w.z.alloc(m4, s);
        w.p0.alloc(m4, s);
        w.z.zero(s);
        w.q.alloc(m, s);
        w.r64.alloc(m, s);
        w.p0.zero(s);
        if (S.warm_start) {
            S.residual64(S.x, S.b, w.r64.ptr, s);
        } else {
            FX_CUDA_CHECK(cudaMemsetAsync(S.x, 0, m * sizeof(double), s));
            FX_CUDA_CHECK(cudaMemcpyAsync(w.r64.ptr, S.b, m * sizeof(double), cudaMemcpyDeviceToDevice, s));
        }
        InstDev<T>& d = hi[i];
        d.n_rows = S.S->n_rows;
        d.chunk0 = chunk0[i];
        d.nchunks = nch[i];
        d.goff = S.S->goff.ptr;
        d.cols = S.S->cols.ptr;
        d.vals = S.vals;
        d.minv = S.minv;
        d.r = w.r.ptr;
        d.z = w.z.ptr;
        d.p0 = w.p0.ptr;
        d.q = w.q.ptr;
        d.x = S.x;
        d.r64 = w.r64.ptr;
        d.scal = d_scal_.ptr + (size_t)i * kNScal;
        d.status = d_status_.ptr + i;
        d.counter = d_counter_.ptr + 4 * i;
        d.part = d_part_.ptr;
        S.status = FX_OK;
        S.iterations = 0;
        S.replacements = 0;
        S.stagnated = false;
    }
    d_inst_.upload(hi, s);
    d_chunks_.upload(all_chunks, s);
}

template <typename T>
double PcgBatch<T>::profile_spmv(PcgSystem<T>& sys, int reps, cudaStream_t s) {
    std::vector<PcgSystem<T>*> v{&sys};
    std::vector<ChunkDev> chunks;
    std::vector<int> c0, nc;
    sys.warm_start = false;
    prepare(v, s, chunks, c0, nc);
    FX_LAUNCH(k_pcg_replace<T>, (unsigned)chunks.size(), kUpdThreads, 0, s, d_chunks_.ptr, d_inst_.ptr, 1, 0.0);
    // p = z (beta = 0 after the first replacement): a nonzero direction, so p.q > 0 and every
    // timed launch does its full work
    FX_LAUNCH(k_pcg_dir<T>, (unsigned)chunks.size(), kUpdThreads, 0, s, d_chunks_.ptr, d_inst_.ptr);
    for (int k = 0; k < 3; ++k)  // warm-up
        FX_LAUNCH(k_pcg_spmv<T>, spmv_grid(chunks.size()), kSpmvThreads, 0, s, d_chunks_.ptr, (int)chunks.size(),
                  d_inst_.ptr);
    EventTimer t;
    t.start(s);
    for (int k = 0; k < reps; ++k)
        FX_LAUNCH(k_pcg_spmv<T>, spmv_grid(chunks.size()), kSpmvThreads, 0, s, d_chunks_.ptr, (int)chunks.size(),
                  d_inst_.ptr);
    return t.stop_ms(s) / reps;
}

template <typename T>
int PcgBatch<T>::solve(std::vector<PcgSystem<T>*>& sys, const PcgOptions& opt, cudaStream_t s,
                       int64_t* launches) {
    const int n = (int)sys.size();
    if (n == 0) return FX_OK;
    std::vector<ChunkDev> all_chunks;
    std::vector<int> chunk0, nch;
    prepare(sys, s, all_chunks, chunk0, nch);
    const double rtol2 = opt.rtol * opt.rtol;
    const bool trace = std::getenv("FX_DEBUG") != nullptr;
    FX_LAUNCH(k_pcg_replace<T>, (unsigned)all_chunks.size(), kUpdThreads, 0, s, d_chunks_.ptr, d_inst_.ptr, 1,
              rtol2);
    if (launches) ++*launches;

    std::vector<double> h_scal((size_t)n * kNScal);
    std::vector<int> h_status(n);
    auto pull = [&]() {
        FX_CUDA_CHECK(cudaMemcpyAsync(h_scal.data(), d_scal_.ptr, h_scal.size() * sizeof(double),
                                      cudaMemcpyDeviceToHost, s));
        FX_CUDA_CHECK(cudaMemcpyAsync(h_status.data(), d_status_.ptr, n * sizeof(int), cudaMemcpyDeviceToHost, s));
        stream_wait(s, "pcg poll");
    };
    pull();
    // a warm-started solve (the FP64 finish of a stalled mixed one) measures its
    // residual against the original right-hand side, not its starting residual
    for (int i = 0; i < n; ++i) {
        double* sc = &h_scal[(size_t)i * kNScal];
        if (sys[i]->warm_start && sys[i]->bnorm2 > 0.0) {
            sc[kBnorm] = sys[i]->bnorm2;
            sc[kThresh] = rtol2 * sys[i]->bnorm2;
            FX_CUDA_CHECK(cudaMemcpyAsync(d_scal_.ptr + (size_t)i * kNScal + kBnorm, &sc[kBnorm], sizeof(double),
                                          cudaMemcpyHostToDevice, s));
            FX_CUDA_CHECK(cudaMemcpyAsync(d_scal_.ptr + (size_t)i * kNScal + kThresh, &sc[kThresh], sizeof(double),
                                          cudaMemcpyHostToDevice, s));
        }
        sys[i]->bnorm2_seen = sc[kBnorm];
    }
    std::vector<char> done(n, 0);
    std::vector<double> best(n, 1e300);
    std::vector<int> stall(n, 0);
    std::vector<double> last_rep(n, 0.0);      // iteration of the last FP64 residual replacement
    std::vector<double> last_improve(n, 0.0);  // iteration at which the best FP64 residual last halved
    for (int i = 0; i < n; ++i) {
        if (!(h_scal[i * kNScal + kBnorm] > 0.0)) {  // b = 0: x = 0 is exact
            done[i] = 1;
            sys[i]->relres = 0.0;
        }
    }
    const int poll = std::max(2, opt.poll & ~1);
    cudaGraphExec_t gexec = nullptr;
    std::vector<ChunkDev> act;
    DBuf<ChunkDev> d_act;
    bool rebuild = true;
    int result = FX_OK;
    auto set_status = [&](int i, int st) {
        FX_CUDA_CHECK(cudaMemcpyAsync(d_status_.ptr + i, &st, sizeof(int), cudaMemcpyHostToDevice, s));
    };
    for (int i = 0; i < n; ++i)
        if (done[i]) set_status(i, kIdle);
    while (true) {
        if (rebuild) {
            act.clear();
            for (auto& c : all_chunks)
                if (!done[c.inst]) act.push_back(c);
            if (act.empty()) break;
            d_act.upload(act, s);
            if (gexec) {
                cudaGraphExecDestroy(gexec);
                gexec = nullptr;
            }
            if (opt.graphs && !debug_sync()) {
                cudaGraph_t g;
                int64_t* saved = g_launch_counter;
                g_launch_counter = nullptr;
                FX_CUDA_CHECK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                for (int k = 0; k < poll; ++k) {
                    FX_LAUNCH(k_pcg_dir<T>, (unsigned)act.size(), kUpdThreads, 0, s, d_act.ptr, d_inst_.ptr);
                    FX_LAUNCH(k_pcg_spmv<T>, spmv_grid(act.size()), kSpmvThreads, 0, s, d_act.ptr, (int)act.size(),
                              d_inst_.ptr);
                    FX_LAUNCH(k_pcg_update<T>, (unsigned)act.size(), kUpdThreads, 0, s, d_act.ptr, d_inst_.ptr);
                }
                FX_CUDA_CHECK(cudaStreamEndCapture(s, &g));
                g_launch_counter = saved;
                FX_CUDA_CHECK(cudaGraphInstantiate(&gexec, g, 0));
                cudaGraphDestroy(g);
            }
            rebuild = false;
        }
        if (gexec) {
            FX_CUDA_CHECK(cudaGraphLaunch(gexec, s));
        } else {
            int64_t* saved = g_launch_counter;
            g_launch_counter = nullptr;
            for (int k = 0; k < poll; ++k) {
                FX_LAUNCH(k_pcg_dir<T>, (unsigned)act.size(), kUpdThreads, 0, s, d_act.ptr, d_inst_.ptr);
                FX_LAUNCH(k_pcg_spmv<T>, spmv_grid(act.size()), kSpmvThreads, 0, s, d_act.ptr, (int)act.size(),
                          d_inst_.ptr);
                FX_LAUNCH(k_pcg_update<T>, (unsigned)act.size(), kUpdThreads, 0, s, d_act.ptr, d_inst_.ptr);
            }
            g_launch_counter = saved;
        }
        if (launches) *launches += 3 * (int64_t)poll;
        pull();
        if (trace)
            for (int i = 0; i < n; ++i)
                std::fprintf(stderr, "[pcg] sys %d status %d iters %.0f rz %.3e rzref %.3e thresh %.3e pq %.3e\n", i,
                             h_status[i], h_scal[i * kNScal + kIters], h_scal[i * kNScal + kRz],
                             h_scal[i * kNScal + kRzRef], h_scal[i * kNScal + kThresh], h_scal[i * kNScal + kPq]);
        // decide per system
        std::vector<int> replace;
        for (int i = 0; i < n; ++i) {
            if (done[i]) continue;
            const double* sc = &h_scal[(size_t)i * kNScal];
            const int st = h_status[i];
            sys[i]->iterations = (long long)sc[kIters];
            if (st == kBreak) {
                // r.z == 0 exactly means an exact solution; anything else is a breakdown
                done[i] = 1;
                sys[i]->status = FX_NUMERICAL;
                if (result == FX_OK) result = FX_NUMERICAL;
                rebuild = true;
                continue;
            }
            bool reached = st == kConv;
            bool drop = sizeof(T) == 4 && sc[kRzRef] > 0.0 && sc[kRz] < opt.reliable_delta * opt.reliable_delta * sc[kRzRef];
            // FP32 recurrences can stall above the replacement trigger: replace periodically too
            bool periodic = sizeof(T) == 4 && sc[kIters] - last_rep[i] >= opt.replace_every;
            if (reached || drop || periodic) {
                replace.push_back(i);
                last_rep[i] = sc[kIters];
            }
            else if (sc[kIters] >= opt.max_iter) {
                done[i] = 1;
                sys[i]->status = FX_CONVERGENCE;
                if (result == FX_OK) result = FX_CONVERGENCE;
                rebuild = true;
            }
        }
        if (!replace.empty()) {
            std::vector<ChunkDev> rc;
            for (int i : replace) {
                PcgSystem<T>& S = *sys[i];
                S.residual64(S.x, S.b, work_[i].r64.ptr, s);
                for (int c = 0; c < nch[i]; ++c) rc.push_back(all_chunks[chunk0[i] + c]);
                S.replacements++;
            }
            DBuf<ChunkDev> d_rc;
            d_rc.upload(rc, s);
            FX_LAUNCH(k_pcg_replace<T>, (unsigned)rc.size(), kUpdThreads, 0, s, d_rc.ptr, d_inst_.ptr, 0, rtol2);
            pull();
            for (int i : replace) {
                const double* sc = &h_scal[(size_t)i * kNScal];
                double rel = std::sqrt(std::max(0.0, sc[kRz64]) / sc[kBnorm]);
                if (trace) std::fprintf(stderr, "[pcg] replace sys %d relres %.3e\n", i, rel);
                sys[i]->relres = rel;
                if (rel < 0.5 * best[i]) {
                    best[i] = rel;
                    stall[i] = 0;
                    last_improve[i] = sc[kIters];
                } else {
                    ++stall[i];
                }
                const bool slow = sc[kIters] - last_improve[i] >= opt.stall_iters || sc[kIters] >= 0.25 * opt.max_iter;
                if (rel <= opt.rtol) {
                    done[i] = 1;
                    set_status(i, kIdle);
                    rebuild = true;
                } else if (sizeof(T) == 8 && opt.accept_rtol > 0.0 && rel <= opt.accept_rtol &&
                           stall[i] >= opt.stall_limit) {
                    // the attainable FP64 residual lies between the tightened target and the
                    // caller's tolerance: converged at that floor
                    done[i] = 1;
                    set_status(i, kIdle);
                    rebuild = true;
                } else if (sizeof(T) == 4 && (stall[i] >= opt.stall_limit || slow)) {
                    done[i] = 1;
                    set_status(i, kIdle);
                    sys[i]->status = FX_CONVERGENCE;
                    sys[i]->stagnated = true;
                    rebuild = true;
                } else if (sc[kIters] >= opt.max_iter) {
                    done[i] = 1;
                    set_status(i, kIdle);
                    sys[i]->status = FX_CONVERGENCE;
                    if (result == FX_OK) result = FX_CONVERGENCE;
                    rebuild = true;
                }
            }
        }
    }
    if (gexec) cudaGraphExecDestroy(gexec);
    stream_wait(s, "stream");
    return result;
}

template class PcgBatch<float>;
template class PcgBatch<double>;

// A kernel of this file's module (preload_kernels() loads all of the module's kernels).
const void* kernels_anchor_pcg() { return reinterpret_cast<const void*>(&k_pcg_update<float>); }

}  // namespace fx
