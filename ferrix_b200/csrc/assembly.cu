#include <atomic>
// BSR(3x3) assembly: symbolic pattern by a device sort-by-key of node-pair
// keys built from the connectivity (once per mesh), numeric values by an
// atomic-free, fixed-order gather of element-pair blocks (every BSR block
// sums its contributing element slots in sorted order), penalty BCs and the
// 3x3 block-Jacobi preconditioner.
//
// Replaces TriMat accumulation + TriMat::to_csr of the reference
// (src/solver/assembler.rs:53,119-148; src/solver/step/static_step.rs:184-198)
// and DiagonalPreconditioner::new (src/solver/preconditioner.rs:36-50). The
// result holds the same sums as the reference's CSR (which sums duplicates),
// stored as dense 3x3 blocks (entries |v| <= 1e-12 kept as values).
#include <cub/cub.cuh>

#include <cmath>

#include "common.hpp"
#include "kernels.hpp"

namespace fx {

static int bits_for(int64_t n) {
    int b = 1;
    while ((int64_t(1) << b) < n) ++b;
    return b;
}

// key = (I << nb) | J, val = element pair slot | (a > b) << 31
__global__ void k_pair_keys(int nelem, int npe, const int32_t* __restrict__ conn, int nb, uint32_t slot_base,
                            int npairs, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals, int64_t out_base) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t total = (int64_t)nelem * npe * npe;
    if (t >= total) return;
    int e = (int)(t / (npe * npe));
    int r = (int)(t % (npe * npe));
    int a = r / npe, b = r % npe;
    uint64_t I = (uint32_t)conn[(int64_t)e * npe + a], J = (uint32_t)conn[(int64_t)e * npe + b];
    int lo = a < b ? a : b, hi = a < b ? b : a;
    uint32_t slot = slot_base + (uint32_t)e * (uint32_t)npairs + (uint32_t)pair_index(npe, lo, hi);
    keys[out_base + t] = (I << nb) | J;
    vals[out_base + t] = slot | (a > b ? 0x80000000u : 0u);
}

__global__ void k_heads(int64_t n, const uint64_t* __restrict__ keys, int32_t* __restrict__ head) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1 : 0;
}

__global__ void k_blocks(int64_t n, const uint64_t* __restrict__ keys, const int32_t* __restrict__ bid, int nb,
                         int64_t* __restrict__ seg, int32_t* __restrict__ blk_row, int32_t* __restrict__ blk_col,
                         int32_t* __restrict__ row_cnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (i == 0 || keys[i] != keys[i - 1]) {
        int b = bid[i] - 1;
        seg[b] = i;
        int I = (int)(keys[i] >> nb);
        blk_row[b] = I;
        blk_col[b] = (int)(keys[i] & ((uint64_t(1) << nb) - 1));
        atomicAdd(&row_cnt[I], 1);  // integer count: order-independent
    }
}

__global__ void k_groups(int n, const int32_t* __restrict__ cnt, int32_t* __restrict__ ng) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int c = cnt[i];
    ng[i] = c > 0 ? (c + 3) / 4 : 1;
}

__global__ void k_fill_cols_pad(int n, const int32_t* __restrict__ goff, int32_t* __restrict__ cols) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    for (int g = goff[i]; g < goff[i + 1]; ++g)
        for (int l = 0; l < 4; ++l) cols[4 * g + l] = i;
}

__global__ void k_place_cols(int64_t nblk, const int32_t* __restrict__ blk_row, const int32_t* __restrict__ blk_col,
                             const int32_t* __restrict__ row_ptr, const int32_t* __restrict__ goff,
                             int32_t* __restrict__ cols, int32_t* __restrict__ diag_k) {
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    int i = blk_row[b];
    int k = (int)(b - row_ptr[i]);
    int j = blk_col[b];
    cols[4 * (int64_t)goff[i] + k] = j;
    if (j == i) diag_k[i] = k;
}

__global__ void k_node_keys(int nelem, int npe, const int32_t* __restrict__ conn, int slot_base,
                            int32_t* __restrict__ keys, int32_t* __restrict__ vals, int64_t out_base) {
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)nelem * npe) return;
    keys[out_base + t] = conn[t];
    vals[out_base + t] = slot_base + (int32_t)t;
}

__global__ void k_count(int64_t n, const int32_t* __restrict__ keys, int32_t* __restrict__ cnt) {
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    atomicAdd(&cnt[keys[i]], 1);
}

template <typename Op>
static void cub_call(Op op, DBuf<uint8_t>& tmp, cudaStream_t s) {
    size_t bytes = 0;
    FX_CUDA_CHECK(op(nullptr, bytes));
    if (tmp.n < bytes) tmp.alloc(bytes, s);
    FX_CUDA_CHECK(op(tmp.ptr, bytes));
}

static void exclusive_scan_i32(const int32_t* in, int32_t* out, int n, DBuf<uint8_t>& tmp, cudaStream_t s) {
    // out has n+1 entries: out[0]=0 .. out[n]=total
    FX_CUDA_CHECK(cudaMemsetAsync(out, 0, sizeof(int32_t), s));
    cub_call([&](void* t, size_t& b) { return cub::DeviceScan::InclusiveSum(t, b, in, out + 1, n, s); }, tmp, s);
}

void build_bsr_structure(const ElemView& g4, const ElemView& g20, int n_nodes, BsrStructure& S, cudaStream_t s) {
    static std::atomic<uint64_t> next_id{1};
    S.id = next_id.fetch_add(1);
    S.n_rows = n_nodes;
    const int64_t p4 = (int64_t)g4.n * 16, p20 = (int64_t)g20.n * 400;
    const int64_t P = p4 + p20;
    if ((int64_t)g4.n * kPairs4 + (int64_t)g20.n * kPairs20 >= (int64_t(1) << 31))
        fail(FX_INVALID_ARGUMENT, "mesh too large for 31-bit element-pair slots");
    // the sort items (ordered node pairs of every element) are counted, scanned and
    // indexed in 32 bits: about twice the slots, so this bound is the tighter one
    if (P >= (int64_t(1) << 31)) fail(FX_INVALID_ARGUMENT, "mesh too large for 32-bit node-pair sort items");
    S.n_pairs = P;
    const int nb = bits_for(n_nodes > 1 ? n_nodes : 2);
    DBuf<uint64_t> keys, keys_s;
    DBuf<uint32_t> vals;
    DBuf<uint8_t> tmp;
    keys.alloc(P, s);
    keys_s.alloc(P, s);
    vals.alloc(P, s);
    S.slot_sorted.alloc(P, s);
    const int T = 256;
    if (g4.n)
        FX_LAUNCH(k_pair_keys, (unsigned)((p4 + T - 1) / T), T, 0, s, g4.n, 4, g4.conn, nb, 0u, kPairs4, keys.ptr,
                  vals.ptr, (int64_t)0);
    if (g20.n)
        FX_LAUNCH(k_pair_keys, (unsigned)((p20 + T - 1) / T), T, 0, s, g20.n, 20, g20.conn, nb,
                  (uint32_t)(g4.n * kPairs4), kPairs20, keys.ptr, vals.ptr, p4);
    const int end_bit = 2 * nb;
    cub_call([&](void* t, size_t& b) {
        return cub::DeviceRadixSort::SortPairs(t, b, keys.ptr, keys_s.ptr, vals.ptr, S.slot_sorted.ptr, P, 0,
                                               end_bit, s);
    }, tmp, s);
    keys.release();
    vals.release();
    DBuf<int32_t> head, bid;
    head.alloc(P, s);
    bid.alloc(P, s);
    FX_LAUNCH(k_heads, (unsigned)((P + T - 1) / T), T, 0, s, P, keys_s.ptr, head.ptr);
    cub_call([&](void* t, size_t& b) { return cub::DeviceScan::InclusiveSum(t, b, head.ptr, bid.ptr, P, s); }, tmp,
             s);
    int32_t nblk = 0;
    FX_CUDA_CHECK(cudaMemcpyAsync(&nblk, bid.ptr + P - 1, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    FX_CUDA_CHECK(cudaStreamSynchronize(s));
    S.n_blocks = nblk;
    head.release();
    S.seg.alloc(nblk + 1, s);
    S.blk_row.alloc(nblk, s);
    DBuf<int32_t> blk_col, cnt;
    blk_col.alloc(nblk, s);
    cnt.alloc(n_nodes, s);
    cnt.zero(s);
    FX_LAUNCH(k_blocks, (unsigned)((P + T - 1) / T), T, 0, s, P, keys_s.ptr, bid.ptr, nb, S.seg.ptr, S.blk_row.ptr,
              blk_col.ptr, cnt.ptr);
    FX_CUDA_CHECK(cudaMemcpyAsync(S.seg.ptr + nblk, &P, sizeof(int64_t), cudaMemcpyHostToDevice, s));
    keys_s.release();
    bid.release();
    S.row_ptr.alloc(n_nodes + 1, s);
    exclusive_scan_i32(cnt.ptr, S.row_ptr.ptr, n_nodes, tmp, s);
    DBuf<int32_t> ng;
    ng.alloc(n_nodes, s);
    FX_LAUNCH(k_groups, (n_nodes + T - 1) / T, T, 0, s, n_nodes, cnt.ptr, ng.ptr);
    S.goff.alloc(n_nodes + 1, s);
    exclusive_scan_i32(ng.ptr, S.goff.ptr, n_nodes, tmp, s);
    int32_t G = 0;
    FX_CUDA_CHECK(cudaMemcpyAsync(&G, S.goff.ptr + n_nodes, sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    FX_CUDA_CHECK(cudaStreamSynchronize(s));
    S.n_groups = G;
    S.cols.alloc((size_t)G * 4, s);
    S.diag_k.alloc(n_nodes, s);
    FX_CUDA_CHECK(cudaMemsetAsync(S.diag_k.ptr, 0xff, sizeof(int32_t) * n_nodes, s));  // -1 = no diagonal block
    FX_LAUNCH(k_fill_cols_pad, (n_nodes + T - 1) / T, T, 0, s, n_nodes, S.goff.ptr, S.cols.ptr);
    FX_LAUNCH(k_place_cols, (unsigned)((nblk + T - 1) / T), T, 0, s, (int64_t)nblk, S.blk_row.ptr, blk_col.ptr,
              S.row_ptr.ptr, S.goff.ptr, S.cols.ptr, S.diag_k.ptr);
    // node -> element-node slots (fixed order: group, element, local node)
    const int64_t q4 = (int64_t)g4.n * 4, q20 = (int64_t)g20.n * 20, Q = q4 + q20;
    DBuf<int32_t> nk, nv, nks;
    nk.alloc(Q, s);
    nv.alloc(Q, s);
    nks.alloc(Q, s);
    S.node_slots.alloc(Q, s);
    if (g4.n) FX_LAUNCH(k_node_keys, (unsigned)((q4 + T - 1) / T), T, 0, s, g4.n, 4, g4.conn, 0, nk.ptr, nv.ptr,
                        (int64_t)0);
    if (g20.n) FX_LAUNCH(k_node_keys, (unsigned)((q20 + T - 1) / T), T, 0, s, g20.n, 20, g20.conn, (int)q4, nk.ptr,
                         nv.ptr, q4);
    if (Q) {
        cub_call([&](void* t, size_t& b) {
            return cub::DeviceRadixSort::SortPairs(t, b, nk.ptr, nks.ptr, nv.ptr, S.node_slots.ptr, Q, 0, nb, s);
        }, tmp, s);
    }
    cnt.zero(s);
    if (Q) FX_LAUNCH(k_count, (unsigned)((Q + T - 1) / T), T, 0, s, Q, nks.ptr, cnt.ptr);
    S.node_ptr.alloc(n_nodes + 1, s);
    exclusive_scan_i32(cnt.ptr, S.node_ptr.ptr, n_nodes, tmp, s);
    FX_CUDA_CHECK(cudaStreamSynchronize(s));
}

// ---- numeric gather: thread per block, fixed slot order
template <typename T>
__global__ void k_bsr_gather(int64_t nblk, const int32_t* __restrict__ blk_row, const int32_t* __restrict__ row_ptr,
                             const int32_t* __restrict__ goff, const int64_t* __restrict__ seg,
                             const uint32_t* __restrict__ slots, const T* __restrict__ ebuf, T* __restrict__ vals) {
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    T acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t s = seg[b]; s < seg[b + 1]; ++s) {
        uint32_t v = slots[s];
        const T* src = ebuf + (size_t)(v & 0x7fffffffu) * 9;
        if (v & 0x80000000u) {
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) acc[3 * r + c] += src[3 * c + r];
        } else {
#pragma unroll
            for (int c = 0; c < 9; ++c) acc[c] += src[c];
        }
    }
    int i = blk_row[b];
    int k = (int)(b - row_ptr[i]);
    int64_t g0 = goff[i];
    int ng = goff[i + 1] - (int)g0;
    int64_t base = (g0 * 9 + k / 4) * 4 + (k & 3);
#pragma unroll
    for (int c = 0; c < 9; ++c) vals[base + (int64_t)c * ng * 4] = acc[c];
}

template <typename T>
void launch_bsr_gather(const BsrStructure& S, const T* ebuf, T* vals, cudaStream_t s) {
    FX_CUDA_CHECK(cudaMemsetAsync(vals, 0, sizeof(T) * S.n_groups * 36, s));
    if (S.n_blocks)
        FX_LAUNCH(k_bsr_gather<T>, (unsigned)((S.n_blocks + 255) / 256), 256, 0, s, S.n_blocks, S.blk_row.ptr,
                  S.row_ptr.ptr, S.goff.ptr, S.seg.ptr, S.slot_sorted.ptr, ebuf, vals);
}
template void launch_bsr_gather<float>(const BsrStructure&, const float*, float*, cudaStream_t);
template void launch_bsr_gather<double>(const BsrStructure&, const double*, double*, cudaStream_t);

__device__ __forceinline__ int64_t diag_index(const int32_t* goff, const int32_t* diag_k, int i, int e) {
    int k = diag_k[i];
    int64_t g0 = goff[i];
    int ng = goff[i + 1] - (int)g0;
    return (g0 * 9 + (int64_t)e * ng + k / 4) * 4 + (k & 3);
}

// ---- penalty (static_step.rs:184-195), merged per DOF
template <typename T>
__global__ void k_penalty(int n, const int32_t* __restrict__ dof, const double* __restrict__ cnt,
                          const double* __restrict__ usum, const int32_t* __restrict__ goff,
                          const int32_t* __restrict__ diag_k, T* __restrict__ vals,
                          const unsigned long long* __restrict__ maxdiag, double* __restrict__ rhs,
                          const double* __restrict__ u) {
    int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n) return;
    double md = __longlong_as_double((long long)*maxdiag);
    if (!(md > 0.0)) return;
    double P = md * 1.0e6;
    int d = dof[m];
    int i = d / 3, c = d % 3;
    if (vals && diag_k[i] >= 0) {
        int64_t idx = diag_index(goff, diag_k, i, 4 * c);  // component (c, c)
        vals[idx] = (T)((double)vals[idx] + cnt[m] * P);
    }
    if (rhs) rhs[d] += P * usum[m] - P * cnt[m] * u[d];
}

template <typename T>
void launch_penalty(const BsrStructure& S, T* vals, const BcView& bc, const unsigned long long* maxdiag,
                    double* rhs, const double* u, cudaStream_t s) {
    if (bc.n)
        FX_LAUNCH(k_penalty<T>, (bc.n + 255) / 256, 256, 0, s, bc.n, bc.dof, bc.cnt, bc.usum, S.goff.ptr,
                  S.diag_k.ptr, vals, maxdiag, rhs, u);
}
template void launch_penalty<float>(const BsrStructure&, float*, const BcView&, const unsigned long long*, double*,
                                    const double*, cudaStream_t);
template void launch_penalty<double>(const BsrStructure&, double*, const BcView&, const unsigned long long*,
                                     double*, const double*, cudaStream_t);

// ---- 3x3 block-Jacobi inverse, FP64 arithmetic; a singular block falls back
// to the scalar rule of DiagonalPreconditioner (1/d when |d| > 1e-9, else 1).
template <typename T>
__global__ void k_block_jacobi(int n, const int32_t* __restrict__ goff, const int32_t* __restrict__ diag_k,
                               const T* __restrict__ vals, T* __restrict__ minv) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double D[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (diag_k[i] >= 0)
        for (int e = 0; e < 9; ++e) D[e] = (double)vals[diag_index(goff, diag_k, i, e)];
    double Di[9];
    double det = inv3(D, Di);
    double scale = fabs(D[0]) * fabs(D[4]) * fabs(D[8]);
    bool ok = det != 0.0 && isfinite(det) && fabs(det) > 1e-14 * scale;
    for (int e = 0; e < 9; ++e) {
        double v;
        if (ok) {
            v = Di[e];
        } else {
            int r = e / 3, c = e % 3;
            v = (r == c) ? (fabs(D[e]) > 1e-9 ? 1.0 / D[e] : 1.0) : 0.0;
        }
        minv[9 * (int64_t)i + e] = (T)v;
    }
}

template <typename T>
void launch_block_jacobi(const BsrStructure& S, const T* vals, T* minv, cudaStream_t s) {
    if (S.n_rows)
        FX_LAUNCH(k_block_jacobi<T>, (S.n_rows + 255) / 256, 256, 0, s, S.n_rows, S.goff.ptr, S.diag_k.ptr, vals,
                  minv);
}
template void launch_block_jacobi<float>(const BsrStructure&, const float*, float*, cudaStream_t);
template void launch_block_jacobi<double>(const BsrStructure&, const double*, double*, cudaStream_t);

// ---- expanded CSR for host inspection: row 3i+r has 3*cnt_i entries
template <typename T>
__global__ void k_bsr_to_csr(int64_t nblk, const int32_t* __restrict__ blk_row, const int32_t* __restrict__ row_ptr,
                             const int32_t* __restrict__ goff, const int32_t* __restrict__ cols,
                             const T* __restrict__ vals, const int64_t* __restrict__ indptr,
                             int64_t* __restrict__ indices, double* __restrict__ data) {
    int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblk) return;
    int i = blk_row[b];
    int k = (int)(b - row_ptr[i]);
    int64_t g0 = goff[i];
    int ng = goff[i + 1] - (int)g0;
    int j = cols[4 * g0 + k];
    for (int r = 0; r < 3; ++r) {
        int64_t o = indptr[3 * i + r] + 3 * k;
        for (int c = 0; c < 3; ++c) {
            indices[o + c] = 3 * (int64_t)j + c;
            data[o + c] = (double)vals[(g0 * 9 + (int64_t)(3 * r + c) * ng + k / 4) * 4 + (k & 3)];
        }
    }
}

template <typename T>
void launch_bsr_to_csr(const BsrStructure& S, const T* vals, const int64_t* indptr, int64_t* indices, double* data,
                       cudaStream_t s) {
    if (S.n_blocks)
        FX_LAUNCH(k_bsr_to_csr<T>, (unsigned)((S.n_blocks + 255) / 256), 256, 0, s, S.n_blocks, S.blk_row.ptr,
                  S.row_ptr.ptr, S.goff.ptr, S.cols.ptr, vals, indptr, indices, data);
}
template void launch_bsr_to_csr<float>(const BsrStructure&, const float*, const int64_t*, int64_t*, double*,
                                       cudaStream_t);
template void launch_bsr_to_csr<double>(const BsrStructure&, const double*, const int64_t*, int64_t*, double*,
                                        cudaStream_t);

// A kernel of this file's module (preload_kernels() loads all of the module's kernels).
const void* kernels_anchor_assembly() { return reinterpret_cast<const void*>(&k_pair_keys); }

}  // namespace fx
