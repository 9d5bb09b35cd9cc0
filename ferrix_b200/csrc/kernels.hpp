// Host-visible declarations of the device kernels' launchers and the device
// data structures they operate on.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.hpp"
#include "device.cuh"

namespace fx {

struct ElemView {
    int n = 0;
    const int32_t* conn = nullptr;
    const int32_t* mat = nullptr;
};

struct DeviceTables {
    DBuf<double> n20_d, dn20_d, w20, dn20_nodes;
    DBuf<float> n20_f, dn20_f;
    DBuf<uint8_t> pair20;
    void init(cudaStream_t s);
    RuleTables view() const;
};

// ---- element kernels (elements.cu)
template <typename T>
void launch_stiffness(const ElemView& g4, const ElemView& g20, const double* X, const double* u, const double* Tcur,
                      const MatDev& md, const RuleTables& rt, T* ebuf, unsigned long long* maxdiag, int* err,
                      cudaStream_t s);
void launch_apply(const ElemView& g4, const ElemView& g20, const double* X, const double* uconf, const double* v,
                  const double* tinit, const double* tcur, double cv, double cth, const MatDev& md,
                  const RuleTables& rt, double* fe, int* err, cudaStream_t s);
void launch_node_gather(int n_nodes, const int32_t* ptr, const int32_t* slots, const double* fe, double* out,
                        cudaStream_t s);
// nodal-averaged stress and mechanical strain (6 Voigt components each, per node)
void launch_nodal_stress(const ElemView& g4, const ElemView& g20, const double* X, const double* u,
                         const double* tinit, const double* tcur, const MatDev& md, const RuleTables& rt, int n_nodes,
                         const int32_t* node_ptr, const int32_t* node_slots, double* slot_buf, double* S, double* E,
                         int* err, cudaStream_t s);

// ---- BSR3 structure (assembly.cu)
// Block row i holds cnt_i = row_ptr[i+1]-row_ptr[i] blocks sorted by column,
// stored in ng_i = goff[i+1]-goff[i] = max(1, ceil(cnt_i/4)) groups of 4.
// cols: int4 per group (padding = i). vals: 9 component planes per row, each
// ng_i vec4 long: value (e, k) of block k at vec4 index goff[i]*9 + e*ng_i + k/4,
// lane k%4. Slot lists: the element-pair slots contributing to block b are
// slot_sorted[seg[b] .. seg[b+1]) (bit 31 = transposed).
struct BsrStructure {
    uint64_t id = 0;  // distinct for every structure built in the process
    int n_rows = 0;
    int64_t n_blocks = 0, n_groups = 0, n_pairs = 0;
    DBuf<int32_t> row_ptr, goff, cols, diag_k, blk_row;
    DBuf<int64_t> seg;
    DBuf<uint32_t> slot_sorted;
    // node -> element-node slots (for the fixed-order force gather)
    DBuf<int32_t> node_ptr, node_slots;
};

void build_bsr_structure(const ElemView& g4, const ElemView& g20, int n_nodes, BsrStructure& S, cudaStream_t s);

template <typename T>
void launch_bsr_gather(const BsrStructure& S, const T* ebuf, T* vals, cudaStream_t s);

// Penalty rows: one entry per constrained DOF (duplicates merged on the host).
struct BcView {
    int n = 0;
    const int32_t* dof = nullptr;
    const double* cnt = nullptr;   // number of BC records on the DOF
    const double* usum = nullptr;  // sum of the records' target values
};

// K_ii += cnt * 1e6 * maxdiag on the BSR diagonal; rhs_i += P (usum - cnt u_i) when rhs != null.
template <typename T>
void launch_penalty(const BsrStructure& S, T* vals, const BcView& bc, const unsigned long long* maxdiag,
                    double* rhs, const double* u, cudaStream_t s);
// 3x3 block-Jacobi inverse of the (penalised) diagonal blocks.
template <typename T>
void launch_block_jacobi(const BsrStructure& S, const T* vals, T* minv, cudaStream_t s);
// Expanded CSR (3x3 blocks, explicit zeros) for host inspection.
template <typename T>
void launch_bsr_to_csr(const BsrStructure& S, const T* vals, const int64_t* indptr, int64_t* indices, double* data,
                       cudaStream_t s);

// ---- vector kernels (vectors.cu)
void launch_axpby(int64_t n, double a, const double* x, double b, const double* y, double* out, cudaStream_t s);
void launch_scatter_set(int n, const int32_t* idx, const double* val, double* out, cudaStream_t s);
// out[dof] -= cnt * P * x[dof] over BC rows (penalty part of K x).
void launch_penalty_apply(const BcView& bc, const unsigned long long* maxdiag, const double* x, double* out,
                          cudaStream_t s);
// Deterministic masked norms: out[0] = sum_{!mask} a^2, out[1] = sum_{!mask} b^2.
void launch_masked_norms(int64_t n, const double* a, const double* b, const uint8_t* mask, double* partials,
                         double* out, cudaStream_t s);

}  // namespace fx
