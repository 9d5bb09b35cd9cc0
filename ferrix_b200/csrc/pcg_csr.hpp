// Scalar-CSR FP64 Jacobi PCG (see pcg_csr.cu).
#pragma once

#include "pcg.hpp"

namespace fx {

struct CsrSystem {
    int64_t n = 0, nnz = 0;
    DBuf<int64_t> ip;
    DBuf<int32_t> ind;
    DBuf<double> val, dinv;
    // scalar CSR of an FP64 BSR3 matrix (3 rows per block row) + Jacobi inverse diagonal
    void from_bsr(const BsrStructure& S, const double* vals64, cudaStream_t s);
    // a caller's host CSR (int64 row offsets and columns, columns checked by the caller)
    void from_host(int64_t rows, const int64_t* ip, const int64_t* ind, const double* val, cudaStream_t s);
};

class CsrPcg {
   public:
    // x = solution (device, overwritten). absolute: stop on sqrt(r.z) < rtol (reference
    // IterativeSolver semantics) instead of sqrt(r.z / b.D^-1 b) < rtol.
    int solve(CsrSystem& A, const double* b, double* x, const PcgOptions& opt, bool absolute, cudaStream_t s,
              int64_t* launches, long long* iters, double* relres);

   private:
    DBuf<double> r_, z_, p0_, p1_, q_, part_, scal_;
    DBuf<int> status_, counter_;
};

}  // namespace fx
