// Dense FP64 building blocks of the reconstructor and of the Cee/Cvv chain.
#ifndef MOAO_DENSE_H
#define MOAO_DENSE_H

#include <cuda_runtime.h>

#include "moao_internal.h"

namespace moao {

// Which part of the STORED B matrix a GEMM may read (the rest is taken as 0):
// used to multiply by a symmetric matrix held in its lower triangle.
enum TriMode { TRI_FULL = 0, TRI_LOWER = 1, TRI_STRICT_LOWER = 2 };

struct GemmArgs {
  long M = 0, N = 0, K = 0;
  double alpha = 1, beta = 0;
  const double* A = nullptr;  // M x K, column-major, lda
  long lda = 0;
  const double* B = nullptr;  // K x N (transB = false) or N x K (transB = true)
  long ldb = 0;
  bool transB = false;
  TriMode triB = TRI_FULL;
  double* C = nullptr;        // M x N, column-major, ldc
  long ldc = 0;
  bool lowerC = false;        // write only C(i, j) with i >= j (SYRK / SYR2K)
  int cfg = 1;                // tile configuration of the large products (128x64 CTA tiles;
                              // 0: K 16 per stage, 4 stages; 1: K 32, 2 stages (default);
                              // 2: K 32, 3 stages; 3: K 16, 6 stages)
};
constexpr int kGemmConfigs = 4;

// C = alpha * A * op(B) + beta * C in FP64 on the DMMA tensor-core path.
moao_status gemm_f64(const GemmArgs& g, cudaStream_t s, long long* launches);

// Factor the n x n (n <= 64) diagonal block A (lower triangle read) in place:
// A <- L (lower; the upper triangle is left untouched) and Linv <- L^-1 (lower,
// zeros above the diagonal, ldi). On a non-positive pivot the 1-based global
// column (col0 + local column + 1) is stored in *d_info if it is still 0.
moao_status potrf_inv_leaf(double* A, long lda, double* Linv, long ldi, int n, long col0,
                           int* d_info, cudaStream_t s, long long* launches);

// Elementwise helpers (column-major).
moao_status copy_matrix(const double* src, long lds, double* dst, long ldd, long m, long n,
                        cudaStream_t s);
moao_status fill_matrix(double* A, long lda, long m, long n, double v, cudaStream_t s,
                        long long* launches);
// Cee <- sym(tril(Cpp)): the net effect of laset('U',0,0) + lacpy('L') +
// geadd('T') + scal(diag, 0.5) in lapack/compute/cee_cvv.cpp:73-92.
moao_status sym_from_lower(const double* Cpp, long ldp, double* Cee, long lde, long n,
                           cudaStream_t s, long long* launches);

}  // namespace moao

#endif  // MOAO_DENSE_H
