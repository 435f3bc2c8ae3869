/*
 * moao_b200 — building blocks exposed for tests and tuning. These have no
 * counterpart in the reference; they let the test suite check the tensor-core
 * kernels in isolation.
 */
#ifndef MOAO_B200_DEBUG_H
#define MOAO_B200_DEBUG_H

#include "moao_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Tensor-core GEMM on the context stream (device pointers):
 *   kind 0 (bf16): C[f32, M x N, col-major, ldc] = alpha * sum_p A_{pa[p]} B_{pb[p]}^T + beta * C
 *   kind 1 (int8): C[f64] += alpha * 2^(erow[r] + ecol[c] + shift) * sum_p A_{pa[p]} B_{pb[p]}^T
 *   kind 2 (fp16): C[f32] = alpha * 2^(erow[r] + ecol[c] + shift) * sum_p A_{pa[p]} B_{pb[p]}^T
 *                  + beta * C (erow and ecol NULL: no scaling)
 * A holds na slices of M x K row-major (lda elements per row), slice i at
 * A + i * M * lda; B holds nb slices of N x K row-major likewise. lower = 1
 * writes only C(r, c) with r >= c. Synchronises and returns MOAO_ERR_TIMEOUT
 * if a bounded device wait expired. */
moao_status moao_debug_tc_gemm(moao_ctx* ctx, int kind, long M, long N, long K, const void* A,
                               long lda, int na, const void* B, long ldb, int nb, int npairs,
                               const int* pa, const int* pb, void* C, long ldc, float alpha,
                               float beta, const int* erow, const int* ecol, int shift, int lower);

/* The mixed path's refinement residual on its own (device pointers, context
 * stream): E (m x n, ldE) = Ctm - R sym(Cmm), Cmm n x n read through its lower
 * triangle, both operands rounded to the context's int8 slice precision
 * (moao_ctx_set_mixed, default 5 slices = 35 bits). scheme 0: the int8 slice
 * products (pairs of slice indices summing to at most slices + 1); scheme 1:
 * exact products by the Chinese remainder theorem. Synchronises. */
moao_status moao_debug_residual(moao_ctx* ctx, int scheme, long m, long n, const double* R,
                                long ldR, const double* Cmm, long ldCmm, const double* Ctm,
                                long ldCtm, double* E, long ldE);

/* Moduli the CRT residual uses for a product over K terms of two operands of
 * ns-slice precision (0: none suffice, or K >= 131,072 breaks the exact int32
 * sums, and the slice products run instead). Host only. */
int moao_debug_crt_moduli(int ns, long K);

#ifdef __cplusplus
}
#endif

#endif /* MOAO_B200_DEBUG_H */
