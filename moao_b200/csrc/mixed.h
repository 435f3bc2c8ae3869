// Mixed-precision reconstructor: conversion / slicing kernels and the driver.
#ifndef MOAO_MIXED_H
#define MOAO_MIXED_H

#include <cuda_runtime.h>

#include <cstdint>

#include "moao_internal.h"

namespace moao {

constexpr int kMaxOzakiSlices = 6;

// Exact products by the Chinese remainder theorem. An operand of ns-slice
// precision is the integer X = rint(x 2^(7 ns - 1 - e)) of its row (column)
// exponent e, |X| <= 2^(7 ns - 1); its residues modulo pairwise coprime
// m_i <= 256 are int8 values, one exact int8 GEMM per modulus gives the
// product's residues, and mixed-radix (Garner) reconstruction the product
// itself, exact while |product| < M / 2 (M = the moduli's product).
constexpr int kCrtMaxModuli = 13;
constexpr int kCrtMod[kCrtMaxModuli] = {256, 255, 253, 251, 247, 241, 239,
                                        233, 229, 227, 223, 217, 211};
// Moduli needed for a product over K terms of two ns-slice operands: the
// fewest leading kCrtMod whose product exceeds 2 K 2^(2 (7 ns - 1)); 0 when
// none suffice or K breaks the int32 accumulation (K * 2^14 >= 2^31).
int crt_moduli_for(int ns, long K);

// Kernels launched so far on this thread by the helpers declared here.
long long helper_launches();
constexpr int kMaxBfSlices = 3;

constexpr int kMaxOffsetRanges = 32;

// Block-constant offsets of a symmetric matrix: value[w] is part of every entry
// (i, j) with both i and j in [begin[w], end[w]). Ranges do not overlap.
struct OffsetRanges {
  int n = 0;
  int begin[kMaxOffsetRanges] = {};
  int end[kMaxOffsetRanges] = {};
  double value[kMaxOffsetRanges] = {};
};

// Destinations of the bf16 slices of one block (null p[0] = not wanted); each
// pointer addresses the block's first element in its slice.
struct BfSlices {
  void* p[kMaxBfSlices];
};

moao_status cvt_f32_to_f64(const float* s, long lds, double* d, long ldd, long m, long n,
                           bool lower, cudaStream_t st);
moao_status cvt_f64_to_f32(const double* s, long lds, float* d, long ldd, long m, long n,
                           bool lower, cudaStream_t st);
moao_status add_f32_to_f64(const float* s, long lds, double* d, long ldd, long m, long n,
                           cudaStream_t st);
// bf16 split of an FP64 column-major m x n block into ns slices (slice k =
// bf16 of what the previous slices left), written row-major (stride ldr) and/or
// column-major (stride ldc).
moao_status split_bf16(const double* src, long lds, long m, long n, int ns, BfSlices rmaj,
                       long ldr, BfSlices cmaj, long ldc, cudaStream_t st);
// Per-row (erow[m]) and/or per-column (ecol[n]) exponents of a column-major
// m x n block: the smallest e with max |x| < 2^e, minus bias (null skips one).
moao_status scale_exponents(const double* A, long lda, long m, long n, int bias, int* erow,
                            int* ecol, cudaStream_t st);
moao_status scale_exponents(const float* A, long lda, long m, long n, int bias, int* erow,
                            int* ecol, cudaStream_t st);
// fp16 split of x * 2^-e into ns slices: row-major copy scaled by erow[r],
// column-major copy by ecol[c] (either copy may be skipped with a null p[0]).
moao_status split_f16(const double* src, long lds, long m, long n, int ns, BfSlices rmaj,
                      long ldr, const int* erow, BfSlices cmaj, long ldc, const int* ecol,
                      cudaStream_t st);
moao_status split_f16(const float* src, long lds, long m, long n, int ns, BfSlices rmaj,
                      long ldr, const int* erow, BfSlices cmaj, long ldc, const int* ecol,
                      cudaStream_t st);
// Row exponents (erow[m], minus bias) and row-major fp16 slices (stride ldx) of
// an FP32 column-major m x kb block in one pass, kb <= 1024; slice columns
// kb..kpad-1 are zeroed.
moao_status split_rows_f16(const float* src, long lds, long m, long kb, int ns, BfSlices out,
                           long ldx, long kpad, int* erow, int bias, cudaStream_t st);
// int8 slices of the rows of A (m x n, column-major): per-row exponents in e[m],
// slice s at out + s*m*ldo, row-major with row stride ldo.
moao_status ozaki_split_rows(const double* A, long lda, long m, long n, int ns, int* e,
                             int8_t* out, long ldo, cudaStream_t st);
// Residues (nmod of them, int8, centred) of the rows of A at ns-slice
// precision, with the row exponents e[m] already computed (ozaki_split_rows
// computes the same exponents): residue i at out + i*m*ldo, row-major.
moao_status crt_split_rows(const double* A, long lda, long m, long n, int ns, int nmod,
                           const int* e, int8_t* out, long ldo, cudaStream_t st);
// Residues of the columns of sym(A) - offsets (lower-stored n x n A) at
// ns-slice precision; computes the column exponents f[n]; residue i at
// out + i*n*ldo with row j holding column j.
moao_status crt_split_sym(const double* A, long lda, long n, int ns, int nmod, int* f,
                          unsigned long long* colmax, int8_t* out, long ldo, const int* rid,
                          const OffsetRanges& off, cudaStream_t st);
// E (m x n, lde) = C (ldc) + alpha * P 2^(e[r] + f[c] - 2 (7 ns - 1)), P the
// product whose residues modulo kCrtMod[i] are Z + i*m*n (uint8 in [0, m_i),
// column-major, ld m).
moao_status crt_combine(const uint8_t* Z, long m, long n, int nmod, int ns, const int* e,
                        const int* f, const double* C, long ldc, double alpha, double* E,
                        long lde, cudaStream_t st);
// int8 slices of the columns of sym(A) - offsets for a lower-stored n x n A
// (rid: range of every index or -1, null for no offsets): per-column exponents
// in f[n]; slice s at out + s*n*ldo with row j holding column j.
moao_status ozaki_split_sym(const double* A, long lda, long n, int ns, int* f,
                            unsigned long long* colmax, int8_t* out, long ldo, const int* rid,
                            const OffsetRanges& off, cudaStream_t st);

// ---- offsets handled by the Woodbury identity (mixed.cpp)
// Lower triangle of (A - offsets) in FP32.
moao_status cvt_lower_minus_offsets(const double* s, long lds, float* d, long ldd, long n,
                                    const int* rid, const OffsetRanges& off, cudaStream_t st);
// Y (ldy x n, column-major, FP32) = indicator rows: Y(w, j) = 1 for j in range w,
// 0 elsewhere (rows off.n .. ldy-1 included).
moao_status fill_range_indicators(float* Y, long ldy, long n, const OffsetRanges& off,
                                  cudaStream_t st);
// out(i, w) = sum over j in range w of Z(i, j), Z m x n column-major; out m x
// off.n column-major (ld m), accumulated in FP64.
moao_status range_sums(const float* Z, long ldz, long m, const OffsetRanges& off, double* out,
                       cudaStream_t st);
moao_status range_sums(const double* Z, long ldz, long m, const OffsetRanges& off, double* out,
                       cudaStream_t st);
// Y2 (k x n, ld k, FP64) = S (k x k, column-major, device) * Y (rows 0..k-1 of ldy x n).
moao_status mul_small_left(const double* S, int k, const float* Y, long ldy, long n, double* Y2,
                           cudaStream_t st);
// R(i, j) (+)= Z(i, j) - sum_w ZU(i, w) Y2(w, j) for an m x n Z (FP32) and R (FP64).
moao_status woodbury_apply(const float* Z, long ldz, long m, long n, const double* ZU, int k,
                           const double* Y2, double* R, long ldr, bool accumulate,
                           cudaStream_t st);
// rid[j] = the range holding index j, or -1.
moao_status fill_range_ids(int* rid, long n, const OffsetRanges& off, cudaStream_t st);
// Sinv (k x k, column-major) = (diag(1 / value) + YU)^-1 on the device, k = off.n;
// sets *bad to 1 when a pivot is zero.
moao_status capacitance_inverse(const double* YU, const OffsetRanges& off, double* Sinv, int* bad,
                                cudaStream_t st);
// E(i, j) -= RU(i, w) value[w] for j in range w (the offsets' part of R*A).
moao_status subtract_offset_products(double* E, long lde, long m, long n, const double* RU,
                                     const int* rid, const OffsetRanges& off, cudaStream_t st);

}  // namespace moao

#endif  // MOAO_MIXED_H
