// Mixed-precision reconstructor: conversion / slicing kernels and the driver.
#ifndef MOAO_MIXED_H
#define MOAO_MIXED_H

#include <cuda_runtime.h>

#include <cstdint>

#include "moao_internal.h"

namespace moao {

constexpr int kMaxOzakiSlices = 6;
constexpr int kMaxBfSlices = 3;

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
// int8 slices of the rows of A (m x n, column-major): per-row exponents in e[m],
// slice s at out + s*m*ldo, row-major with row stride ldo.
moao_status ozaki_split_rows(const double* A, long lda, long m, long n, int ns, int* e,
                             int8_t* out, long ldo, cudaStream_t st);
// int8 slices of the columns of sym(A) for a lower-stored n x n A: per-column
// exponents in f[n]; slice s at out + s*n*ldo with row j holding column j.
moao_status ozaki_split_sym(const double* A, long lda, long n, int ns, int* f,
                            unsigned long long* colmax, int8_t* out, long ldo, cudaStream_t st);

}  // namespace moao

#endif  // MOAO_MIXED_H
