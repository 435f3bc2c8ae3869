// Mixed-precision reconstructor: conversion / slicing kernels and the driver.
#ifndef MOAO_MIXED_H
#define MOAO_MIXED_H

#include <cuda_runtime.h>

#include <cstdint>

#include "moao_internal.h"

namespace moao {

constexpr int kMaxOzakiSlices = 6;

moao_status cvt_f32_to_f64(const float* s, long lds, double* d, long ldd, long m, long n,
                           bool lower, cudaStream_t st);
moao_status cvt_f64_to_f32(const double* s, long lds, float* d, long ldd, long m, long n,
                           bool lower, cudaStream_t st);
moao_status add_f32_to_f64(const float* s, long lds, double* d, long ldd, long m, long n,
                           cudaStream_t st);
// hi/lo bf16 split of an FP64 column-major m x n block; row-major targets
// (hi_r, lo_r, row stride ldr) and/or column-major targets (hi_c, lo_c, ldc),
// either pair may be null. Pointers address the block's first element.
moao_status split_bf16(const double* src, long lds, long m, long n, void* hi_r, void* lo_r,
                       long ldr, void* hi_c, void* lo_c, long ldc, cudaStream_t st);
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
