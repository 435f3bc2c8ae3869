// tcgen05 tensor-core GEMM (see tc_gemm.cu).
#ifndef MOAO_TC_GEMM_H
#define MOAO_TC_GEMM_H

#include <cuda.h>
#include <cuda_runtime.h>

#include "moao_internal.h"

namespace moao {

constexpr int kTcMaxMaps = 6;
constexpr int kTcMaxSegs = 8;
// kTcF16: fp16 operands (kind::f16 like bf16, FP32 accumulation); with
// erow/ecol the FP32 epilogue scales by 2^(erow[r] + ecol[c] + shift), so the
// operands can be stored scaled per row into fp16's range.
enum TcKind { kTcBf16 = 0, kTcI8 = 1, kTcF16 = 2 };
enum TcEpilogue { kTcEpiF32 = 0, kTcEpiF64Scaled = 1, kTcEpiMod8 = 2 };
// kTcEpiMod8 (int8 operands): C (uint8, column-major) = acc mod modulus, in [0, modulus).

// A K-major operand: rows x kcols elements, row stride in elements.
struct TcTensor {
  alignas(64) CUtensorMap map;
  int kind = 0;
  int kstep = 0;     // K elements per pipeline stage (64 bf16, 128 int8)
  int box_rows = 0;  // role: 128 for an A operand, 256 for a B operand
};

// One K segment: A tensor a over K elements [ka, ka + nk*kstep) times B tensor
// b over [kb, kb + nk*kstep).
struct TcSegment {
  int a, b;
  int ka, kb, nk;
  int kstep;  // filled in by tc_gemm
};

struct TcGemm {
  int kind = kTcBf16;
  int epi = kTcEpiF32;
  long M = 0, N = 0;
  const TcTensor* A[kTcMaxMaps] = {};
  int nA = 0;
  const TcTensor* B[kTcMaxMaps] = {};
  int nB = 0;
  TcSegment seg[kTcMaxSegs] = {};
  int nseg = 0;
  int a_row0 = 0, b_row0 = 0;  // rows of A / B that map to C row / column 0
  int lower = 0, diag_off = 0; // only C(r, c) with r + diag_off >= c
  float alpha = 1.f, beta = 0.f;
  void* C = nullptr;           // float (kTcEpiF32), double (kTcEpiF64Scaled) or uint8
                               // (kTcEpiMod8), column-major
  long ldc = 0;
  const int* erow = nullptr;   // kTcEpiF64Scaled: C += acc * 2^(erow[r] + ecol[c] + shift);
                               // kTcEpiF32 (optional): acc scaled the same way
  const int* ecol = nullptr;
  int shift = 0;
  int modulus = 0;             // kTcEpiMod8: 2..256
  int* err = nullptr;          // device flag: nonzero after a bounded wait expired
  int max_ctas = 0;            // cap on the persistent grid (0: one CTA per SM)
  int pair = 0;                // 1: 256 x 256 tiles on clusters of two CTAs where M > 128
                               // (the context's tc_pair, off by default)
  unsigned long long spin_limit = 0;  // polls of each bounded wait (0: 2^28)
};

// Describes a row-major (K-contiguous) device matrix for TMA. The output tile is
// 128 x 256 (256 x 256 on a pair of CTAs): box_rows names the operand's role,
// 128 for A and 256 for B; the TMA boxes are 128 rows either way.
moao_status make_tc_map(TcTensor* t, const void* base, int kind, long long rows, long long kcols,
                        long long row_stride_elems, int box_rows = 128);
moao_status tc_gemm(const TcGemm& g, cudaStream_t s, long long* launches);

}  // namespace moao

#endif  // MOAO_TC_GEMM_H
