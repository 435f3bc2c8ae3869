// Mixed-precision reconstructor R = Ctm Cmm^-1 with FP64 iterative refinement.
//
// Factorisation (right-looking, panel nb, multiple of 64):
//   A32 = float(Cmm) holds the trailing matrix.
//   diagonal block: FP64 Cholesky + inverse (potrf_inv_block), kept in dinv
//   panel: L_panel = double(A32 panel) * Dinv^T in FP64, stored FP32 in A32 and
//          as bf16 slices (3 by default: ~24 significant bits) in two layouts:
//          Lr (row-major, row r = L(r, :)) and Lc (row j = L(:, j)), both K-major
//          operands of the tensor-core GEMM
//   trailing: A32_22 -= L L^T on the lower tiles as the slice products s_i s_j
//          with i + j < slices (6 products for 3 slices, 3 for 2) accumulated in
//          FP32 in TMEM (tc_gemm, one segment per product)
// Solve (R = Ctm L^-T L^-1, right-looking forward then backward): block
//   products with Dinv in FP64, long updates with the bf16 split factor on the
//   tensor cores, state in FP32.
// Refinement: E = Ctm - R sym(Cmm) with the int8 slice products of the Ozaki
//   scheme (exact int32 accumulation, per-diagonal power-of-two scaling into
//   FP64), dR = E (L L^T)^-1 by the mixed solve with the leading slice product
//   only (fp16x2) or 2 bf16 slices (a correction needs ~1e-2 relative accuracy
//   only), R += dR; repeated while ||E||/||Ctm|| is
//   above the tolerance (at most max_refine times).
// Offsets: when the caller declares block-constant offsets of Cmm
// (Cmm = B + U D U^T, U the indicator columns of index ranges, D diagonal; the
// LGS tip-tilt constant of the covariance model is one per LGS and axis), the
// factorisation is of B, whose entries are not dominated by the constants
// (FP32 keeps their low bits), and the solves add the offsets back by the
// Woodbury identity:
//   X M^-1 = Z - (Z U) S^-1 Y,  Z = X M_B^-1,  Y = U^T M_B^-1,  S = D^-1 + Y U.
// The refinement residual takes the product with B from the int8 slices (the
// column scales of B are not set by the constants either) and the offsets'
// part R U D U^T from FP64 range sums of R.
// Cmm is read through its lower triangle and overwritten with the (FP32)
// factor at the end, Ctm with R in FP64, like the FP64 path; with offsets the
// factor written is that of B.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "context.h"
#include "mixed.h"
#include "tc_gemm.h"

namespace moao {
namespace {

long round_up(long x, long a) { return (x + a - 1) / a * a; }

__global__ void sumsq_kernel(const double* __restrict__ A, long lda, long m, long n,
                             double* __restrict__ out) {
  double s = 0;
  const long total = m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const double v = A[(e / m) * lda + e % m];
    s += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

// A (m x n, ld m) += B (m x n, ld m).
__global__ void add_f64_kernel(double* __restrict__ A, const double* __restrict__ B, long total) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x)
    A[e] += B[e];
}

moao_status sumsq(moao_ctx* ctx, const double* A, long lda, long m, long n, double* d_out,
                  double* h_out) {
  MOAO_CUDA_TRY(cudaMemsetAsync(d_out, 0, sizeof(double), ctx->stream));
  sumsq_kernel<<<148 * 4, 256, 0, ctx->stream>>>(A, lda, m, n, d_out);
  ++ctx->launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  MOAO_CUDA_TRY(cudaMemcpyAsync(h_out, d_out, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return MOAO_OK;
}

struct Maps {
  TcTensor lrA[kMaxBfSlices];  // Lr slices as A operands (128-row boxes)
  TcTensor lrB[kMaxBfSlices];  // Lr slices as B operands (256-row boxes)
  TcTensor lcB[kMaxBfSlices];  // Lc slices as B operands
  TcTensor xA[kMaxBfSlices];   // solve-panel slices as A operands (m rows)
  TcTensor yA[kMaxBfSlices];   // the same slices for the 128-row offset solve
  TcTensor pA[kMaxBfSlices];   // the same slices for a factor panel (nmeas rows)
  TcTensor drB[kMaxBfSlices];  // rows of the inverse diagonal blocks (fp16 format)
  TcTensor dcB[kMaxBfSlices];  // columns of the inverse diagonal blocks (fp16 format)
};

constexpr long kYRows = 128;  // rows of the offset-indicator solve (one tile)


// Products s_i * s_j of bf16 slices kept for a given slice count, smallest
// first: the tensor core's FP32 accumulation truncates each addition (a bias of
// ~2^-28 of the running sum per term, measured), so the small correction
// products are summed before the dominant hi*hi product grows the accumulator.
struct Products {
  int n;
  int a[6], b[6];
};
Products products_for(int slices) {
  if (slices >= 3) return Products{6, {2, 1, 0, 1, 0, 0}, {0, 1, 2, 0, 1, 0}};
  if (slices == 1) return Products{1, {0}, {0}};
  return Products{3, {1, 0, 0}, {0, 1, 0}};
}

// Tensor-core update C(f32, M x N, ldc) -= sum_p A_{a_p} B_{b_p}^T over K blocks
// [ka, ka + nk*64) of the A slices and [kb, ...) of the B slices.
moao_status tc_update(moao_ctx* ctx, const TcTensor* A, int a_row0, int ka, const TcTensor* B,
                      int b_row0, int kb, int nk, const Products& pr, long M, long N, float* C,
                      long ldc, bool lower, int* err, double flops, const int* erow = nullptr,
                      const int* ecol = nullptr, int max_ctas = 0) {
  TcGemm g;
  g.max_ctas = max_ctas;
  g.spin_limit = ctx->wait_polls;
  g.pair = ctx->tc_pair;
  g.kind = A[0].kind;
  g.erow = erow;
  g.ecol = ecol;
  g.epi = kTcEpiF32;
  g.M = M;
  g.N = N;
  int na = 0, nbm = 0;
  for (int p = 0; p < pr.n; ++p) {
    na = std::max(na, pr.a[p] + 1);
    nbm = std::max(nbm, pr.b[p] + 1);
  }
  for (int i = 0; i < na; ++i) g.A[i] = &A[i];
  for (int i = 0; i < nbm; ++i) g.B[i] = &B[i];
  g.nA = na;
  g.nB = nbm;
  for (int p = 0; p < pr.n; ++p) g.seg[p] = TcSegment{pr.a[p], pr.b[p], ka, kb, nk, 0};
  g.nseg = pr.n;
  g.a_row0 = a_row0;
  g.b_row0 = b_row0;
  g.lower = lower ? 1 : 0;
  g.alpha = -1.f;
  g.beta = 1.f;
  g.C = C;
  g.ldc = ldc;
  g.err = err;
  KernelTimer kt(ctx, "tc_split", flops * pr.n);
  return tc_gemm(g, ctx->stream, &ctx->launches);
}

// SMs left to the next diagonal block beside the rest of the trailing update:
// ctx->lookahead_sms while the update is long, growing to ctx->lookahead_max as
// the trailing matrix shrinks (below 24,576 rows the update no longer outlasts
// the diagonal block, whose small GEMMs then set the pace).
int lookahead_for(const moao_ctx* ctx, long rest) {
  const int base = ctx->lookahead_sms, top = std::max(base, ctx->lookahead_max);
  if (rest >= 24576) return base;
  if (rest >= 12288) return std::min(top, std::max(base, (base + top) / 2));
  return top;
}

// fp16 operands: power-of-two scales of the stored factor and solve slices.
//   erp: per panel p, the row exponents of L(:, panel p) (erp + p*n, indexed by row)
//   ecf: per column j of L, its exponent (the Lc copy, row j = L(:, j))
//   ex:  row exponents of the current solve block
struct Scales {
  bool f16 = false;
  int* erp = nullptr;
  int* ecf = nullptr;
  int* ex = nullptr;
  int* edr = nullptr;  // row exponents of the inverse diagonal blocks (indexed by global row)
  int* edc = nullptr;  // column exponents of the inverse diagonal blocks
};
constexpr int kF16Bias = 14;  // stored slices below 2^14 in magnitude (fp16 max 65504)

// Slices of an m x kb solve block (column-major, leading dimension lds) into xr
// for the tensor core: fp16 slices straight from the FP32 state, or bf16 slices
// of an FP64 block.
template <typename T>
moao_status split_block(const Scales& sc, const T* src, long lds, long m, long kb, int slices,
                        const BfSlices& xr, long ldx, cudaStream_t s) {
  BfSlices none{};
  const long kpad = std::min(round_up(kb, 64), ldx);
  if constexpr (std::is_same<T, float>::value) {
    if (sc.f16 && kb <= 1024)  // exponents, slices and zero padding in one pass
      return split_rows_f16(src, lds, m, kb, slices, xr, ldx, kpad, sc.ex, kF16Bias, s);
  }
  if (kpad > kb)  // the tensor core reads K in steps of 64: padding columns must hold zeros
    for (int k = 0; k < slices; ++k)
      MOAO_CUDA_TRY(cudaMemset2DAsync(static_cast<uint16_t*>(xr.p[k]) + kb, ldx * sizeof(uint16_t),
                                      0, (kpad - kb) * sizeof(uint16_t), m, s));
  if (!sc.f16) {
    if constexpr (std::is_same<T, double>::value)
      return split_bf16(src, lds, m, kb, slices, xr, ldx, none, 0, s);
    else
      return set_error(MOAO_ERR_UNSUPPORTED, "bf16 split of an FP32 block");
  }
  MOAO_TRY(scale_exponents(src, lds, m, kb, kF16Bias, sc.ex, nullptr, s));
  return split_f16(src, lds, m, kb, slices, xr, ldx, sc.ex, none, 0, nullptr, s);
}

// fp16 format: C32 (m x kb, ldc) = W (m x kb, FP32, ldw; C32 itself is allowed)
// times the inverse diagonal block starting at row k0, transposed (forward:
// Dinv^T, rows of the drB copy) or not (backward: Dinv, rows of the dcB copy),
// on the tensor cores.
moao_status block_product(moao_ctx* ctx, const Scales& sc, const TcTensor* A, const float* W,
                          long ldw, long m, long k0, long kb, const TcTensor* B, const int* eB,
                          const Products& pr, float* C32, long ldc, const BfSlices& xr, long ldx,
                          int slices, int* err) {
  MOAO_TRY(split_block(sc, W, ldw, m, kb, slices, xr, ldx, ctx->stream));
  TcGemm g;
  g.spin_limit = ctx->wait_polls;
  g.pair = ctx->tc_pair;
  g.kind = A[0].kind;
  g.epi = kTcEpiF32;
  g.M = m;
  g.N = kb;
  int na = 0, nbm = 0;
  for (int p = 0; p < pr.n; ++p) {
    na = std::max(na, pr.a[p] + 1);
    nbm = std::max(nbm, pr.b[p] + 1);
  }
  for (int i = 0; i < na; ++i) g.A[i] = &A[i];
  for (int i = 0; i < nbm; ++i) g.B[i] = &B[i];
  g.nA = na;
  g.nB = nbm;
  for (int p = 0; p < pr.n; ++p)
    g.seg[p] = TcSegment{pr.a[p], pr.b[p], 0, 0, (int)((kb + 63) / 64), 0};
  g.nseg = pr.n;
  g.b_row0 = (int)k0;
  g.alpha = 1.f;
  g.beta = 0.f;
  g.C = C32;
  g.ldc = ldc;
  g.erow = sc.ex;
  g.ecol = eB + k0;
  g.err = err;
  KernelTimer kt(ctx, "tc_split", 2.0 * m * kb * kb * pr.n);
  return tc_gemm(g, ctx->stream, &ctx->launches);
}

// In-place mixed solve on T32 (m x n, ld m): T <- T L^-T L^-1, with the long
// updates as the given slice products.
moao_status mixed_solve(moao_ctx* ctx, long n, long m, float* T32, const double* dinv,
                        const TcTensor* xA, const Maps& mp, double* W1, double* W2,
                        void* const* xs, long ldx, const Products& pr, int slices, int* err,
                        const Scales& sc) {
  const long nb = ctx->nb;
  cudaStream_t s = ctx->stream;
  BfSlices xr{};
  for (int k = 0; k < slices; ++k) xr.p[k] = xs[k];
  for (long k0 = 0; k0 < n; k0 += nb) {
    const long kb = std::min(nb, n - k0);
    float* Tk = T32 + k0 * m;
    if (sc.f16) {
      MOAO_TRY(block_product(ctx, sc, xA, Tk, m, m, k0, kb, mp.drB, sc.edr, pr, Tk, m, xr, ldx,
                             slices, err));
    } else {
      MOAO_TRY(cvt_f32_to_f64(Tk, m, W1, m, m, kb, false, s));
      MOAO_TRY(gemm(ctx, m, kb, kb, 1.0, W1, m, dinv + k0, n, true, 0.0, W2, m));
      MOAO_TRY(cvt_f64_to_f32(W2, m, Tk, m, m, kb, false, s));
    }
    const long rest = n - k0 - kb;
    if (rest > 0) {
      if (sc.f16) MOAO_TRY(split_block(sc, (const float*)Tk, m, m, kb, slices, xr, ldx, s));
      else MOAO_TRY(split_block(sc, (const double*)W2, m, m, kb, slices, xr, ldx, s));
      MOAO_TRY(tc_update(ctx, xA, 0, 0, mp.lrB, (int)(k0 + kb), (int)k0, (int)((kb + 63) / 64),
                         pr, m, rest, T32 + (k0 + kb) * m, m, false, err, 2.0 * m * rest * kb,
                         sc.f16 ? sc.ex : nullptr,
                         sc.f16 ? sc.erp + (k0 / nb) * n + (k0 + kb) : nullptr));
    }
  }
  const long nblk = (n + nb - 1) / nb;
  for (long b = nblk - 1; b >= 0; --b) {
    const long k0 = b * nb, kb = std::min(nb, n - k0);
    float* Tk = T32 + k0 * m;
    if (sc.f16) {
      MOAO_TRY(block_product(ctx, sc, xA, Tk, m, m, k0, kb, mp.dcB, sc.edc, pr, Tk, m, xr, ldx,
                             slices, err));
    } else {
      MOAO_TRY(cvt_f32_to_f64(Tk, m, W1, m, m, kb, false, s));
      MOAO_TRY(gemm(ctx, m, kb, kb, 1.0, W1, m, dinv + k0, n, false, 0.0, W2, m));
      MOAO_TRY(cvt_f64_to_f32(W2, m, Tk, m, m, kb, false, s));
    }
    if (k0 > 0) {
      if (sc.f16) MOAO_TRY(split_block(sc, (const float*)Tk, m, m, kb, slices, xr, ldx, s));
      else MOAO_TRY(split_block(sc, (const double*)W2, m, m, kb, slices, xr, ldx, s));
      MOAO_TRY(tc_update(ctx, xA, 0, 0, mp.lcB, 0, (int)k0, (int)((kb + 63) / 64), pr, m, k0,
                         T32, m, false, err, 2.0 * m * k0 * kb, sc.f16 ? sc.ex : nullptr,
                         sc.f16 ? sc.ecf : nullptr));
    }
  }
  return MOAO_OK;
}

}  // namespace

// C (FP64, M x N, ldc) += alpha * A B^T from int8 slices (Ozaki splitting):
// ta[0..nsa) hold the slices of A's rows (128-row boxes), tb[0..nsb) those of
// B's rows (256-row boxes), K columns each, slice s of a row with exponent e
// holding digits of x * 2^(6 - e) * 128^s. The products of slices p and q
// (0-based) with p + q + 2 <= dmax are accumulated exactly in int32 on the
// tensor cores and added in FP64 scaled by 2^(erow[r] + ecol[c] - 12 -
// 7 (p + q)): one launch per anti-diagonal p + q, split where the int32 sum
// could overflow (|digit| <= 64, so 4096 K per product).
moao_status ozaki_gemm(moao_ctx* ctx, const TcTensor* ta, int nsa, const TcTensor* tb, int nsb,
                       int dmax, long M, long N, long K, float alpha, double* C, long ldc,
                       const int* erow, const int* ecol, int* err) {
  if (nsa < 1 || nsa > kMaxOzakiSlices || nsb < 1 || nsb > kMaxOzakiSlices)
    return set_error(MOAO_ERR_BAD_ARG, "ozaki_gemm: slice counts");
  const long pair_cap = std::min<long>(
      kTcMaxSegs, std::max(1L, (long)(2147483647.0 / (4096.0 * (double)std::max(K, 1L)))));
  for (int d = 2; d <= dmax; ++d) {
    std::vector<std::pair<int, int>> pairs;
    for (int p = 1; p <= nsa; ++p)
      if (d - p >= 1 && d - p <= nsb) pairs.push_back({p - 1, d - p - 1});
    for (size_t b0 = 0; b0 < pairs.size(); b0 += pair_cap) {
      TcGemm g;
      g.spin_limit = ctx->wait_polls;
      g.pair = ctx->tc_pair;
      g.kind = kTcI8;
      g.epi = kTcEpiF64Scaled;
      g.M = M;
      g.N = N;
      for (int i = 0; i < nsa; ++i) g.A[i] = &ta[i];
      for (int i = 0; i < nsb; ++i) g.B[i] = &tb[i];
      g.nA = nsa;
      g.nB = nsb;
      const size_t b1 = std::min(pairs.size(), b0 + (size_t)pair_cap);
      for (size_t q = b0; q < b1; ++q)
        g.seg[g.nseg++] = TcSegment{pairs[q].first, pairs[q].second, 0, 0, (int)((K + 127) / 128), 0};
      g.alpha = alpha;
      g.C = C;
      g.ldc = ldc;
      g.erow = erow;
      g.ecol = ecol;
      g.shift = -12 - 7 * (d - 2);
      g.err = err;
      KernelTimer kt(ctx, "tc_int8", 2.0 * M * (double)N * K * (double)(b1 - b0));
      MOAO_TRY(tc_gemm(g, ctx->stream, &ctx->launches));
    }
  }
  return MOAO_OK;
}

// One int8 GEMM per modulus (exact int32 sums, K < 2^17), reduced modulo it in
// the epilogue.
moao_status crt_gemm(moao_ctx* ctx, const TcTensor* ta, const TcTensor* tb, int nmod, long M,
                     long N, long K, uint8_t* Z, int* err) {
  if (nmod < 2 || nmod > kCrtMaxModuli || K >= (1L << 17))
    return set_error(MOAO_ERR_BAD_ARG, "crt_gemm: moduli or K");
  for (int i = 0; i < nmod; ++i) {
    TcGemm g;
    g.spin_limit = ctx->wait_polls;
    g.pair = ctx->tc_pair;
    g.kind = kTcI8;
    g.epi = kTcEpiMod8;
    g.modulus = kCrtMod[i];
    g.M = M;
    g.N = N;
    g.A[0] = &ta[i];
    g.B[0] = &tb[i];
    g.nA = g.nB = 1;
    g.seg[0] = TcSegment{0, 0, 0, 0, (int)((K + 127) / 128), 0};
    g.nseg = 1;
    g.C = Z + (size_t)i * M * N;
    g.ldc = M;
    g.err = err;
    KernelTimer kt(ctx, "tc_int8", 2.0 * M * (double)N * K);
    MOAO_TRY(tc_gemm(g, ctx->stream, &ctx->launches));
  }
  return MOAO_OK;
}

MixedSizes mixed_sizes(long n, long m, long nb, int nsl, int ns, int nranges, bool crt) {
  const long ldn = round_up(n, 64), ldq = round_up(n, 128);
  MixedSizes z;
  z.nmod = crt ? crt_moduli_for(ns, n) : 0;
  z.a32 = sizeof(float) * (size_t)n * n;
  z.lr = nsl * sizeof(uint16_t) * (size_t)n * ldn;
  z.t32 = sizeof(float) * (size_t)m * n;
  z.w = sizeof(double) * (size_t)std::max(n, m) * nb;
  z.x = nsl * sizeof(uint16_t) * (size_t)std::max(n, m) * nb;
  z.r64 = sizeof(double) * (size_t)m * n;
  z.qa = (size_t)ns * m * ldq;  // the slices of R_k stay for a Cee from the refinement
  z.qb = z.nmod ? 0 : (size_t)ns * n * ldq;
  z.qr = (size_t)z.nmod * m * ldq;
  z.qs = (size_t)z.nmod * n * ldq;
  z.z = (size_t)z.nmod * m * n;
  z.ea = sizeof(int) * (size_t)m;
  z.fb = sizeof(int) * (size_t)n;
  z.colmax = sizeof(unsigned long long) * (size_t)n;
  z.norm = sizeof(double) * 2;
  z.dinv = sizeof(double) * (size_t)std::max(n, 1L) * nb;
  z.info = 3 * sizeof(int);
  z.exps = sizeof(int) * ((size_t)((n + nb - 1) / nb) * n + (size_t)n +
                          (size_t)std::max(std::max(m, n), 128L) + 2 * (size_t)n);
  z.dsl = 2 * nsl * sizeof(uint16_t) * (size_t)n * nb;
  if (nranges > 0)
    z.offsets = sizeof(int) * (size_t)n + sizeof(float) * (size_t)128 * n +
                sizeof(double) * ((size_t)nranges * n + (size_t)std::max(m, (long)nranges) * nranges +
                                  (size_t)nranges * nranges);
  return z;
}

// Adds the helper kernels launched during its lifetime to the context's count.
struct HelperCount {
  moao_ctx* ctx;
  long long h0 = helper_launches();
  explicit HelperCount(moao_ctx* c) : ctx(c) {}
  ~HelperCount() { ctx->launches += helper_launches() - h0; }
};

moao_status reconstructor_mixed(moao_ctx* ctx, long n, long m, double* Cmm, long ldCmm,
                                double* Ctm, long ldCtm, bool reuse, moao_solve_report* rep) {
  HelperCount hc(ctx);
  const long nb = ctx->nb;
  cudaStream_t s = ctx->stream;
  const long ldn = round_up(n, 64);    // bf16 row stride of the factor copies
  const long ldq = round_up(n, 128);   // int8 row stride of the slices
  const int ns = ctx->ozaki_slices;
  const long ldx = nb;
  // ---- workspace
  const bool f16 = ctx->factor_format == MOAO_FACTOR_F16X2;
  const int tck = f16 ? kTcF16 : kTcBf16;
  const int nsl = f16 ? 2 : std::max(2, std::min(kMaxBfSlices, ctx->bf16_slices));
  const MixedSizes z = mixed_sizes(n, m, nb, nsl, ns, ctx->offsets.n, ctx->residual_crt != 0);
  const int nmod = z.nmod;  // > 0: the residual by CRT products
  MOAO_TRY(ctx->mx_a32.ensure(z.a32));
  MOAO_TRY(ctx->mx_lr.ensure(z.lr));
  MOAO_TRY(ctx->mx_lc.ensure(z.lr));
  MOAO_TRY(ctx->mx_t32.ensure(z.t32));
  MOAO_TRY(ctx->mx_w1.ensure(z.w));
  MOAO_TRY(ctx->mx_w2.ensure(z.w));
  MOAO_TRY(ctx->mx_x.ensure(z.x));
  MOAO_TRY(ctx->mx_r64.ensure(z.r64));
  MOAO_TRY(ctx->mx_e64.ensure(z.r64));
  MOAO_TRY(ctx->mx_qa.ensure(z.qa));
  MOAO_TRY(ctx->mx_qb.ensure(z.qb));
  MOAO_TRY(ctx->mx_qr.ensure(z.qr));
  MOAO_TRY(ctx->mx_qs.ensure(z.qs));
  MOAO_TRY(ctx->mx_z.ensure(z.z));
  MOAO_TRY(ctx->mx_ea.ensure(z.ea));
  MOAO_TRY(ctx->mx_fb.ensure(z.fb));
  MOAO_TRY(ctx->mx_colmax.ensure(z.colmax));
  MOAO_TRY(ctx->mx_norm.ensure(z.norm));
  MOAO_TRY(ctx->ws_dinv.ensure(z.dinv));
  MOAO_TRY(ctx->ws_w.ensure(z.dinv));
  MOAO_TRY(ctx->ws_info.ensure(z.info));
  MOAO_TRY(ctx->mx_exps.ensure(z.exps));
  Scales sc;
  sc.f16 = f16;
  sc.erp = ctx->mx_exps.as<int>();
  sc.ecf = sc.erp + (size_t)((n + nb - 1) / nb) * n;
  sc.ex = sc.ecf + n;
  sc.edr = sc.ex + std::max(std::max(m, n), 128L);
  sc.edc = sc.edr + n;
  uint16_t *dr = nullptr, *dcl = nullptr;  // inverse diagonal blocks: row / column copies
  if (f16) {
    MOAO_TRY(ctx->mx_dsl.ensure(z.dsl));
    dr = ctx->mx_dsl.as<uint16_t>();
    dcl = dr + (size_t)nsl * n * nb;
  }
  float* A32 = ctx->mx_a32.as<float>();
  uint16_t* lr = ctx->mx_lr.as<uint16_t>();
  uint16_t* lc = ctx->mx_lc.as<uint16_t>();
  void* xs[kMaxBfSlices] = {};
  for (int k = 0; k < nsl; ++k)
    xs[k] = ctx->mx_x.as<uint16_t>() + (size_t)k * std::max(n, m) * ldx;
  float* T32 = ctx->mx_t32.as<float>();
  double* W1 = ctx->mx_w1.as<double>();
  double* W2 = ctx->mx_w2.as<double>();
  double* R64 = ctx->mx_r64.as<double>();
  double* E64 = ctx->mx_e64.as<double>();
  int8_t* qa = ctx->mx_qa.as<int8_t>();
  int8_t* qb = ctx->mx_qb.as<int8_t>();
  int8_t* qr = ctx->mx_qr.as<int8_t>();
  int8_t* qs = ctx->mx_qs.as<int8_t>();
  uint8_t* Zr = ctx->mx_z.as<uint8_t>();
  int* ea = ctx->mx_ea.as<int>();
  int* fb = ctx->mx_fb.as<int>();
  double* dinv = ctx->ws_dinv.as<double>();
  int* d_info = ctx->ws_info.as<int>();
  int* err = d_info + 1;

  // ---- declared offsets of Cmm (Woodbury)
  const OffsetRanges& off = ctx->offsets;
  const int nro = off.n;  // offset ranges
  for (int w = 0; w < nro; ++w)
    if (off.end[w] > n)
      return set_error(MOAO_ERR_BAD_ARG, "mixed reconstructor: an offset range ends beyond nmeas");
  int* rid = nullptr;
  float* Y32 = nullptr;
  double *Y2 = nullptr, *ZU = nullptr, *Sinv = nullptr;
  if (nro > 0) {
    MOAO_TRY(ctx->mx_rid.ensure(sizeof(int) * (size_t)n));
    MOAO_TRY(ctx->mx_y.ensure(sizeof(float) * (size_t)kYRows * n));
    MOAO_TRY(ctx->mx_y2.ensure(sizeof(double) * (size_t)nro * n));
    MOAO_TRY(ctx->mx_zu.ensure(sizeof(double) * (size_t)std::max(m, (long)nro) * nro));
    MOAO_TRY(ctx->mx_sinv.ensure(sizeof(double) * (size_t)nro * nro));
    rid = ctx->mx_rid.as<int>();
    Y32 = ctx->mx_y.as<float>();
    Y2 = ctx->mx_y2.as<double>();
    ZU = ctx->mx_zu.as<double>();
    Sinv = ctx->mx_sinv.as<double>();
  }

  Maps mp;
  for (int k = 0; k < nsl; ++k) {
    uint16_t* lrk = lr + (size_t)k * n * ldn;
    uint16_t* lck = lc + (size_t)k * n * ldn;
    MOAO_TRY(make_tc_map(&mp.lrA[k], lrk, tck, n, n, ldn));
    MOAO_TRY(make_tc_map(&mp.lrB[k], lrk, tck, n, n, ldn, 256));
    MOAO_TRY(make_tc_map(&mp.lcB[k], lck, tck, n, n, ldn, 256));
    MOAO_TRY(make_tc_map(&mp.xA[k], xs[k], tck, m, nb, ldx));
    MOAO_TRY(make_tc_map(&mp.yA[k], xs[k], tck, kYRows, nb, ldx));
    if (f16) {
      MOAO_TRY(make_tc_map(&mp.pA[k], xs[k], tck, n, nb, ldx));
      MOAO_TRY(make_tc_map(&mp.drB[k], dr + (size_t)k * n * nb, tck, n, nb, nb, 256));
      MOAO_TRY(make_tc_map(&mp.dcB[k], dcl + (size_t)k * n * nb, tck, n, nb, nb, 256));
    }
  }
  BfSlices xsl{};
  for (int k = 0; k < nsl; ++k) xsl.p[k] = xs[k];
  // The correction dR only needs ~1e-2 relative accuracy: with fp16x2 the leading
  // slice product alone (11 bits per operand row) gives the same R at ELT size
  // (rel-Fro 4.23e-6 against 4.21e-6 with 3 products) for a third of the work.
  const int csl = ctx->corr_slices > 0 ? std::max(1, std::min(nsl, ctx->corr_slices)) : (f16 ? 1 : 2);
  const Products full = products_for(nsl), corr = products_for(csl);

  // In graph mode (stream capture) nothing here waits for the device or reads
  // device memory on the host: failures stay in d_info[0..2] for the caller and
  // refinement runs exactly max_refine corrections.
  const bool graph = ctx->graph_mode;
  cudaEvent_t* ev = ctx->ev;
  if (!graph) cudaEventRecord(ev[3], s);
  if (!reuse || ctx->mx_factored_n != n) {
    MOAO_CUDA_TRY(cudaMemsetAsync(d_info, 0, 3 * sizeof(int), s));
    if (nro > 0) MOAO_TRY(fill_range_ids(rid, n, off, s));
    MOAO_TRY(cvt_lower_minus_offsets(Cmm, ldCmm, A32, n, n, rid, off, s));
    // the ragged last diagonal block leaves K columns of its copies unused: zeros
    if (f16) MOAO_CUDA_TRY(cudaMemsetAsync(dr, 0, z.dsl, s));
    // Diagonal block at k0: FP64 factor and inverse (dinv), FP32 factor back into
    // A32, fp16 copies of the inverse. Runs on stream st.
    auto diag_block = [&](long k0, long kb, cudaStream_t st) -> moao_status {
      cudaStream_t keep = ctx->stream;
      ctx->stream = st;  // potrf_inv_block launches on the context's stream
      float* Akk = A32 + k0 + k0 * n;
      moao_status r = cvt_f32_to_f64(Akk, n, W1, kb, kb, kb, true, st);
      if (r == MOAO_OK)
        r = potrf_inv_block(ctx, W1, kb, dinv + k0, n, kb, k0, d_info, ctx->ws_w.as<double>());
      if (r == MOAO_OK) r = cvt_f64_to_f32(W1, kb, Akk, n, kb, kb, true, st);
      if (r == MOAO_OK && f16) {
        // fp16 copies of the inverse diagonal block: its rows (for X Dinv^T) and its
        // columns (for X Dinv), each scaled by a power of two per row
        BfSlices br{}, bc{};
        for (int k = 0; k < nsl; ++k) {
          br.p[k] = dr + (size_t)k * n * nb + (size_t)k0 * nb;
          bc.p[k] = dcl + (size_t)k * n * nb + (size_t)k0 * nb;
        }
        r = scale_exponents(dinv + k0, n, kb, kb, kF16Bias, sc.edr + k0, sc.edc + k0, st);
        if (r == MOAO_OK)
          r = split_f16(dinv + k0, n, kb, kb, nsl, br, nb, sc.edr + k0, bc, nb, sc.edc + k0, st);
      }
      ctx->stream = keep;
      return r;
    };
    // Lookahead (not under capture): once the trailing update has reached the next
    // panel's columns, that panel's diagonal block is factored on the side stream
    // while the rest of the update leaves ctx->lookahead_sms SMs to it.
    const bool ahead = ctx->lookahead_sms > 0 && !graph;
    if (ahead && !ctx->aux) {
      int lo = 0, hi = 0;
      MOAO_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&lo, &hi));
      MOAO_CUDA_TRY(cudaStreamCreateWithPriority(&ctx->aux, cudaStreamNonBlocking, hi));
      for (auto& e : ctx->la_ev)
        MOAO_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    int nsm = 148;
    MOAO_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
    MOAO_TRY(diag_block(0, std::min(nb, n), s));
    for (long k0 = 0; k0 < n; k0 += nb) {
      const long kb = std::min(nb, n - k0);
      const long rest = n - k0 - kb;
      if (rest <= 0) break;
      float* P = A32 + (k0 + kb) + k0 * n;
      if (f16) {
        // panel P <- P Dinv^T on the tensor cores, in place
        MOAO_TRY(block_product(ctx, sc, mp.pA, P, n, rest, k0, kb, mp.drB, sc.edr, full, P, n, xsl,
                               ldx, nsl, err));
      } else {
        MOAO_TRY(cvt_f32_to_f64(P, n, W1, rest, rest, kb, false, s));
        MOAO_TRY(gemm(ctx, rest, kb, kb, 1.0, W1, rest, dinv + k0, n, true, 0.0, W2, rest));
        MOAO_TRY(cvt_f64_to_f32(W2, rest, P, n, rest, kb, false, s));
      }
      BfSlices rr{}, cc{};
      for (int k = 0; k < nsl; ++k) {
        rr.p[k] = lr + (size_t)k * n * ldn + (k0 + kb) * ldn + k0;
        cc.p[k] = lc + (size_t)k * n * ldn + k0 * ldn + (k0 + kb);
      }
      const int* er = nullptr;
      if (f16) {
        int* erk = sc.erp + (k0 / nb) * n + (k0 + kb);  // rows k0+kb.. of panel k0/nb
        MOAO_TRY(scale_exponents((const float*)P, n, rest, kb, kF16Bias, erk, sc.ecf + k0, s));
        MOAO_TRY(split_f16((const float*)P, n, rest, kb, nsl, rr, ldn, erk, cc, ldn, sc.ecf + k0, s));
        er = erk;
      } else {
        MOAO_TRY(split_bf16(W2, rest, rest, kb, nsl, rr, ldn, cc, ldn, s));
      }
      const long k1 = k0 + kb, kb1 = std::min(nb, rest);
      const int nk = (int)(kb / 64);
      if (ahead && rest > kb1) {
        // the next panel's columns first, then its diagonal block beside the rest
        MOAO_TRY(tc_update(ctx, mp.lrA, (int)k1, (int)k0, mp.lrB, (int)k1, (int)k0, nk, full, rest,
                           kb1, A32 + k1 + k1 * n, n, true, err,
                           (double)(2 * rest - kb1) * kb1 * kb, er, er));
        MOAO_CUDA_TRY(cudaEventRecord(ctx->la_ev[0], s));
        MOAO_CUDA_TRY(cudaStreamWaitEvent(ctx->aux, ctx->la_ev[0], 0));
        MOAO_TRY(diag_block(k1, kb1, ctx->aux));
        MOAO_CUDA_TRY(cudaEventRecord(ctx->la_ev[1], ctx->aux));
        const long r2 = rest - kb1;
        MOAO_TRY(tc_update(ctx, mp.lrA, (int)(k1 + kb1), (int)k0, mp.lrB, (int)(k1 + kb1), (int)k0,
                           nk, full, r2, r2, A32 + (k1 + kb1) + (k1 + kb1) * n, n, true, err,
                           (double)r2 * r2 * kb, er ? er + kb1 : nullptr, er ? er + kb1 : nullptr,
                           std::max(1, nsm - lookahead_for(ctx, rest))));
        MOAO_CUDA_TRY(cudaStreamWaitEvent(s, ctx->la_ev[1], 0));
      } else {
        MOAO_TRY(tc_update(ctx, mp.lrA, (int)k1, (int)k0, mp.lrB, (int)k1, (int)k0, nk, full, rest,
                           rest, A32 + k1 + k1 * n, n, true, err, (double)rest * rest * kb, er, er));
        MOAO_TRY(diag_block(k1, kb1, s));
      }
    }
    if (!graph) {
      int info[2] = {0, 0};
      MOAO_CUDA_TRY(cudaMemcpyAsync(info, d_info, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      MOAO_CUDA_TRY(cudaStreamSynchronize(s));
      if (info[1]) return set_error(MOAO_ERR_TIMEOUT, "tensor-core update: bounded wait expired");
      rep->info = info[0];
      if (info[0]) {
        ctx->mx_factored_n = -1;
        return set_error(MOAO_ERR_NOT_SPD, "mixed Cholesky: non-positive pivot at column " +
                                               std::to_string(info[0]));
      }
    }
    // int8 slices (or CRT residues) of sym(Cmm) for the refinement residual
    if (nmod)
      MOAO_TRY(crt_split_sym(Cmm, ldCmm, n, ns, nmod, fb, ctx->mx_colmax.as<unsigned long long>(),
                             qs, ldq, rid, off, s));
    else
      MOAO_TRY(ozaki_split_sym(Cmm, ldCmm, n, ns, fb, ctx->mx_colmax.as<unsigned long long>(), qb,
                               ldq, rid, off, s));
    if (nro > 0) {
      // Y = U^T M_B^-1 (one 128-row solve), S = D^-1 + Y U, Y2 = S^-1 Y
      MOAO_TRY(fill_range_indicators(Y32, kYRows, n, off, s));
      MOAO_TRY(mixed_solve(ctx, n, kYRows, Y32, dinv, mp.yA, mp, W1, W2, xs, ldx, full, nsl, err,
                           sc));
      MOAO_TRY(range_sums(Y32, kYRows, nro, off, ZU, s));
      MOAO_TRY(capacitance_inverse(ZU, off, Sinv, d_info + 2, s));
      MOAO_TRY(mul_small_left(Sinv, nro, Y32, kYRows, n, Y2, s));
    }
    ctx->mx_factored_n = n;
    // Cmm is not read after its int8 slices: a host-buffer caller without an
    // accuracy target (whose fallback would need Cmm) gets the factor now, its
    // copy back overlapping the solves
    if (ctx->host_factor && !(ctx->acc_target > 0) && !ctx->keep_cmm && !graph) {
      MOAO_TRY(cvt_f32_to_f64(A32, n, Cmm, ldCmm, n, n, true, s));
      MOAO_TRY(factor_to_host(ctx, Cmm, ldCmm, n));
      ctx->factor_done = true;
    }
  }
  if (!graph) cudaEventRecord(ev[4], s);
  // ---- solve
  MOAO_TRY(await_inputs(ctx));
  MOAO_TRY(cvt_f64_to_f32(Ctm, ldCtm, T32, m, m, n, false, s));
  MOAO_TRY(mixed_solve(ctx, n, m, T32, dinv, mp.xA, mp, W1, W2, xs, ldx, full, nsl, err, sc));
  if (nro > 0) {
    MOAO_TRY(range_sums(T32, m, m, off, ZU, s));
    MOAO_TRY(woodbury_apply(T32, m, m, n, ZU, nro, Y2, R64, m, false, s));
  } else {
    MOAO_TRY(cvt_f32_to_f64(T32, m, R64, m, m, n, false, s));
  }
  if (!graph) cudaEventRecord(ev[5], s);
  // ---- refinement
  TcTensor ta[kCrtMaxModuli], tb[kCrtMaxModuli];
  if (nmod) {
    for (int i = 0; i < nmod; ++i) {
      MOAO_TRY(make_tc_map(&ta[i], qr + (size_t)i * m * ldq, kTcI8, m, n, ldq));
      MOAO_TRY(make_tc_map(&tb[i], qs + (size_t)i * n * ldq, kTcI8, n, n, ldq, 256));
    }
  } else {
    for (int i = 0; i < ns; ++i) {
      MOAO_TRY(make_tc_map(&ta[i], qa + (size_t)i * m * ldq, kTcI8, m, n, ldq));
      MOAO_TRY(make_tc_map(&tb[i], qb + (size_t)i * n * ldq, kTcI8, n, n, ldq, 256));
    }
  }
  double* dnorm = ctx->mx_norm.as<double>();
  double ctm2 = 0, e2 = 0;
  if (!graph) MOAO_TRY(sumsq(ctx, Ctm, ldCtm, m, n, dnorm, &ctm2));
  ctx->rstate_valid = false;
  bool ran_residual = false;
  auto residual = [&]() -> moao_status {
    ran_residual = true;
    // E = Ctm - R sym(Cmm): exact CRT products of the ns-slice operands, or
    // the int8 slice products (the slices of R_k are kept either way for a
    // Cee from this refinement)
    MOAO_TRY(ozaki_split_rows(R64, m, m, n, ns, ea, qa, ldq, s));
    if (nmod) {
      MOAO_TRY(crt_split_rows(R64, m, m, n, ns, nmod, ea, qr, ldq, s));
      MOAO_TRY(crt_gemm(ctx, ta, tb, nmod, m, n, n, Zr, err));
      MOAO_TRY(crt_combine(Zr, m, n, nmod, ns, ea, fb, Ctm, ldCtm, -1.0, E64, m, s));
    } else {
      MOAO_CUDA_TRY(cudaMemcpy2DAsync(E64, m * sizeof(double), Ctm, ldCtm * sizeof(double),
                                      m * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
      MOAO_TRY(ozaki_gemm(ctx, ta, ns, tb, ns, ns + 1, m, n, n, -1.f, E64, m, ea, fb, err));
    }
    if (nro > 0) {  // the offsets' part of R Cmm
      MOAO_TRY(range_sums(R64, m, m, off, ZU, s));
      MOAO_TRY(subtract_offset_products(E64, m, m, n, ZU, rid, off, s));
    }
    if (!graph) {
      MOAO_TRY(sumsq(ctx, E64, m, m, n, dnorm, &e2));
      rep->refine_resid = std::sqrt(e2 / std::max(ctm2, 1e-300));
    }
    return MOAO_OK;
  };
  // Accuracy guard (ctx->acc_target > 0, not under capture): the error of the
  // returned R is estimated as ||dR|| / ||R|| of the last correction (the error
  // of R before it) times the residual's reduction by that correction, which
  // needs the residual once more at the end. A miss is reported in
  // rep->fallback and R is not written: the caller runs the FP64 path.
  const bool guard = ctx->acc_target > 0 && !graph;
  double r_before = -1.0, dr2 = 0.0;
  int steps = 0;
  for (; steps < ctx->max_refine; ++steps) {
    MOAO_TRY(residual());
    if (!graph && rep->refine_resid <= ctx->refine_tol) break;
    r_before = rep->refine_resid;
    MOAO_TRY(cvt_f64_to_f32(E64, m, T32, m, m, n, false, s));
    MOAO_TRY(mixed_solve(ctx, n, m, T32, dinv, mp.xA, mp, W1, W2, xs, ldx, corr, csl, err, sc));
    if (guard) {
      // the correction in FP64 in E64 (free until the next residual), its norm, R += it
      if (nro > 0) {
        MOAO_TRY(range_sums(T32, m, m, off, ZU, s));
        MOAO_TRY(woodbury_apply(T32, m, m, n, ZU, nro, Y2, E64, m, false, s));
      } else {
        MOAO_TRY(cvt_f32_to_f64(T32, m, E64, m, m, n, false, s));
      }
      MOAO_TRY(sumsq(ctx, E64, m, m, n, dnorm, &dr2));
      add_f64_kernel<<<148 * 8, 256, 0, s>>>(R64, E64, m * n);
      ++ctx->launches;
      MOAO_CUDA_TRY(cudaGetLastError());
    } else if (nro > 0) {
      MOAO_TRY(range_sums(T32, m, m, off, ZU, s));
      MOAO_TRY(woodbury_apply(T32, m, m, n, ZU, nro, Y2, R64, m, true, s));
    } else {
      MOAO_TRY(add_f32_to_f64(T32, m, R64, m, m, n, s));
    }
  }
  if ((ctx->final_residual || guard) && !graph) MOAO_TRY(residual());
  rep->refine_steps = steps;
  if (guard) {
    double r2 = 0.0;
    MOAO_TRY(sumsq(ctx, R64, m, m, n, dnorm, &r2));
    double est;
    if (r_before < 0)  // no correction ran (the first residual met the tolerance)
      est = rep->refine_resid;
    else
      est = std::sqrt(dr2 / std::max(r2, 1e-300)) * (rep->refine_resid / std::max(r_before, 1e-300));
    rep->est_error = std::max(rep->est_error, est);
    if (!(est <= ctx->acc_target)) {
      rep->fallback = 1;
      int herr[2] = {0, 0};
      MOAO_CUDA_TRY(cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
      MOAO_CUDA_TRY(cudaStreamSynchronize(s));
      if (herr[0]) return set_error(MOAO_ERR_TIMEOUT, "tensor-core kernel: bounded wait expired");
      return MOAO_OK;  // Ctm and Cmm untouched
    }
  }
  // ---- outputs: R in FP64, the FP32 factor into the lower triangle of Cmm
  MOAO_CUDA_TRY(cudaMemcpy2DAsync(Ctm, ldCtm * sizeof(double), R64, m * sizeof(double),
                                  m * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
  if (graph) return MOAO_OK;
  // (slices of R_k, E_k) is a consistent pair: the guard's correction wrote into
  // E64 only before its final residual
  ctx->rstate_valid = ran_residual;
  ctx->rstate_n = n;
  ctx->rstate_m = m;
  cudaEventRecord(ev[6], s);
  int herr[2] = {0, 0};
  MOAO_CUDA_TRY(cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
  MOAO_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr[0]) return set_error(MOAO_ERR_TIMEOUT, "tensor-core kernel: bounded wait expired");
  if (herr[1])
    return set_error(MOAO_ERR_BAD_ARG,
                     "mixed reconstructor: offsets give a singular capacitance matrix");
  float ms = 0;
  cudaEventElapsedTime(&ms, ev[3], ev[4]);
  rep->ms_factor += ms;
  cudaEventElapsedTime(&ms, ev[4], ev[5]);
  rep->ms_solve += ms;
  cudaEventElapsedTime(&ms, ev[5], ev[6]);
  rep->ms_refine += ms;
  return MOAO_OK;
}

// E = Ctm - R sym(Cmm) by the refinement's residual alone (test entry point).
moao_status debug_residual(moao_ctx* ctx, int scheme, long m, long n, const double* R, long ldR,
                           const double* Cmm, long ldCmm, const double* Ctm, long ldCtm,
                           double* E, long ldE) {
  HelperCount hc(ctx);
  cudaStream_t s = ctx->stream;
  const int ns = ctx->ozaki_slices;
  const long ldq = round_up(n, 128);
  const int nmod = scheme == 1 ? crt_moduli_for(ns, n) : 0;
  if (scheme == 1 && !nmod) return set_error(MOAO_ERR_BAD_ARG, "debug_residual: no moduli cover n");
  const int nq = nmod ? nmod : ns;
  DevBuf qa, qb, z, ex, cm, info;
  struct Release {
    DevBuf* b[6];
    ~Release() {
      for (DevBuf* x : b) x->release();
    }
  } release_all{{&qa, &qb, &z, &ex, &cm, &info}};
  MOAO_TRY(qa.ensure((size_t)nq * m * ldq));
  MOAO_TRY(qb.ensure((size_t)nq * n * ldq));
  MOAO_TRY(ex.ensure(sizeof(int) * (size_t)(m + n)));
  MOAO_TRY(cm.ensure(sizeof(unsigned long long) * (size_t)n));
  MOAO_TRY(info.ensure(sizeof(int)));
  int* ea = ex.as<int>();
  int* fb = ea + m;
  int* err = info.as<int>();
  MOAO_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
  OffsetRanges none{};
  TcTensor ta[kCrtMaxModuli], tb[kCrtMaxModuli];
  for (int i = 0; i < nq; ++i) {
    MOAO_TRY(make_tc_map(&ta[i], qa.as<int8_t>() + (size_t)i * m * ldq, kTcI8, m, n, ldq));
    MOAO_TRY(make_tc_map(&tb[i], qb.as<int8_t>() + (size_t)i * n * ldq, kTcI8, n, n, ldq, 256));
  }
  if (nmod) {
    MOAO_TRY(z.ensure((size_t)nmod * m * n));
    MOAO_TRY(crt_split_sym(Cmm, ldCmm, n, ns, nmod, fb, cm.as<unsigned long long>(),
                           qb.as<int8_t>(), ldq, nullptr, none, s));
    // row exponents as the slices use them, then the residues
    MOAO_TRY(ozaki_split_rows(R, ldR, m, n, 1, ea, qa.as<int8_t>(), ldq, s));
    MOAO_TRY(crt_split_rows(R, ldR, m, n, ns, nmod, ea, qa.as<int8_t>(), ldq, s));
    MOAO_TRY(crt_gemm(ctx, ta, tb, nmod, m, n, n, z.as<uint8_t>(), err));
    MOAO_TRY(crt_combine(z.as<uint8_t>(), m, n, nmod, ns, ea, fb, Ctm, ldCtm, -1.0, E, ldE, s));
  } else {
    MOAO_TRY(ozaki_split_sym(Cmm, ldCmm, n, ns, fb, cm.as<unsigned long long>(),
                             qb.as<int8_t>(), ldq, nullptr, none, s));
    MOAO_TRY(ozaki_split_rows(R, ldR, m, n, ns, ea, qa.as<int8_t>(), ldq, s));
    MOAO_CUDA_TRY(cudaMemcpy2DAsync(E, ldE * sizeof(double), Ctm, ldCtm * sizeof(double),
                                    m * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
    MOAO_TRY(ozaki_gemm(ctx, ta, ns, tb, ns, ns + 1, m, n, n, -1.f, E, ldE, ea, fb, err));
  }
  int herr = 0;
  MOAO_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
  MOAO_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr) return set_error(MOAO_ERR_TIMEOUT, "debug_residual: bounded wait expired");
  return MOAO_OK;
}

moao_status finish_mixed(moao_ctx* ctx, long n, double* Cmm, long ldCmm) {
  HelperCount hc(ctx);
  MOAO_TRY(cvt_f32_to_f64(ctx->mx_a32.as<float>(), n, Cmm, ldCmm, n, n, true, ctx->stream));
  ctx->mx_factored_n = -1;
  return MOAO_OK;
}

}  // namespace moao
