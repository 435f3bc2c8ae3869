// Orchestration of the FP64 dense stages on one stream.
//
//   potrf_f64        tiled right-looking Cholesky: recursive diagonal blocks
//                    (64-wide leaves factored and inverted in shared memory),
//                    panel solve as a product with the inverse diagonal block,
//                    trailing SYRK on the lower tiles only.
//   solve_right_f64  R = Ctm L^-T L^-1: right-looking forward pass X L^T = Ctm,
//                    then backward pass R L = X, each a sequence of block
//                    products with the stored inverse diagonal blocks.
//   moao_cee_cvv     lapack/compute/cee_cvv.cpp:50-125 step for step.
#include <algorithm>
#include <cstring>

#include "context.h"
#include "dense.h"

namespace moao {

constexpr int kLeaf = 64;

moao_status gemm(moao_ctx* ctx, long M, long N, long K, double alpha, const double* A, long lda,
                 const double* B, long ldb, bool transB, double beta, double* C, long ldc,
                 bool lowerC, TriMode tri) {
  GemmArgs g;
  g.M = M; g.N = N; g.K = K; g.alpha = alpha; g.beta = beta;
  g.A = A; g.lda = lda; g.B = B; g.ldb = ldb; g.transB = transB; g.triB = tri;
  g.C = C; g.ldc = ldc; g.lowerC = lowerC;
  g.cfg = ctx->gemm_cfg;
  // algorithmic flops: 2MNK, halved when only a triangle of C or of B counts
  double fl = 2.0 * M * N * K;
  if (lowerC) fl = (double)M * N * K + (double)std::min(M, N) * K;
  if (tri != TRI_FULL) fl *= 0.5;
  KernelTimer kt(ctx, "gemm_f64", fl);
  return gemm_f64(g, ctx->stream, &ctx->launches);
}

// Factor the nb x nb diagonal block A (lda) and write its inverse into D (ldd).
// W is scratch of at least nb*nb/4 doubles... (nb/2 x nb/2 + margin).
moao_status potrf_inv_block(moao_ctx* ctx, double* A, long lda, double* D, long ldd, long nb,
                            long col0, int* d_info, double* W) {
  if (nb <= kLeaf) {
    KernelTimer kt(ctx, "potrf_leaf", (double)nb * nb * nb * (1.0 / 3 + 1.0 / 3));
    return potrf_inv_leaf(A, lda, D, ldd, (int)nb, col0, d_info, ctx->stream, &ctx->launches);
  }
  const long n1 = kLeaf * ((nb + 2 * kLeaf - 1) / (2 * kLeaf));
  const long n2 = nb - n1;
  double* A11 = A;
  double* A21 = A + n1;
  double* A22 = A + n1 + n1 * lda;
  double* D11 = D;
  double* D21 = D + n1;
  double* D22 = D + n1 + n1 * ldd;
  MOAO_TRY(potrf_inv_block(ctx, A11, lda, D11, ldd, n1, col0, d_info, W));
  // L21 = A21 L11^-T
  MOAO_TRY(gemm(ctx, n2, n1, n1, 1.0, A21, lda, D11, ldd, true, 0.0, W, n2));
  MOAO_TRY(copy_matrix(W, n2, A21, lda, n2, n1, ctx->stream));
  // A22 -= L21 L21^T (lower)
  MOAO_TRY(gemm(ctx, n2, n2, n1, -1.0, A21, lda, A21, lda, true, 1.0, A22, lda, true));
  MOAO_TRY(potrf_inv_block(ctx, A22, lda, D22, ldd, n2, col0 + n1, d_info, W));
  // D21 = -D22 L21 D11 ; D12 = 0
  MOAO_TRY(gemm(ctx, n2, n1, n1, 1.0, A21, lda, D11, ldd, false, 0.0, W, n2));
  MOAO_TRY(gemm(ctx, n2, n1, n2, -1.0, D22, ldd, W, n2, false, 0.0, D21, ldd));
  MOAO_TRY(fill_matrix(D + n1 * ldd, ldd, n1, n2, 0.0, ctx->stream, &ctx->launches));
  return MOAO_OK;
}

moao_status potrf_f64(moao_ctx* ctx, double* A, long lda, long n, double* dinv, int* d_info) {
  const long nb = ctx->nb;
  MOAO_TRY(ctx->ws_w.ensure(sizeof(double) * (size_t)std::max(n, 1L) * nb));
  double* W = ctx->ws_w.as<double>();
  for (long k0 = 0; k0 < n; k0 += nb) {
    const long kb = std::min(nb, n - k0);
    double* Akk = A + k0 + k0 * lda;
    double* Dk = dinv + k0;  // rows k0.., ld n
    MOAO_TRY(potrf_inv_block(ctx, Akk, lda, Dk, n, kb, k0, d_info, W));
    const long rest = n - k0 - kb;
    if (rest <= 0) break;
    double* P = A + (k0 + kb) + k0 * lda;
    // panel: P <- P L_kk^-T
    MOAO_TRY(gemm(ctx, rest, kb, kb, 1.0, P, lda, Dk, n, true, 0.0, W, rest));
    MOAO_TRY(copy_matrix(W, rest, P, lda, rest, kb, ctx->stream));
    // trailing: A22 -= P P^T on the lower tiles
    double* A22 = A + (k0 + kb) + (k0 + kb) * lda;
    MOAO_TRY(gemm(ctx, rest, rest, kb, -1.0, P, lda, P, lda, true, 1.0, A22, lda, true));
  }
  return MOAO_OK;
}

moao_status solve_right_f64(moao_ctx* ctx, const double* L, long ldl, long n, const double* dinv,
                            double* B, long ldb, long m) {
  const long nb = ctx->nb;
  MOAO_TRY(ctx->ws_w.ensure(sizeof(double) * (size_t)std::max(m, 1L) * nb));
  double* W = ctx->ws_w.as<double>();
  // Forward: X L^T = B.
  for (long k0 = 0; k0 < n; k0 += nb) {
    const long kb = std::min(nb, n - k0);
    double* Bk = B + k0 * ldb;
    MOAO_TRY(gemm(ctx, m, kb, kb, 1.0, Bk, ldb, dinv + k0, n, true, 0.0, W, m));
    MOAO_TRY(copy_matrix(W, m, Bk, ldb, m, kb, ctx->stream));
    const long rest = n - k0 - kb;
    if (rest > 0)
      MOAO_TRY(gemm(ctx, m, rest, kb, -1.0, Bk, ldb, L + (k0 + kb) + k0 * ldl, ldl, true, 1.0,
                    B + (k0 + kb) * ldb, ldb));
  }
  // Backward: R L = X.
  const long nblk = (n + nb - 1) / nb;
  for (long b = nblk - 1; b >= 0; --b) {
    const long k0 = b * nb, kb = std::min(nb, n - k0);
    double* Bk = B + k0 * ldb;
    MOAO_TRY(gemm(ctx, m, kb, kb, 1.0, Bk, ldb, dinv + k0, n, false, 0.0, W, m));
    MOAO_TRY(copy_matrix(W, m, Bk, ldb, m, kb, ctx->stream));
    if (k0 > 0)
      MOAO_TRY(gemm(ctx, m, k0, kb, -1.0, Bk, ldb, L + k0, ldl, false, 1.0, B, ldb));
  }
  return MOAO_OK;
}

moao_status await_inputs(moao_ctx* ctx) {
  if (ctx->wait_inputs) {
    MOAO_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->inputs_ready, 0));
    ctx->wait_inputs = false;
  }
  return MOAO_OK;
}

// Column panels of the lower part of the n x n factor (device ld ldCmm) into the
// host buffer (ld host_factor_ld), on the copy stream after the context stream's
// work so far.
moao_status factor_to_host(moao_ctx* ctx, const double* Cmm, long ldCmm, long n) {
  if (ctx->copy_ev.empty()) {
    cudaEvent_t e;
    MOAO_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->copy_ev.push_back(e);
  }
  MOAO_CUDA_TRY(cudaEventRecord(ctx->copy_ev[0], ctx->stream));
  MOAO_CUDA_TRY(cudaStreamWaitEvent(ctx->copy, ctx->copy_ev[0], 0));
  const long w = 512;
  for (long c0 = 0; c0 < n; c0 += w) {
    const long c1 = std::min(n, c0 + w);
    MOAO_CUDA_TRY(cudaMemcpy2DAsync(ctx->host_factor + c0 * ctx->host_factor_ld + c0,
                                    sizeof(double) * ctx->host_factor_ld, Cmm + c0 * ldCmm + c0,
                                    sizeof(double) * ldCmm, sizeof(double) * (n - c0), c1 - c0,
                                    cudaMemcpyDeviceToHost, ctx->copy));
  }
  return MOAO_OK;
}

// FP64 reconstructor: factor Cmm in place, then the solves of targets g0..ngal-1.
moao_status reconstructor_fp64(moao_ctx* ctx, long nmeas, long nmeasts, double* d_Cmm, long ldCmm,
                               double* d_Ctm, long ldCtm, long g0, long ngal,
                               moao_solve_report* r) {
  MOAO_TRY(ctx->ws_dinv.ensure(sizeof(double) * (size_t)nmeas * ctx->nb));
  MOAO_TRY(ctx->ws_info.ensure(sizeof(int)));
  int* d_info = ctx->ws_info.as<int>();
  MOAO_CUDA_TRY(cudaMemsetAsync(d_info, 0, sizeof(int), ctx->stream));
  cudaEventRecord(ctx->ev[0], ctx->stream);
  MOAO_TRY(potrf_f64(ctx, d_Cmm, ldCmm, nmeas, ctx->ws_dinv.as<double>(), d_info));
  cudaEventRecord(ctx->ev[1], ctx->stream);
  int info = 0;
  MOAO_CUDA_TRY(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  r->info = info;
  if (info != 0) {
    // The reference prints and returns without solving (reconstructor.cpp:34-38).
    return set_error(MOAO_ERR_NOT_SPD, "dpotrf: non-positive pivot at column " +
                                           std::to_string(info));
  }
  if (ctx->host_factor) {  // the factor is final: back to the host beside the solves
    MOAO_TRY(factor_to_host(ctx, d_Cmm, ldCmm, nmeas));
    ctx->factor_done = true;
  }
  MOAO_TRY(await_inputs(ctx));
  for (long g = g0; g < ngal; ++g) {
    double* Ctm_g = d_Ctm + nmeas * nmeasts * g;
    MOAO_TRY(solve_right_f64(ctx, d_Cmm, ldCmm, nmeas, ctx->ws_dinv.as<double>(), Ctm_g, ldCtm,
                             nmeasts));
  }
  cudaEventRecord(ctx->ev[2], ctx->stream);
  MOAO_CUDA_TRY(cudaEventSynchronize(ctx->ev[2]));
  float ms = 0;
  cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
  r->ms_factor += ms;
  cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]);
  r->ms_solve += ms;
  return MOAO_OK;
}

}  // namespace moao

using namespace moao;

extern "C" {

moao_status moao_reconstructor(moao_ctx* ctx, long nmeas, long nmeasts, double* d_Cmm,
                               long ldCmm, double* d_Ctm, long ldCtm, long ngal, moao_prec prec,
                               moao_solve_report* rep) {
  if (!ctx) return set_error(MOAO_ERR_BAD_ARG, "reconstructor: null context");
  if (nmeas < 0 || nmeasts < 0 || ngal < 0 || ldCmm < std::max(1L, nmeas) ||
      ldCtm < std::max(1L, nmeasts) || (nmeas > 0 && (!d_Cmm || !d_Ctm)))
    return set_error(MOAO_ERR_BAD_ARG, "reconstructor: bad sizes or pointers");
  if (prec != MOAO_PREC_FP64 && prec != MOAO_PREC_MIXED)
    return set_error(MOAO_ERR_BAD_ARG, "reconstructor: unknown precision");
  moao_solve_report local{};
  moao_solve_report* r = rep ? rep : &local;
  std::memset(r, 0, sizeof(*r));
  if (nmeas == 0) return MOAO_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  ctx->factor_done = false;
  if (prec == MOAO_PREC_MIXED) {
    long g = 0;
    for (; g < ngal; ++g) {
      // one factorisation serves every target: later targets reuse it
      MOAO_TRY(reconstructor_mixed(ctx, nmeas, nmeasts, d_Cmm, ldCmm,
                                   d_Ctm + nmeas * nmeasts * g, ldCtm, g > 0, r));
      if (r->fallback) break;
    }
    if (r->fallback) {
      // the mixed estimate missed the accuracy target: this and the remaining
      // targets from the FP64 path (Cmm and their Ctm are still as given)
      ctx->mx_factored_n = -1;
      ctx->rstate_valid = false;
      return reconstructor_fp64(ctx, nmeas, nmeasts, d_Cmm, ldCmm, d_Ctm, ldCtm, g, ngal, r);
    }
    if (!ctx->keep_cmm && !ctx->factor_done) MOAO_TRY(finish_mixed(ctx, nmeas, d_Cmm, ldCmm));
    if (ctx->factor_done) ctx->mx_factored_n = -1;  // A32 no longer matches what finish_mixed leaves
    MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return MOAO_OK;
  }
  return reconstructor_fp64(ctx, nmeas, nmeasts, d_Cmm, ldCmm, d_Ctm, ldCtm, 0, ngal, r);
}

moao_status moao_cee_cvv(moao_ctx* ctx, long nmeas, long nmeasts, long nact, double* Cmm,
                         long ldCmm, double* Cpp, long ldCpp, double* Cpm, long ldCpm, double* R,
                         long ldR, double* Dx, long ldDx, double* Cee, long ldCee, double* Cvv,
                         long ldCvv, double* Tmp, long ldTmp) {
  return moao_cee_cvv_prec(ctx, nmeas, nmeasts, nact, Cmm, ldCmm, Cpp, ldCpp, Cpm, ldCpm, R, ldR,
                           Dx, ldDx, Cee, ldCee, Cvv, ldCvv, Tmp, ldTmp, MOAO_PREC_FP64);
}

moao_status moao_cee_cvv_prec(moao_ctx* ctx, long nmeas, long nmeasts, long nact, double* Cmm,
                              long ldCmm, double* Cpp, long ldCpp, double* Cpm, long ldCpm,
                              double* R, long ldR, double* Dx, long ldDx, double* Cee, long ldCee,
                              double* Cvv, long ldCvv, double* Tmp, long ldTmp, moao_prec prec) {
  if (!ctx) return set_error(MOAO_ERR_BAD_ARG, "Cee_Cvv: null context");
  if (prec != MOAO_PREC_FP64 && prec != MOAO_PREC_MIXED)
    return set_error(MOAO_ERR_BAD_ARG, "Cee_Cvv: unknown precision");
  if (nmeas < 0 || nmeasts < 0 || nact < 0)
    return set_error(MOAO_ERR_BAD_ARG, "Cee_Cvv: negative size");
  if (ldCmm < std::max(1L, nmeas) || ldCpp < std::max(1L, nmeasts) ||
      ldCpm < std::max(1L, nmeasts) || ldR < std::max(1L, nmeasts) ||
      ldDx < std::max(1L, nact) || ldCee < std::max(1L, nmeasts) ||
      ldCvv < std::max(1L, nact) || ldTmp < std::max(1L, nact))
    return set_error(MOAO_ERR_BAD_ARG, "Cee_Cvv: leading dimension too small");
  if ((nmeas > 0 && (!Cmm || !R)) || (nmeasts > 0 && (!Cpp || !Cpm || !Cee)) ||
      (nact > 0 && (!Dx || !Cvv || !Tmp)))
    return set_error(MOAO_ERR_BAD_ARG, "Cee_Cvv: null matrix pointer");
  std::lock_guard<std::mutex> lk(ctx->mu);
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  if (prec == MOAO_PREC_MIXED)
    return cee_cvv_mixed(ctx, nmeas, nmeasts, nact, Cmm, ldCmm, Cpp, ldCpp, Cpm, ldCpm, R, ldR, Dx,
                         ldDx, Cee, ldCee, Cvv, ldCvv, Tmp, ldTmp);
  const long nm = nmeas, nt = nmeasts;
  // (1) Cpp <- Cpp - Cpm R^T - R Cpm^T  (syr2k, lower)
  MOAO_TRY(gemm(ctx, nt, nt, nm, -1.0, Cpm, ldCpm, R, ldR, true, 1.0, Cpp, ldCpp, true));
  MOAO_TRY(gemm(ctx, nt, nt, nm, -1.0, R, ldR, Cpm, ldCpm, true, 1.0, Cpp, ldCpp, true));
  // (2) Cpm <- R Cmm  (symm right, Cmm lower-stored)
  MOAO_TRY(gemm(ctx, nt, nm, nm, 1.0, R, ldR, Cmm, ldCmm, false, 0.0, Cpm, ldCpm, false,
                TRI_LOWER));
  MOAO_TRY(gemm(ctx, nt, nm, nm, 1.0, R, ldR, Cmm, ldCmm, true, 1.0, Cpm, ldCpm, false,
                TRI_STRICT_LOWER));
  // (3)-(6) Cee <- sym(tril(Cpp))
  MOAO_TRY(sym_from_lower(Cpp, ldCpp, Cee, ldCee, nt, ctx->stream, &ctx->launches));
  // (7) Cee += Cpm R^T
  MOAO_TRY(gemm(ctx, nt, nt, nm, 1.0, Cpm, ldCpm, R, ldR, true, 1.0, Cee, ldCee));
  // (8) Tmp <- Dx sym(tril(Cee))
  MOAO_TRY(gemm(ctx, nact, nt, nt, 1.0, Dx, ldDx, Cee, ldCee, false, 0.0, Tmp, ldTmp, false,
                TRI_LOWER));
  MOAO_TRY(gemm(ctx, nact, nt, nt, 1.0, Dx, ldDx, Cee, ldCee, true, 1.0, Tmp, ldTmp, false,
                TRI_STRICT_LOWER));
  // (9) Cvv <- Tmp Dx^T
  MOAO_TRY(gemm(ctx, nact, nact, nt, 1.0, Tmp, ldTmp, Dx, ldDx, true, 0.0, Cvv, ldCvv));
  return MOAO_OK;
}

moao_status moao_dense_potrf_inv(moao_ctx* ctx, long n, double* A, long lda, double* Ainv,
                                 long ldi, int* info) {
  if (!ctx || n < 0 || (n > 0 && (!A || !Ainv)) || lda < std::max(1L, n) ||
      ldi < std::max(1L, n))
    return set_error(MOAO_ERR_BAD_ARG, "dense_potrf_inv: bad sizes or pointers");
  if (info) *info = 0;
  if (n == 0) return MOAO_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  MOAO_TRY(ctx->ws_w.ensure(sizeof(double) * (size_t)n * n));
  MOAO_TRY(ctx->ws_info.ensure(3 * sizeof(int)));
  int* d_info = ctx->ws_info.as<int>();
  MOAO_CUDA_TRY(cudaMemsetAsync(d_info, 0, sizeof(int), ctx->stream));
  MOAO_TRY(potrf_inv_block(ctx, A, lda, Ainv, ldi, n, 0, d_info, ctx->ws_w.as<double>()));
  int h = 0;
  MOAO_CUDA_TRY(cudaMemcpyAsync(&h, d_info, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (info) *info = h;
  if (h) return set_error(MOAO_ERR_NOT_SPD, "dense_potrf_inv: non-positive pivot at column " +
                                                std::to_string(h));
  return MOAO_OK;
}

moao_status moao_dense_gemm(moao_ctx* ctx, int transB, int lowerC, long M, long N, long K,
                            double alpha, const double* A, long lda, const double* B, long ldb,
                            double beta, double* C, long ldc) {
  if (!ctx) return set_error(MOAO_ERR_BAD_ARG, "dense_gemm: null context");
  if (M < 0 || N < 0 || K < 0) return set_error(MOAO_ERR_BAD_ARG, "dense_gemm: negative size");
  if (M == 0 || N == 0) return MOAO_OK;
  if (!C || (K > 0 && (!A || !B))) return set_error(MOAO_ERR_BAD_ARG, "dense_gemm: null matrix");
  std::lock_guard<std::mutex> lk(ctx->mu);
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  return gemm(ctx, M, N, K, alpha, A, lda, B, ldb, transB != 0, beta, C, ldc, lowerC != 0);
}

}  // extern "C"
