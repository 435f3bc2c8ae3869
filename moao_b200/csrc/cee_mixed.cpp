// Error covariances Cee and Cvv on the int8 tensor cores (mixed precision).
//
// The reference evaluates, in nine BLAS/LAPACK steps (lapack/compute/
// cee_cvv.cpp:50-125),
//   Cee = Ctt - Ctm R^T - R Ctm^T + R Cmm R^T,   Cvv = Dx Cee Dx^T,
// reading Ctt and Cmm through their lower triangles. With the residual of the
// reconstructor E = Ctm - R Cmm (Cmm symmetric), R Cmm R^T = Ctm R^T - E R^T, so
//   Cee = Ctt - R Ctm^T - E R^T
// is the same matrix in exact arithmetic, evaluated here as three products
// with the Ozaki splitting (int8 slices scaled by powers of two per row, exact
// int32 accumulation, FP64 sums):
//   Cee  = sym(tril(Ctt)) - R Ctm^T          nts x nts x nmeas, ns slices each
//   E    = Ctm - R sym(Cmm)                  nts x nmeas x nmeas, ns-slice operands,
//                                            exact CRT products (one int8 GEMM per
//                                            modulus, as the refinement residual)
//   Cee -= E R^T                             3 slices of E: E is a residual, a few
//                                            1e-6 of Ctm, so its product needs only
//                                            ~1e-6 relative accuracy
// then Tmp = Dx sym(tril(Cee)) and Cvv = Tmp Dx^T in FP64 (the reference's
// steps 8 and 9; 3.4e11 flop at ELT size against 3.4e13 for the whole chain).
// The three int8 products cost ~7.5x their FP64 flop count in int8 operations,
// which the tensor cores run ~60x faster than the FP64 pipe.
// Declared offsets of Cmm (moao_ctx_set_offsets) are handled as in the
// refinement residual: the slices are of sym(Cmm) minus the offsets, and the
// offsets' part R U D U^T comes from FP64 range sums of R.
// In-place contract: Cpm ends as R Cmm (= Ctm - E), like the reference's step 2;
// Cpp is read and left as given (the reference leaves the lower triangle of
// Ctt - Ctm R^T - R Ctm^T there); Tmp holds Dx sym(Cee).
#include <cuda_runtime.h>

#include <algorithm>

#include "context.h"
#include "mixed.h"
#include "tc_gemm.h"

namespace moao {
namespace {

long round_up_c(long x, long a) { return (x + a - 1) / a * a; }

// A (m x n, lda) -= B (m x n, ldb), column-major.
__global__ void sub_inplace_kernel(double* __restrict__ A, long lda, const double* __restrict__ B,
                                   long ldb, long m, long n) {
  const long total = m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    A[j * lda + i] -= B[j * ldb + i];
  }
}

constexpr int kErrSlices = 3;  // int8 slices of E's rows

}  // namespace

moao_status cee_cvv_mixed(moao_ctx* ctx, long nm, long nt, long nact, const double* Cmm,
                          long ldCmm, const double* Cpp, long ldCpp, double* Cpm, long ldCpm,
                          const double* R, long ldR, const double* Dx, long ldDx, double* Cee,
                          long ldCee, double* Cvv, long ldCvv, double* Tmp, long ldTmp,
                          bool from_refinement) {
  const bool use_state = from_refinement && ctx->rstate_valid && ctx->rstate_n == nm &&
                         ctx->rstate_m == nt;
  if (!use_state) ctx->rstate_valid = false;  // this call overwrites the state's buffers
  const long long h0 = helper_launches();
  cudaStream_t s = ctx->stream;
  const int ns = ctx->ozaki_slices;
  const long ldq = round_up_c(std::max(nm, 1L), 128);
  const OffsetRanges& off = ctx->offsets;
  const int nro = off.n;
  for (int w = 0; w < nro; ++w)
    if (off.end[w] > nm)
      return set_error(MOAO_ERR_BAD_ARG, "mixed Cee_Cvv: an offset range ends beyond nmeas");
  // E by exact CRT products (as the refinement residual) where the moduli cover it
  const int nmod = (!use_state && ctx->residual_crt) ? crt_moduli_for(ns, nm) : 0;
  if (nt > 0 && nm > 0) {
    MOAO_TRY(ctx->mx_qa.ensure((size_t)ns * nt * ldq));
    if (!use_state && !nmod) MOAO_TRY(ctx->mx_qb.ensure((size_t)ns * nm * ldq));
    if (nmod) {
      MOAO_TRY(ctx->mx_qr.ensure((size_t)nmod * nt * ldq));
      MOAO_TRY(ctx->mx_qs.ensure((size_t)nmod * nm * ldq));
      MOAO_TRY(ctx->mx_z.ensure((size_t)nmod * nt * nm));
    }
    MOAO_TRY(ctx->cx_qc.ensure((size_t)std::max(ns, kErrSlices) * nt * ldq));
    MOAO_TRY(ctx->mx_ea.ensure(sizeof(int) * (size_t)nt));
    MOAO_TRY(ctx->cx_ec.ensure(2 * sizeof(int) * (size_t)nt));
    MOAO_TRY(ctx->mx_fb.ensure(sizeof(int) * (size_t)nm));
    MOAO_TRY(ctx->mx_colmax.ensure(sizeof(unsigned long long) * (size_t)nm));
    MOAO_TRY(ctx->mx_e64.ensure(sizeof(double) * (size_t)nt * nm));
    MOAO_TRY(ctx->ws_info.ensure(3 * sizeof(int)));
    int8_t* qa = ctx->mx_qa.as<int8_t>();
    int8_t* qb = ctx->mx_qb.as<int8_t>();
    int8_t* qc = ctx->cx_qc.as<int8_t>();
    int* ea = ctx->mx_ea.as<int>();
    int* ec = ctx->cx_ec.as<int>();
    int* ee = ec + nt;
    int* fb = ctx->mx_fb.as<int>();
    double* E64 = ctx->mx_e64.as<double>();
    int* err = ctx->ws_info.as<int>() + 1;
    MOAO_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), s));
    int* rid = nullptr;
    double* RU = nullptr;
    if (nro > 0) {
      MOAO_TRY(ctx->mx_rid.ensure(sizeof(int) * (size_t)nm));
      MOAO_TRY(ctx->mx_zu.ensure(sizeof(double) * (size_t)std::max(nt, (long)nro) * nro));
      rid = ctx->mx_rid.as<int>();
      RU = ctx->mx_zu.as<double>();
      MOAO_TRY(fill_range_ids(rid, nm, off, s));
    }
    TcTensor taR[kMaxOzakiSlices], tbR[kMaxOzakiSlices], tbC[kMaxOzakiSlices],
        tbS[kMaxOzakiSlices], taE[kErrSlices];
    for (int i = 0; i < ns; ++i) {
      MOAO_TRY(make_tc_map(&taR[i], qa + (size_t)i * nt * ldq, kTcI8, nt, nm, ldq));
      MOAO_TRY(make_tc_map(&tbR[i], qa + (size_t)i * nt * ldq, kTcI8, nt, nm, ldq, 256));
      MOAO_TRY(make_tc_map(&tbC[i], qc + (size_t)i * nt * ldq, kTcI8, nt, nm, ldq, 256));
      if (!use_state && !nmod)
        MOAO_TRY(make_tc_map(&tbS[i], qb + (size_t)i * nm * ldq, kTcI8, nm, nm, ldq, 256));
    }
    for (int i = 0; i < kErrSlices; ++i)
      MOAO_TRY(make_tc_map(&taE[i], qc + (size_t)i * nt * ldq, kTcI8, nt, nm, ldq));
    TcTensor tr[kCrtMaxModuli], ts[kCrtMaxModuli];
    for (int i = 0; i < nmod; ++i) {
      MOAO_TRY(make_tc_map(&tr[i], ctx->mx_qr.as<int8_t>() + (size_t)i * nt * ldq, kTcI8, nt, nm,
                           ldq));
      MOAO_TRY(make_tc_map(&ts[i], ctx->mx_qs.as<int8_t>() + (size_t)i * nm * ldq, kTcI8, nm, nm,
                           ldq, 256));
    }
    // slices of R's rows (or the refinement's R_k) and of Ctm's rows
    if (!use_state) MOAO_TRY(ozaki_split_rows(R, ldR, nt, nm, ns, ea, qa, ldq, s));
    MOAO_TRY(ozaki_split_rows(Cpm, ldCpm, nt, nm, ns, ec, qc, ldq, s));
    // Cee = sym(tril(Ctt)) - R Ctm^T
    MOAO_TRY(sym_from_lower(Cpp, ldCpp, Cee, ldCee, nt, s, &ctx->launches));
    MOAO_TRY(ozaki_gemm(ctx, taR, ns, tbC, ns, ns + 1, nt, nt, nm, -1.f, Cee, ldCee, ea, ec, err));
    if (!use_state && nmod) {
      // E = Ctm - R sym(Cmm) by exact CRT products of the sliced operands
      MOAO_TRY(crt_split_sym(Cmm, ldCmm, nm, ns, nmod, fb, ctx->mx_colmax.as<unsigned long long>(),
                             ctx->mx_qs.as<int8_t>(), ldq, rid, off, s));
      MOAO_TRY(crt_split_rows(R, ldR, nt, nm, ns, nmod, ea, ctx->mx_qr.as<int8_t>(), ldq, s));
      MOAO_TRY(crt_gemm(ctx, tr, ts, nmod, nt, nm, nm, ctx->mx_z.as<uint8_t>(), err));
      MOAO_TRY(crt_combine(ctx->mx_z.as<uint8_t>(), nt, nm, nmod, ns, ea, fb, Cpm, ldCpm, -1.0,
                           E64, nt, s));
      if (nro > 0) {  // the offsets' part of R Cmm
        MOAO_TRY(range_sums(R, ldR, nt, off, RU, s));
        MOAO_TRY(subtract_offset_products(E64, nt, nt, nm, RU, rid, off, s));
      }
    } else if (!use_state) {
      // E = Ctm - R sym(Cmm) (the refinement state holds it for R_k)
      MOAO_CUDA_TRY(cudaMemcpy2DAsync(E64, nt * sizeof(double), Cpm, ldCpm * sizeof(double),
                                      nt * sizeof(double), nm, cudaMemcpyDeviceToDevice, s));
      MOAO_TRY(ozaki_split_sym(Cmm, ldCmm, nm, ns, fb, ctx->mx_colmax.as<unsigned long long>(),
                               qb, ldq, rid, off, s));
      MOAO_TRY(ozaki_gemm(ctx, taR, ns, tbS, ns, ns + 1, nt, nm, nm, -1.f, E64, nt, ea, fb, err));
      if (nro > 0) {  // the offsets' part of R Cmm
        MOAO_TRY(range_sums(R, ldR, nt, off, RU, s));
        MOAO_TRY(subtract_offset_products(E64, nt, nt, nm, RU, rid, off, s));
      }
    }
    // Cee -= E R^T (Ctm's slices are no longer needed: E's go in their place)
    MOAO_TRY(ozaki_split_rows(E64, nt, nt, nm, kErrSlices, ee, qc, ldq, s));
    MOAO_TRY(ozaki_gemm(ctx, taE, kErrSlices, tbR, ns, kErrSlices + 1, nt, nt, nm, -1.f, Cee,
                        ldCee, ee, ea, err));
    if (!use_state) {
      // Cpm <- R Cmm = Ctm - E
      sub_inplace_kernel<<<148 * 8, 256, 0, s>>>(Cpm, ldCpm, E64, nt, nt, nm);
      ++ctx->launches;
      MOAO_CUDA_TRY(cudaGetLastError());
    }
  } else if (nt > 0) {
    MOAO_TRY(sym_from_lower(Cpp, ldCpp, Cee, ldCee, nt, s, &ctx->launches));
  }
  // (8) Tmp <- Dx sym(tril(Cee)); (9) Cvv <- Tmp Dx^T, in FP64
  MOAO_TRY(gemm(ctx, nact, nt, nt, 1.0, Dx, ldDx, Cee, ldCee, false, 0.0, Tmp, ldTmp, false,
                TRI_LOWER));
  MOAO_TRY(gemm(ctx, nact, nt, nt, 1.0, Dx, ldDx, Cee, ldCee, true, 1.0, Tmp, ldTmp, false,
                TRI_STRICT_LOWER));
  MOAO_TRY(gemm(ctx, nact, nact, nt, 1.0, Tmp, ldTmp, Dx, ldDx, true, 0.0, Cvv, ldCvv));
  ctx->launches += helper_launches() - h0;
  if (ctx->graph_mode || nt == 0 || nm == 0) return MOAO_OK;
  int herr = 0;
  MOAO_CUDA_TRY(cudaMemcpyAsync(&herr, ctx->ws_info.as<int>() + 1, sizeof(int),
                                cudaMemcpyDeviceToHost, s));
  MOAO_CUDA_TRY(cudaStreamSynchronize(s));
  if (herr) return set_error(MOAO_ERR_TIMEOUT, "tensor-core kernel: bounded wait expired");
  return MOAO_OK;
}

}  // namespace moao
