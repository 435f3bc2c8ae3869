// Per-device context: stream, cached device geometry, factorisation workspace.
#ifndef MOAO_CONTEXT_H
#define MOAO_CONTEXT_H

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "moao_b200_tomo.hpp"
#include "moao_internal.h"
#include "dense.h"
#include "mixed.h"

struct moao_tomo {
  Tomo_struct<double> t;
};

namespace moao {

// A device buffer that only grows.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  unsigned long long generation = 0;  // bumped by every (re)allocation and release
  moao_status ensure(size_t n);
  void release();
  template <typename T>
  T* as() const { return static_cast<T*>(p); }
};

// Device-time accounting per kernel family (see moao_ctx_set_kernel_timing).
struct FamilyStats {
  long long launches = 0;
  double ms = 0, work = 0;
};

struct GeomEntry {
  unsigned long long version = ~0ull;
  DevGeometry g;
  DevBuf buf;  // backing store of every array in g
};

}  // namespace moao

struct moao_ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  long long launches = 0;
  int nb = 1024;  // outer panel width of the blocked factorisation
  moao_prec host_prec = MOAO_PREC_FP64;  // precision of moao_reconstructor_host
  bool keep_cmm = false;  // mixed path: leave Cmm as given (no factor written back)
  bool graph_mode = false;  // mixed path under stream capture: no host waits or reads
  std::mutex mu;
  std::map<const moao_tomo*, moao::GeomEntry> geom;
  moao::DevBuf ws_w, ws_dinv, ws_info, ws_tmp, ws_host_t, ws_corner;
  // mixed-precision workspace
  moao::DevBuf mx_a32, mx_lr, mx_lc, mx_t32, mx_w1, mx_w2, mx_x, mx_r64, mx_e64, mx_qa, mx_qb,
      mx_ea, mx_fb, mx_colmax, mx_norm;
  // refinement residual by the Chinese remainder theorem: residues of R's rows
  // and of sym(Cmm)'s columns, and of the product, one per modulus
  moao::DevBuf mx_qr, mx_qs, mx_z;
  moao::DevBuf mx_rid, mx_y, mx_y2, mx_zu, mx_sinv, mx_exps, mx_dsl;
  // mixed Cee/Cvv chain: int8 slices of Ctm's rows (then of E's), their exponents
  moao::DevBuf cx_qc, cx_ec;
  long mx_factored_n = -1;  // size of the factorisation held in mx_* (reuse across targets)
  // Block-constant offsets of Cmm known to the caller (moao_ctx_set_offsets):
  // the mixed path factors Cmm minus them and adds them back exactly.
  moao::OffsetRanges offsets;
  int bf16_slices = 3;       // bf16 slices of the factor (3: ~24 bits, 6 products)
  int factor_format = 1;     // MOAO_FACTOR_F16X2 (default) or MOAO_FACTOR_BF16X3
  int corr_slices = 0;       // factor slices in the correction solves (0: 1 for fp16x2, 2 for bf16x3)
  int ozaki_slices = 5;      // int8 slices per operand of the refinement residual
  int residual_crt = 1;      // refinement residual as exact CRT products (moao_ctx_set_residual)
  int max_refine = 1;        // refinement corrections per target
  double refine_tol = 0.0;   // stop refining once ||E||/||Ctm|| is at or below this
  int final_residual = 0;    // evaluate the residual once more after the last correction
  // polls of each bounded wait inside the tensor-core kernel (0: its default, 2^28);
  // a wait that runs out makes the call return MOAO_ERR_TIMEOUT
  unsigned long long wait_polls = 0;
  // mixed reconstructor: estimated relative error of R above which the FP64
  // path runs instead (0: no estimate, no fallback)
  double acc_target = 0.0;
  cudaEvent_t ev[8] = {};
  // Mixed factorisation lookahead: the next diagonal block is factored on aux
  // (created on first use) while the trailing update leaves this many SMs free
  // (0: no lookahead).
  int lookahead_sms = 8;
  int lookahead_max = 8;  // SMs left to it in the last panels (moao_ctx_set_lookahead_max)
  int gemm_cfg = 1;       // tile configuration of the large FP64 products (GemmArgs::cfg)
  int tc_pair = 0;        // tensor-core products on CTA pairs (TcGemm::pair)
  // Host-buffer cache of the drop-in path (moao_ctx_set_host_cache): the device
  // copy that moao_matcov_tile_host left of a whole Cmm (in ws_tmp) or Ctm (in
  // ws_host_t), keyed by the host buffer, its shape and the workspace's
  // generation; moao_reconstructor_host then skips that upload.
  struct HostTile {
    const double* h = nullptr;
    long ld = 0, rows = 0, cols = 0;
    unsigned long long gen = 0;
  };
  bool host_cache = false;
  HostTile cache_cmm, cache_ctm;
  cudaStream_t aux = nullptr;
  cudaEvent_t la_ev[2] = {};
  // host-buffer entry points: device-to-host copies of finished column blocks
  // on a second stream while the next block is computed (created on first use)
  cudaStream_t copy = nullptr;
  std::vector<cudaEvent_t> copy_ev;
  // moao_reconstructor_host: Ctm arrives on the copy stream (the solves wait for
  // inputs_ready), and the finished factor leaves for host_factor on the copy
  // stream while the solves run; factor_done says it has been written to Cmm
  bool wait_inputs = false;
  cudaEvent_t inputs_ready = nullptr;
  double* host_factor = nullptr;
  long host_factor_ld = 0;
  bool factor_done = false;
  // After a mixed reconstructor whose refinement evaluated a residual, mx_qa /
  // mx_ea hold the int8 slices of an R_k and mx_e64 its residual E_k = Ctm - R_k Cmm
  // (nmeas rstate_n, nmeasts rstate_m): what a Cee from the refinement needs.
  bool rstate_valid = false;
  long rstate_n = 0, rstate_m = 0;
  // kernel timing
  bool timing = false;
  std::map<std::string, moao::FamilyStats> stats;
  struct Pending {
    std::string family;
    cudaEvent_t a, b;
    double work;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> event_pool;

  // Every workspace buffer of the context (not the geometry caches).
  std::vector<moao::DevBuf*> workspaces() {
    return {&ws_w,  &ws_dinv, &ws_info, &ws_tmp, &ws_host_t, &ws_corner, &mx_a32, &mx_lr,  &mx_lc,    &mx_t32,
            &mx_w1, &mx_w2,   &mx_x,    &mx_r64, &mx_e64, &mx_qa,  &mx_qb,    &mx_ea,
            &mx_fb, &mx_colmax, &mx_norm, &mx_rid, &mx_y, &mx_y2, &mx_zu, &mx_sinv, &mx_exps,
            &mx_dsl, &cx_qc, &cx_ec};
  }
  // Device bytes held by the workspaces and the geometry caches.
  size_t bytes_held() {
    size_t b = 0;
    for (moao::DevBuf* d : workspaces()) b += d->bytes;
    for (auto& kv : geom) b += kv.second.buf.bytes;
    return b;
  }
};

namespace moao {

struct TcTensor;

// Brackets the launches issued during its lifetime with events when the
// context's kernel timing is on.
class KernelTimer {
 public:
  KernelTimer(moao_ctx* ctx, const char* family, double work);
  ~KernelTimer();
 private:
  moao_ctx* ctx_;
  const char* family_;
  double work_;
  cudaEvent_t a_ = nullptr;
};
// Folds completed event pairs into the per-family totals (synchronises).
moao_status collect_kernel_stats(moao_ctx* ctx);

// Uploads (or reuses) the device copy of a tomo's geometry tables.
moao_status device_geometry(moao_ctx* ctx, const moao_tomo* t, const DevGeometry** out);

// FP64 blocked Cholesky (lower, in place) of the n x n matrix A; fills dinv
// (n x nb, ld n) with the inverse of every diagonal block. info receives the
// first failing column (1-based) or 0.
moao_status potrf_f64(moao_ctx* ctx, double* A, long lda, long n, double* dinv, int* d_info);
// C = alpha A op(B) + beta C in FP64, with optional lower-only C / triangular B
// (see dense.h); accounted as kernel family gemm_f64.
moao_status gemm(moao_ctx* ctx, long M, long N, long K, double alpha, const double* A, long lda,
                 const double* B, long ldb, bool transB, double beta, double* C, long ldc,
                 bool lowerC = false, TriMode tri = TRI_FULL);
// Factor the nb x nb diagonal block A in place (FP64) and write its inverse into D.
moao_status potrf_inv_block(moao_ctx* ctx, double* A, long lda, double* D, long ldd, long nb,
                            long col0, int* d_info, double* W);
// Device bytes of the mixed path's workspace for nmeas n, nmeasts m, panel nb,
// nsl bf16 slices, ns int8 slices and nranges declared offset ranges.
struct MixedSizes {
  size_t a32 = 0, lr = 0, t32 = 0, w = 0, x = 0, r64 = 0, qa = 0, qb = 0, ea = 0, fb = 0,
         colmax = 0, norm = 0, dinv = 0, info = 0, offsets = 0, exps = 0, dsl = 0, qr = 0, qs = 0,
         z = 0;
  int nmod = 0;  // moduli of the CRT residual (0: int8 slice products)
  size_t total() const {
    return a32 + 2 * lr + t32 + 2 * w + x + 2 * r64 + qa + qb + ea + fb + colmax + norm +
           2 * dinv + info + offsets + exps + dsl + qr + qs + z;
  }
};
// crt: the refinement residual by CRT products where the moduli cover it
MixedSizes mixed_sizes(long n, long m, long nb, int nsl, int ns, int nranges, bool crt);
// Mixed-precision reconstructor for one target (see mixed.cpp); reuse = 1 keeps
// the factorisation of the previous call.
moao_status reconstructor_mixed(moao_ctx* ctx, long n, long m, double* Cmm, long ldCmm,
                                double* Ctm, long ldCtm, bool reuse, moao_solve_report* rep);
// Destroys the batch engine's sub-contexts and tuning table of ctx.
void release_batch_state(moao_ctx* ctx);
// Writes the mixed factorisation's (FP32) factor into the lower triangle of Cmm.
moao_status finish_mixed(moao_ctx* ctx, long n, double* Cmm, long ldCmm);
// E = Ctm - R sym(Cmm) by the refinement residual alone (scheme 0: int8 slice
// products, 1: CRT products); for tests.
moao_status debug_residual(moao_ctx* ctx, int scheme, long m, long n, const double* R, long ldR,
                           const double* Cmm, long ldCmm, const double* Ctm, long ldCtm,
                           double* E, long ldE);
// The host-buffer path's overlap hooks: the stream waits for inputs that arrive on
// the copy stream, and the finished lower factor in Cmm (ld n) goes back to the
// host on the copy stream while the solves run.
moao_status await_inputs(moao_ctx* ctx);
moao_status factor_to_host(moao_ctx* ctx, const double* Cmm, long ldCmm, long n);
// C (FP64, M x N, ldc) += alpha * A B^T from int8 Ozaki slices of the rows of
// A (ta[0..nsa), 128-row boxes) and of B (tb[0..nsb), 256-row boxes), K columns,
// keeping the slice products p + q + 2 <= dmax (0-based p, q); erow / ecol are
// the row exponents of A and B (see mixed.cpp). Accounted as family tc_int8.
moao_status ozaki_gemm(moao_ctx* ctx, const TcTensor* ta, int nsa, const TcTensor* tb, int nsb,
                       int dmax, long M, long N, long K, float alpha, double* C, long ldc,
                       const int* erow, const int* ecol, int* err);
// Residues of A B^T (M x N over K < 2^17) modulo the first nmod CRT moduli from
// the operands' residues (ta / tb, one per modulus): one exact int8 GEMM per
// modulus into Z + i*M*N (uint8, column-major, ld M). Accounted as tc_int8.
moao_status crt_gemm(moao_ctx* ctx, const TcTensor* ta, const TcTensor* tb, int nmod, long M,
                     long N, long K, uint8_t* Z, int* err);
// Cee and Cvv with the int8 tensor cores (cee_mixed.cpp); same arguments and
// in-place contract as moao_cee_cvv except that Cpp is left as given. With
// from_refinement and a matching refinement state on the context, Cee is
// evaluated at that state's R_k and E_k (Cmm and R are then not read, Cpm is left
// as given): Cee is stationary in R, so this differs from Cee at the final R by
// second order in R_k's error.
moao_status cee_cvv_mixed(moao_ctx* ctx, long nmeas, long nmeasts, long nact, const double* Cmm,
                          long ldCmm, const double* Cpp, long ldCpp, double* Cpm, long ldCpm,
                          const double* R, long ldR, const double* Dx, long ldDx, double* Cee,
                          long ldCee, double* Cvv, long ldCvv, double* Tmp, long ldTmp,
                          bool from_refinement = false);
// R = B * L^-T * L^-1 in place on B (m x n, ldb) using the factor and dinv.
moao_status solve_right_f64(moao_ctx* ctx, const double* L, long ldl, long n, const double* dinv,
                            double* B, long ldb, long m);

}  // namespace moao

#endif  // MOAO_CONTEXT_H
