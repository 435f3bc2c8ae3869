/*
 * moao_b200 — C ABI of the B200-native MOAO tomographic-reconstructor path.
 *
 * Plain pointers and sizes only. Every matrix is column-major with an explicit
 * leading dimension, exactly like the reference's host buffers. Entry points
 * whose name ends in `_host` take HOST buffers and reproduce the reference's
 * in-place semantics (they copy to the device, compute there, and copy the
 * results back); every other matrix argument is a DEVICE pointer and the call
 * is asynchronous on the context's stream.
 *
 * Nothing here prints or exits; every call returns a moao_status.
 */
#ifndef MOAO_B200_H
#define MOAO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MOAO_OK = 0,
  MOAO_ERR_BAD_ARG = 1,     /* invalid size, type or pointer                  */
  MOAO_ERR_NOT_SPD = 2,     /* Cholesky met a non-positive pivot (see report) */
  MOAO_ERR_OOM = 3,         /* device allocation or admission failed          */
  MOAO_ERR_CUDA = 4,        /* a CUDA runtime call failed                     */
  MOAO_ERR_IO = 5,          /* parameter / input file could not be read       */
  MOAO_ERR_TIMEOUT = 6,     /* a bounded device or host wait ran out          */
  MOAO_ERR_UNSUPPORTED = 7, /* option not available in this build            */
  MOAO_ERR_BUSY = 8,        /* request queue full / request not finished      */
  MOAO_ERR_CANCELLED = 9    /* request cancelled before it ran                */
} moao_status;

typedef enum {
  MOAO_PREC_FP64 = 0,  /* every stage in FP64 (parity path)                    */
  MOAO_PREC_MIXED = 1  /* tensor-core trailing updates + FP64 refinement of R  */
} moao_prec;

/* Human-readable name of a status code (static string). */
const char* moao_status_string(moao_status s);
/* Last error detail recorded on this thread (static buffer, never NULL). */
const char* moao_last_error(void);

/* ------------------------------------------------------------------------ */
/* System model (host side).                                                */
/* Replaces Tomo_struct<T>(sys, atm)  common/tomo_struct/tomo_struct.cpp:11  */
/* ------------------------------------------------------------------------ */
typedef struct moao_tomo moao_tomo;

typedef struct {
  int nW, nLgs, nNgs, nTarget, nLayer, Nx;
  long nmeas;   /* getNMeas   common/tomo_struct/tomo_struct.cpp:570 */
  long nmeasts; /* getNMeasTS common/tomo_struct/tomo_struct.cpp:577 */
  double diam, obs, lgsCst;
  int nssp_ts;  /* Nssp of the truth sensor (intersample np = nssp_ts + 1) */
} moao_tomo_info;

/* Reads sys-params.txt and an atmosphere profile (reference positional format). */
moao_status moao_tomo_create(const char* sys_file, const char* atm_file, moao_tomo** out);
/* Tomo_struct::updateAtm  common/tomo_struct/tomo_struct.cpp:213 */
moao_status moao_tomo_update_atm(moao_tomo* t, const char* atm_file);
/* Replace the profile from arrays (serving path, no file). L0 per layer. */
moao_status moao_tomo_set_profile(moao_tomo* t, int nLayer, const double* cn2,
                                  const double* h, const double* L0);
/* Tomo_struct::setTarget  common/tomo_struct/tomo_struct.cpp:278 */
moao_status moao_tomo_set_target(moao_tomo* t, int target);
moao_status moao_tomo_get_info(const moao_tomo* t, moao_tomo_info* out);
/* Copies a named geometry table (u, v, X, Y, sspSizeL, L0diff, cn2, h, Nsubap,
 * Nssp, noiseNGS, noiseLGSxx, noiseLGSyy, noiseLGSxy, alphaX, alphaY, lgsExt,
 * lgsTheta, mr) into out (capacity cap doubles). Returns the table length, or
 * -1 for an unknown name. out may be NULL to query the length. */
long moao_tomo_table(const moao_tomo* t, const char* name, double* out, long cap);
void moao_tomo_destroy(moao_tomo* t);

/* ------------------------------------------------------------------------ */
/* Device context: one per GPU. Owns a stream, cached device geometry and the */
/* factorisation workspace.                                                  */
/* ------------------------------------------------------------------------ */
typedef struct moao_ctx moao_ctx;

moao_status moao_ctx_create(int device, moao_ctx** out);
void moao_ctx_destroy(moao_ctx* ctx);
/* Run on an external cudaStream_t (NULL = the legacy default stream). */
moao_status moao_ctx_set_stream(moao_ctx* ctx, void* stream);
/* Go back to the context's own (non-blocking) stream. */
moao_status moao_ctx_use_own_stream(moao_ctx* ctx);
void* moao_ctx_stream(moao_ctx* ctx);
moao_status moao_ctx_synchronize(moao_ctx* ctx);
/* Storage of the factor and solve operands on the tensor cores in the mixed
 * path: MOAO_FACTOR_F16X2 (default) = 2 fp16 slices scaled by a power of two
 * per row (~22 bits, 3 products); MOAO_FACTOR_BF16X3 = 3 bf16 slices (~24
 * bits, 6 products). After refinement both reach the same R; F16X2 does half
 * the tensor work and stores a third less. No reference counterpart. */
enum { MOAO_FACTOR_BF16X3 = 0, MOAO_FACTOR_F16X2 = 1 };
moao_status moao_ctx_set_factor_format(moao_ctx* ctx, int format);

/* Block-constant offsets of Cmm known to the caller, for the mixed-precision
 * reconstructor: value[w] is part of every entry (i, j) with begin[w] <= i, j
 * < end[w] (0..32 non-overlapping ranges, values > 0; nranges 0 clears). The
 * mixed path then factors Cmm minus the offsets, whose entries keep their low
 * bits in FP32, and adds the offsets back exactly (Woodbury identity; the
 * refinement residual still uses Cmm as given). The result does not depend on
 * whether offsets are declared, only the refinement's convergence does. No
 * reference counterpart. */
moao_status moao_ctx_set_offsets(moao_ctx* ctx, int nranges, const int* begin, const int* end,
                                 const double* value);
/* The offsets of the covariance model itself: the LGS constant (lgsCst) on the
 * x-x and y-y blocks of every LGS (common/kernels/matcov_kernels.cpp:311-321 of
 * the reference adds it to each such element). */
moao_status moao_ctx_set_offsets_from_tomo(moao_ctx* ctx, const moao_tomo* tomo);

/* Lookahead in the mixed factorisation: the next diagonal block is factored on
 * a side stream of the context while the trailing update leaves sms SMs to it
 * (default 8; 0 turns the lookahead off, at most 64). Same results either way;
 * turn it off when other work should have every SM. No reference counterpart. */
moao_status moao_ctx_set_lookahead(moao_ctx* ctx, int sms);
/* SMs left to the next diagonal block in the last panels of the mixed
 * factorisation, where the trailing update has shrunk (below 24,576 rows: the
 * midpoint of the two settings, below 12,288: this one); values at or below the
 * lookahead setting keep it throughout. No reference counterpart. */
moao_status moao_ctx_set_lookahead_max(moao_ctx* ctx, int sms);
/* Host-buffer cache of the drop-in path (off by default). When on, a whole Cmm
 * (type 1, offsets 0, nrows == ncols) or Ctm (type 3, offsets 0) generated by
 * moao_matcov_tile_host stays on the device, and moao_reconstructor_host skips
 * the upload of a buffer that is the same host pointer with the same shape and
 * leading dimension (Ctm: ngal 1, ldCtm == nmeasts). The caller promises not
 * to modify those host buffers between the two calls (the reference's driver,
 * lapack/moao_lapack.cpp, generates them and passes them on unchanged); every
 * output is still written to the host buffers. Turning it on or off forgets
 * the cached tiles. No reference counterpart. */
moao_status moao_ctx_set_host_cache(moao_ctx* ctx, int on);
/* Tile configuration of the large FP64 products (128 x 64 CTA tiles, 8 warps):
 * 0: K 16 per stage, 4-stage cp.async ring, two CTAs per SM; 1: K 32, 2 stages,
 * two CTAs per SM (default); 2: K 32, 3 stages, one CTA per SM; 3: K 16,
 * 6 stages, one CTA per SM. Bitwise the same results. The batch autotuner picks
 * it per size class. No reference counterpart. */
moao_status moao_ctx_set_gemm_tile(moao_ctx* ctx, int cfg);

/* Tensor-core products of the mixed path (fp16 slice products and the int8
 * residual) on clusters of two CTAs: 256 x 256 tiles with M = 256 MMAs issued
 * by the first CTA of each pair (on = 1), or one CTA per 128 x 256 tile
 * (on = 0, the default; measured 2 % faster on the ELT build). The same
 * products, summed in the same order per element. No reference counterpart. */
moao_status moao_ctx_set_tc_pair(moao_ctx* ctx, int on);

/* Refinement residual E = Ctm - R Cmm of the mixed reconstructor: scheme 1
 * (the default) computes the product of the two operands rounded to the int8
 * slice precision (moao_ctx_set_mixed, default 5 slices = 35 bits per operand)
 * exactly, by the Chinese remainder theorem: residues modulo 11 pairwise
 * coprime moduli <= 256 at nmeas 47,552 (one exact int8 tensor-core GEMM
 * each) and mixed-radix reconstruction in 128-bit integers. Scheme 0 sums the
 * int8 slice products whose slice indices add up to at most slices + 1 (15 at
 * 5 slices). Scheme 1 falls back to 0 where its moduli would not cover the
 * product (nmeas >= 131,072). No reference counterpart. */
moao_status moao_ctx_set_residual(moao_ctx* ctx, int scheme);

/* Accuracy target of the mixed reconstructor (relative Frobenius error of R;
 * 0, the default, turns the check off). With a target, the mixed path also
 * evaluates the residual after its last correction and estimates the error of
 * R as ||dR|| / ||R|| of that correction times the residual's reduction by it;
 * if the estimate exceeds the target (refinement stalls on ill-conditioned
 * systems), the FP64 path computes R from the untouched Cmm and Ctm instead,
 * the report's fallback is 1 and the call still returns MOAO_OK (Cmm then holds
 * the FP64 factor). The estimate is in the report's est_error. No reference
 * counterpart. */
moao_status moao_ctx_set_accuracy(moao_ctx* ctx, double target);

/* Bound of every wait inside the tensor-core kernel of the mixed paths, in
 * polls of its mbarrier (0 restores the default, 2^28: seconds). A wait that
 * runs out ends the kernel early (its copies and tensor-core operations in
 * flight drained, its tensor memory freed) and the call returns
 * MOAO_ERR_TIMEOUT with its outputs undefined; the context stays usable. Applies
 * to this context's own calls (not the batch engine's sub-contexts). No
 * reference counterpart. */
moao_status moao_ctx_set_wait_limit(moao_ctx* ctx, long long polls);

/* Precision of moao_reconstructor_host and moao_cee_cvv_host (default
 * MOAO_PREC_FP64, the reference's behaviour). No reference counterpart. */
moao_status moao_ctx_set_host_precision(moao_ctx* ctx, moao_prec prec);

/* Number of kernels this library launched on the context since creation. */
long long moao_ctx_launch_count(const moao_ctx* ctx);
/* Panel width of the blocked factorisation (default 1024; multiple of 64). */
moao_status moao_ctx_set_block(moao_ctx* ctx, int nb);

/* Options of the mixed-precision reconstructor: bf16 slices of the factor in
 * the first solve (2: ~16 significant bits, 3 products; 3: ~24 bits, 6
 * products; default 3; these two apply to MOAO_FACTOR_BF16X3), slices of the
 * factor in the correction solves (1 to the format's slice count; 1 uses only
 * the leading slice products; 0, the default, picks 1 for MOAO_FACTOR_F16X2
 * and 2 for BF16X3: a correction needs ~1e-2 relative accuracy), int8
 * slices per operand of the refinement residual (2..6, default 5; with the CRT
 * residual of moao_ctx_set_residual they set the operands' precision, 7 bits
 * per slice less one, and the moduli count follows), refinement
 * corrections per target (0..8, default 1), residual tolerance that stops
 * refinement early (default 0) and whether to evaluate the residual again after
 * the last correction (so the report's refine_resid describes the returned R;
 * default 0). */
moao_status moao_ctx_set_mixed(moao_ctx* ctx, int bf16_slices, int corr_slices, int ozaki_slices,
                               int max_refine, double tol, int final_residual);

/* Per-kernel-family device timing. When enabled, every launch of the library's
 * kernels is bracketed by CUDA events on the context stream and accumulated per
 * family together with its algorithmic work (flops for contractions, elements
 * for covariance generation). Families: "gemm_f64", "potrf_leaf", "matcov",
 * "tc_bf16", "tc_int8". */
moao_status moao_ctx_set_kernel_timing(moao_ctx* ctx, int enable);
/* Synchronises, then reports launches, total device ms and total work of one
 * family since the last reset. */
moao_status moao_ctx_kernel_stats(moao_ctx* ctx, const char* family, long long* launches,
                                  double* ms, double* work);
moao_status moao_ctx_reset_kernel_stats(moao_ctx* ctx);

/* ------------------------------------------------------------------------ */
/* Covariance generation.                                                    */
/* Replaces MOAO_COMMON::matcov_tile  common/compute/matcov.cpp:17           */
/*   type_mat 1: Cmm (lower triangle only, like uplo='l')                   */
/*   type_mat 3: Ctm (full)    type_mat 4: Ctt (full)                        */
/*   type_mat 5: Cmm with both triangles written (symmetric fill, no         */
/*               counterpart in the reference; used by the fused pipeline)  */
/* ------------------------------------------------------------------------ */
moao_status moao_matcov_tile(moao_ctx* ctx, const moao_tomo* t, double* d_data,
                             int nrows, int ncols, int xoffset, int yoffset,
                             int lda, int type_mat);
moao_status moao_matcov_tile_host(moao_ctx* ctx, const moao_tomo* t, double* h_data,
                                  int nrows, int ncols, int xoffset, int yoffset,
                                  int lda, int type_mat);

/* ------------------------------------------------------------------------ */
/* Reconstructor R = Ctm . Cmm^-1.                                           */
/* Replaces MOAO_LAPACK::reconstructor  lapack/compute/reconstructor.cpp:32  */
/*   potrf('L', Cmm); per target g: trsm(R,L,T,N) then trsm(R,L,N,N).       */
/* Cmm is overwritten by its lower Cholesky factor (upper triangle left       */
/* untouched) and Ctm by R, ngal targets of nmeasts x nmeas each, stored      */
/* nmeas*nmeasts apart.                                                      */
/* ------------------------------------------------------------------------ */
typedef struct {
  int info;              /* 0, or the 1-based column of a non-positive pivot */
  int refine_steps;      /* mixed path: FP64 refinement steps taken           */
  double refine_resid;   /* mixed path: ||Ctm - R Cmm||_F / ||Ctm||_F at exit  */
  double ms_factor;      /* device time of the Cholesky factorisation         */
  double ms_solve;       /* device time of the two triangular solves           */
  double ms_refine;      /* device time of the refinement                      */
  int fallback;          /* mixed path with an accuracy target: 1 when the     */
                         /* estimate missed it and the FP64 path produced R    */
  double est_error;      /* mixed path with an accuracy target: estimated      */
                         /* relative Frobenius error of the mixed R            */
} moao_solve_report;

moao_status moao_reconstructor(moao_ctx* ctx, long nmeas, long nmeasts, double* d_Cmm,
                               long ldCmm, double* d_Ctm, long ldCtm, long ngal,
                               moao_prec prec, moao_solve_report* rep);
moao_status moao_reconstructor_host(moao_ctx* ctx, long nmeas, long nmeasts, double* Cmm,
                                    long ldCmm, double* Ctm, long ldCtm, long ngal,
                                    moao_solve_report* rep);

/* FP64 reconstructor that allocates no device memory. It has no counterpart in
 * the reference. For callers that cannot allocate while they run: a real-time
 * adaptive-optics controller that must refresh its reconstructor between frames
 * without an allocation stalling in the driver, or an application whose memory
 * pool already owns all of the GPU.
 * Same contract as moao_reconstructor with MOAO_PREC_FP64 (device pointers, Cmm
 * becomes its lower factor, each target's Ctm becomes R; nmeas 0 is a no-op and
 * ngal 0 factors without solving), on the given cudaStream_t (NULL = legacy
 * default stream), which must belong to the current device (otherwise
 * MOAO_ERR_BAD_ARG); returns after the stream has finished the work. Limit:
 * nmeas <= 2048 and nmeasts <= 2048; larger sizes return MOAO_ERR_BAD_ARG.
 * Scratch lives in one fixed 8 MiB device array that every GPU loading the
 * library holds until exit; all calls share it, so calls that overlap on the
 * GPU (other threads, other streams) race and must be serialised by the
 * caller. Each call looks the array's address up in the current CUDA context
 * (cudaGetSymbolAddress, no allocation); the first call in a context loads the
 * library's device code, so make that first call before any stream capture.
 * On a non-positive pivot, *info (if not NULL) receives the 1-based column and
 * MOAO_ERR_NOT_SPD is returned. */
moao_status moao_reconstructor_noalloc(long nmeas, long nmeasts, double* d_Cmm, long ldCmm,
                                       double* d_Ctm, long ldCtm, long ngal, void* stream,
                                       int* info);

/* ---- Dense FP64 building blocks on device buffers (column-major), the ones
 * the blocked factorisation uses, for callers that distribute the
 * factorisation themselves (moao_b200/sharded.py: one Cmm spread over several
 * GPUs). No reference counterpart (the reference's distributed path is
 * ScaLAPACK's pdpotrf, scalapack/moao_scalapack.c).
 * moao_dense_potrf_inv: A (n x n, lower read) <- its Cholesky factor L (lower;
 * the upper triangle is left as is), Ainv <- L^-1 (lower, zeros above); waits
 * for the result; on a non-positive pivot *info (if not NULL) receives the
 * 1-based column and MOAO_ERR_NOT_SPD is returned.
 * moao_dense_gemm: C = alpha A op(B) + beta C, op(B) = B^T if transB, A M x K,
 * C M x N; lowerC writes only C(i, j) with i >= j. Asynchronous on the
 * context's stream. */
moao_status moao_dense_potrf_inv(moao_ctx* ctx, long n, double* A, long lda, double* Ainv,
                                 long ldi, int* info);
moao_status moao_dense_gemm(moao_ctx* ctx, int transB, int lowerC, long M, long N, long K,
                            double alpha, const double* A, long lda, const double* B, long ldb,
                            double beta, double* C, long ldc);

/* ------------------------------------------------------------------------ */
/* Error covariances.                                                        */
/* Replaces MOAO_LAPACK::Cee_Cvv  lapack/compute/cee_cvv.cpp:50-125          */
/*   Cee = Ctt - Ctm R^T - R Ctm^T + R Cmm R^T ;  Cvv = Dx Cee Dx^T           */
/* Same in-place contract: Cpp (Ctt) and Cpm (Ctm) are destroyed, Tmp is     */
/* scratch, Cmm is read as a symmetric matrix from its lower triangle.       */
/* ------------------------------------------------------------------------ */
moao_status moao_cee_cvv(moao_ctx* ctx, long nmeas, long nmeasts, long nact,
                         double* Cmm, long ldCmm, double* Cpp, long ldCpp,
                         double* Cpm, long ldCpm, double* R, long ldR,
                         double* Dx, long ldDx, double* Cee, long ldCee,
                         double* Cvv, long ldCvv, double* Tmp, long ldTmp);
/* Cee_Cvv in a chosen precision. MOAO_PREC_FP64 is moao_cee_cvv. MOAO_PREC_MIXED
 * uses the reconstructor's residual E = Ctm - R Cmm: in exact arithmetic
 * R Cmm R^T = Ctm R^T - E R^T, so Cee = Ctt - R Ctm^T - E R^T; the products
 * R Ctm^T, R Cmm and E R^T run on the int8 tensor cores with the Ozaki
 * splitting (exact int32 accumulation, FP64 sums; the context's int8 slice
 * count, moao_ctx_set_mixed, and its declared offsets of Cmm apply), and
 * Tmp = Dx Cee, Cvv = Tmp Dx^T in FP64. In-place contract of the mixed path: Cpm
 * ends as R Cmm, Cpp (Ctt, lower triangle read) is left as given, Tmp holds
 * Dx sym(Cee). The mixed path synchronises the context stream before it
 * returns (it reads the kernels' error flag). No reference counterpart. */
moao_status moao_cee_cvv_prec(moao_ctx* ctx, long nmeas, long nmeasts, long nact,
                              double* Cmm, long ldCmm, double* Cpp, long ldCpp,
                              double* Cpm, long ldCpm, double* R, long ldR,
                              double* Dx, long ldDx, double* Cee, long ldCee,
                              double* Cvv, long ldCvv, double* Tmp, long ldTmp,
                              moao_prec prec);
/* Host buffers; precision from moao_ctx_set_host_precision (default FP64). */
moao_status moao_cee_cvv_host(moao_ctx* ctx, long nmeas, long nmeasts, long nact,
                              double* Cmm, long ldCmm, double* Cpp, long ldCpp,
                              double* Cpm, long ldCpm, double* R, long ldR,
                              double* Dx, long ldDx, double* Cee, long ldCee,
                              double* Cvv, long ldCvv, double* Tmp, long ldTmp);

/* ------------------------------------------------------------------------ */
/* Intersample PSF.                                                          */
/* Replaces intersample_prepare / intersample_init / intersample_process /   */
/* intersample_free  common/tomo_struct/intersample.cpp:74-333               */
/* ------------------------------------------------------------------------ */
typedef struct moao_isample moao_isample;

typedef struct {
  long N;          /* FFT support (max(512, 8*2^floor(ln(np)+0.5)))   */
  long np;         /* Nssp of the truth sensor + 1                    */
  long nidx;       /* nact*nact                                       */
  double lambda;   /* 1.65e-6 m                                       */
  double dactupix; /* N/(3(np-1)) + 1                                 */
} moao_isample_info;

/* intersample_prepare + intersample_init with caller-provided tables instead of
 * idx.fits / abs2fi.fits / otftel.fits (host arrays; idx is 1-based, nidx long;
 * abs2fi and otf_tel are N*N doubles). */
moao_status moao_intersample_create(moao_ctx* ctx, long nidx, long np, double Dtel,
                                    const long* idx, const double* abs2fi,
                                    const double* otf_tel, moao_isample** out);
moao_status moao_intersample_get_info(const moao_isample* is, moao_isample_info* out);
/* PSF (N x N, FFTW-unnormalised like the reference) from a DEVICE Cvv (nact^2,
 * column-major) into a DEVICE buffer d_psf of N*N doubles. */
moao_status moao_intersample_process(moao_isample* is, const double* d_Cvv, double* d_psf);
/* The three tables without files or the reference's Python tooling, for a truth
 * sensor of nssp subapertures across on a telescope of diameter Dtel and
 * central obscuration obs, DM influence coupling `coupling` (the tooling uses
 * 0.2): the DM actuators (cython/pipeline/commande.py:57-79), idx
 * (generate_file.py:57-76), abs2fi (generate_file.py:79-86) and the telescope
 * OTF (intersample.pyx:151-200). *nact and *N receive the actuator count and
 * the FFT support; idx (nact^2, 1-based, column-major pairs), abs2fi and otf_tel
 * (N x N each) are filled where not NULL (host arrays). With all three NULL
 * only the sizes are computed (ctx may then be NULL); the FFT tables run on
 * the device (the library's FFT). No reference counterpart: the reference reads
 * FITS files. */
moao_status moao_intersample_inputs(moao_ctx* ctx, long nssp, double Dtel, double obs,
                                    double coupling, long* nact, long* N, long* idx,
                                    double* abs2fi, double* otf_tel);
/* moao_intersample_create with the tables of moao_intersample_inputs. */
moao_status moao_intersample_create_synth(moao_ctx* ctx, long nssp, double Dtel, double obs,
                                          double coupling, moao_isample** out);
/* Same with host Cvv in and host PSF out. */
moao_status moao_intersample_process_host(moao_isample* is, const double* Cvv, double* psf);
void moao_intersample_destroy(moao_isample* is);

/* ---- Serving: a persistent request loop on one GPU (no reference
 * counterpart: the reference runs one synchronous driver loop,
 * lapack/moao_lapack.cpp:95-190). Systems (geometry from a parameter file,
 * optional Dx and PSF tables) are registered once; requests carry their own
 * profile and target and arrive at any time. Each is admitted, in arrival
 * order, when a slot (a worker with its own stream and resident workspaces)
 * is idle and the request's device footprint fits the HBM budget beside what
 * the other slots hold, so the device work of concurrent requests overlaps.
 * Results go to the caller's host buffers. Thread-safe. */
typedef struct moao_server moao_server;
typedef struct {
  int device;            /* CUDA device */
  int slots;             /* concurrent requests, 1..16 */
  double hbm_budget_gb;  /* admission budget; <= 0: 90% of the free memory at creation */
  int queue_capacity;    /* queued requests before submit returns BUSY (<= 0: 4096) */
  int nb;                /* panel width (<= 0: library default) */
  int dry_run;           /* 1: host-only model (tests): a request waits dry_run_ms, no GPU */
} moao_server_opts;
typedef struct {
  int system;            /* id from moao_server_add_system */
  int nlayer;            /* profile of this request (copied at submit) */
  const double *cn2, *h, *L0;
  int target;            /* truth-sensor target */
  moao_prec prec;
  double* R;             /* host out: nmeasts x nmeas (ld nmeasts), or NULL */
  double* Cvv;           /* host out: nact x nact, or NULL (system needs Dx) */
  double* psf;           /* host out: N x N, or NULL (system needs the PSF tables) */
  double dry_run_ms;     /* duration of this request in dry_run mode */
} moao_request;
typedef struct {
  moao_status status;    /* MOAO_ERR_BUSY while queued or running */
  int info;              /* Cholesky failure column when NOT_SPD */
  int slot;              /* slot that ran it */
  int refine_steps;
  double refine_resid;
  double queue_ms, run_ms, latency_ms;  /* submit->start, start->done, submit->done */
  double start_ms, end_ms;              /* start and end, ms since server creation */
  double footprint_gb;   /* device bytes admitted for it */
  char message[256];     /* error text when status is an error */
} moao_request_result;
typedef struct {
  long long submitted, completed, failed, cancelled, rejected;
  int max_in_flight;       /* peak concurrent requests */
  double peak_admitted_gb; /* peak device bytes held by slots and admitted requests */
  double budget_gb;
} moao_server_stats;

moao_status moao_server_create(const moao_server_opts* opts, moao_server** out);
/* nact > 0 registers Dx (nact x nmeasts, column-major) for Cvv; idx (nact^2),
 * abs2fi and otf_tel (N x N) add the PSF step. Host-only. */
moao_status moao_server_add_system(moao_server* s, const char* sys_file, const char* atm_file,
                                   long nact, const double* Dx, const long* idx,
                                   const double* abs2fi, const double* otf_tel, int* system_id);
/* The same with the PSF tables synthesised in C++/CUDA for the system's truth
 * sensor (moao_intersample_inputs with the given DM coupling, 0.2 in the
 * reference's tooling): no tables from the caller, no Python. nact must be the
 * synthesised DM's actuator count (moao_intersample_inputs with NULL tables
 * gives it without a GPU); Dx is nact x nmeasts. */
moao_status moao_server_add_system_synth(moao_server* s, const char* sys_file,
                                         const char* atm_file, long nact, const double* Dx,
                                         double coupling, int* system_id);
moao_status moao_server_system_info(moao_server* s, int system, long* nmeas, long* nmeasts,
                                    long* nact, long* psf_n);
/* MOAO_ERR_OOM if the request alone exceeds the budget, MOAO_ERR_BUSY if the
 * queue is full. */
moao_status moao_serve_submit(moao_server* s, const moao_request* r, long long* id);
/* out->status: MOAO_ERR_BUSY (pending), MOAO_ERR_CANCELLED, or the result. */
moao_status moao_serve_poll(moao_server* s, long long id, moao_request_result* out);
/* Blocks until done (timeout_s < 0: no limit); MOAO_ERR_TIMEOUT otherwise. */
moao_status moao_serve_wait(moao_server* s, long long id, double timeout_s,
                            moao_request_result* out);
/* Only before the request starts; MOAO_ERR_BUSY after. */
moao_status moao_serve_cancel(moao_server* s, long long id);
moao_status moao_server_get_stats(moao_server* s, moao_server_stats* out);
/* Cancels queued requests, lets running ones finish, frees everything. */
void moao_server_destroy(moao_server* s);

/* ---- Batched instances: many independent reconstructor builds (covariance
 * generation of Cmm and Ctm from each instance's tomo, factorisation, solves)
 * captured as one CUDA graph over several streams and launched once. Each
 * stream keeps one Cmm / Ctm pair and workspace sized for its largest
 * instance, so device memory is streams x largest, not the sum. Instances run
 * longest first onto the least-loaded stream.
 * Instances with nmeas <= packed_max are instead packed into ONE persistent
 * tile-task kernel (64 x 64 FP64 tiles; the factorisation and both solves of
 * all of them as one level-sorted task list whose CTAs claim tasks from an
 * atomic counter and wait on tile version counters with bounded waits), in a
 * branch of the same graph beside the streams; they hold their own Cmm / Ctm.
 * The tile-task DAG follows the reference's runtime-scheduled tile algorithm
 * (chameleon/compute/reconstructor.cpp:27-55); the batch API itself has no
 * reference counterpart. */
typedef struct {
  const moao_tomo* tomo;  /* system, profile and target of this instance */
  double* d_R;            /* device out: nmeasts x nmeas (ld nmeasts), or NULL */
  int nb;                 /* panel width (tile size); 0: tuned or default */
  /* outputs */
  int status;             /* MOAO_OK, MOAO_ERR_NOT_SPD, MOAO_ERR_TIMEOUT, MOAO_ERR_BAD_ARG */
  int info;               /* failing Cholesky column */
  int nb_used, stream;
  int packed;             /* 1: built by the persistent tile-task kernel (FP64) */
} moao_batch_item;
typedef struct {
  moao_prec prec;         /* mixed: fixed max_refine corrections, no residual checks */
  int streams;            /* most streams to use; 0: tuned (default 4) */
  double hbm_budget_gb;   /* device bytes for the streams' buffers; <= 0: 85% of free */
  long packed_max;        /* nmeas bound of the packed instances; 0: tuned (default
                             none), < 0: none */
  int gemm_tile;          /* FP64 tile configuration + 1 for every instance
                             (moao_ctx_set_gemm_tile); 0: tuned per size class */
  /* outputs */
  double ms_device;       /* device time of the graph launch */
  double ms_build;        /* host time to capture and instantiate the graph */
  long long graph_nodes;
  int streams_used, failed;
  double device_gb;       /* device bytes of the streams' buffers and workspaces */
  int packed_count;       /* instances built by the tile-task kernel */
  long long packed_tasks; /* tasks in its list */
} moao_batch_opts;
moao_status moao_batch_reconstructors(moao_ctx* ctx, int count, moao_batch_item* items,
                                      moao_batch_opts* opts);
/* Autotuner: for each nmeas size class (< 2k, 4k, 8k, 16k, 32k, larger) present
 * in the samples, the panel width (from nb_candidates, default 128, 256, 384,
 * 512, 768, 1024; those above nmeas skipped) with the shortest measured
 * single-instance build, then at that width the FP64 tile configuration
 * (moao_ctx_set_gemm_tile) with the shortest build; then, from the smallest class up while it wins, the
 * classes whose samples build faster together in the tile-task kernel (64 x 64
 * tiles) than as graph instances (the packed_max bound); then the stream count
 * (2, 4, 8) with the shortest batch of all samples; stored on the context. */
moao_status moao_autotune(moao_ctx* ctx, int count, const moao_tomo* const* samples,
                          moao_prec prec, const int* nb_candidates, int ncand);
/* Tuned (or default) panel width per size class (6 entries) and stream count. */
moao_status moao_tuning_get(moao_ctx* ctx, moao_prec prec, int* nb_per_class, int* streams);
/* The packed kernel's task list for instances of the given sizes, host-only (no
 * GPU): 5 ints per task (instance, type, i, j, k; types 0..6 = POTRF(k),
 * TRSM(i,k), UPDATE(i,j,k), forward update (r=i, c=j, source column k),
 * forward diagonal (r=i, c=k), backward update (r=i, c=j, source column k),
 * backward diagonal (r=i, c=k)), in the order the kernel claims them; at most
 * cap tasks are written, *ntasks receives the total and *levels the number of
 * DAG levels. For inspection and for replaying the schedule on the host. */
moao_status moao_packed_task_list(int count, const long* nmeas, const long* nmeasts, int* tasks,
                                  long cap, long* ntasks, int* levels);
/* Tuned FP64 tile configuration per size class (6 entries). */
moao_status moao_tuning_get_gemm(moao_ctx* ctx, moao_prec prec, int* cfg_per_class);
/* Tuned nmeas bound of the packed instances (0: none). */
moao_status moao_tuning_get_packed(moao_ctx* ctx, moao_prec prec, long* packed_max);
moao_status moao_tuning_save(moao_ctx* ctx, const char* path);
moao_status moao_tuning_load(moao_ctx* ctx, const char* path);

/* ---- FITS images (primary HDU, 1-D or 2-D), the file format of the
 * reference's inputs and check outputs (common/io/fits.cpp;
 * common/tomo_struct/intersample.cpp:208-300 reads idx, abs2fi, otftel).
 * Readers convert any BITPIX (8, 16, 32, 64, -32, -64) and apply BZERO/BSCALE;
 * out may be NULL to query NAXIS1/NAXIS2 (NAXIS2 = 1 for a 1-D image). Data
 * order is the file's: NAXIS1 fastest. Host-only: no GPU needed. */
moao_status moao_fits_read_f64(const char* path, long* naxis1, long* naxis2, double* out,
                               long cap);
moao_status moao_fits_read_i64(const char* path, long* naxis1, long* naxis2, long long* out,
                               long cap);
moao_status moao_fits_write_f64(const char* path, long naxis1, long naxis2, const double* data);
moao_status moao_fits_write_i64(const char* path, long naxis1, long naxis2,
                                const long long* data);

#ifdef __cplusplus
}
#endif

#endif /* MOAO_B200_H */
