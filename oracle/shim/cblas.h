/* TEST INFRASTRUCTURE ONLY — CBLAS declarations for compiling the reference's
 * lapack/compute/{reconstructor,cee_cvv}.cpp unchanged into oracle/_ref.
 * The image has no cblas.h; scipy's bundled OpenBLAS exports the standard CBLAS
 * entry points (LP64: 32-bit int) under a "scipy_" prefix, and this header maps
 * the standard names onto them. Enum values are the CBLAS standard's. */
#ifndef MOAO_ORACLE_SHIM_CBLAS_H
#define MOAO_ORACLE_SHIM_CBLAS_H

#ifdef __cplusplus
extern "C" {
#endif

#define OPENBLAS_CONST const
typedef int blasint;

enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 };
enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113 };
enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 };
enum CBLAS_DIAG { CblasNonUnit = 131, CblasUnit = 132 };
enum CBLAS_SIDE { CblasLeft = 141, CblasRight = 142 };

#define MOAO_SHIM_BLAS3(P, T)                                                                   \
  void scipy_cblas_##P##trsm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO,                \
                             enum CBLAS_TRANSPOSE, enum CBLAS_DIAG, blasint, blasint, T,        \
                             const T*, blasint, T*, blasint);                                   \
  void scipy_cblas_##P##syr2k(enum CBLAS_ORDER, enum CBLAS_UPLO, enum CBLAS_TRANSPOSE, blasint, \
                              blasint, T, const T*, blasint, const T*, blasint, T, T*, blasint); \
  void scipy_cblas_##P##symm(enum CBLAS_ORDER, enum CBLAS_SIDE, enum CBLAS_UPLO, blasint,       \
                             blasint, T, const T*, blasint, const T*, blasint, T, T*, blasint); \
  void scipy_cblas_##P##gemm(enum CBLAS_ORDER, enum CBLAS_TRANSPOSE, enum CBLAS_TRANSPOSE,      \
                             blasint, blasint, blasint, T, const T*, blasint, const T*,         \
                             blasint, T, T*, blasint);                                          \
  void scipy_cblas_##P##scal(blasint, T, T*, blasint);

MOAO_SHIM_BLAS3(s, float)
MOAO_SHIM_BLAS3(d, double)

#define cblas_strsm scipy_cblas_strsm
#define cblas_ssyr2k scipy_cblas_ssyr2k
#define cblas_ssymm scipy_cblas_ssymm
#define cblas_sgemm scipy_cblas_sgemm
#define cblas_sscal scipy_cblas_sscal
#define cblas_dtrsm scipy_cblas_dtrsm
#define cblas_dsyr2k scipy_cblas_dsyr2k
#define cblas_dsymm scipy_cblas_dsymm
#define cblas_dgemm scipy_cblas_dgemm
#define cblas_dscal scipy_cblas_dscal

#ifdef __cplusplus
}
#endif

#endif
