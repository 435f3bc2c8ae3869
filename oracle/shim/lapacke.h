/* TEST INFRASTRUCTURE ONLY — the LAPACKE entry points the reference's
 * lapack/compute code calls (potrf, lacpy, laset), mapped onto scipy's bundled
 * OpenBLAS, which exports them with a "scipy_" prefix (LP64). See cblas.h. */
#ifndef MOAO_ORACLE_SHIM_LAPACKE_H
#define MOAO_ORACLE_SHIM_LAPACKE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef int lapack_int;
#define LAPACK_ROW_MAJOR 101
#define LAPACK_COL_MAJOR 102

#define MOAO_SHIM_LAPACKE(P, T)                                                         \
  lapack_int scipy_LAPACKE_##P##potrf(int, char, lapack_int, T*, lapack_int);           \
  lapack_int scipy_LAPACKE_##P##lacpy(int, char, lapack_int, lapack_int, const T*,      \
                                      lapack_int, T*, lapack_int);                      \
  lapack_int scipy_LAPACKE_##P##laset(int, char, lapack_int, lapack_int, T, T, T*, lapack_int);

MOAO_SHIM_LAPACKE(s, float)
MOAO_SHIM_LAPACKE(d, double)

#define LAPACKE_spotrf scipy_LAPACKE_spotrf
#define LAPACKE_slacpy scipy_LAPACKE_slacpy
#define LAPACKE_slaset scipy_LAPACKE_slaset
#define LAPACKE_dpotrf scipy_LAPACKE_dpotrf
#define LAPACKE_dlacpy scipy_LAPACKE_dlacpy
#define LAPACKE_dlaset scipy_LAPACKE_dlaset

#ifdef __cplusplus
}
#endif

#endif
