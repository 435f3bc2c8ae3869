/* TEST INFRASTRUCTURE ONLY — the part of FFTW 3's API (3.3.7, the version the
 * reference's README pins) that common/tomo_struct/intersample.cpp calls, so
 * that file compiles unchanged into oracle/_ref. FFTW is not in the image; the
 * transforms are implemented in oracle/ref_dense_shim.cpp from the DFT's
 * definition with FFTW's conventions: unnormalised, forward sign -1, r2c output
 * and c2r input of n0 x (n1/2 + 1) complex values in row-major order. */
#ifndef MOAO_ORACLE_SHIM_FFTW3_H
#define MOAO_ORACLE_SHIM_FFTW3_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct moao_shim_fftw_plan* fftw_plan;
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
