// Drop-in C++ entry points with the reference's signatures, so its drivers
// (lapack/moao_lapack.cpp, lapack/check_moao_lapack.cpp) link against this
// library unchanged:
//
//   MOAO_COMMON::matcov_tile   common/compute/matcov.hpp:15-18
//   MOAO_LAPACK::reconstructor lapack/compute/reconstructor.hpp:19-21
//   MOAO_LAPACK::Cee_Cvv       lapack/compute/cee_cvv.hpp:19-21
//   MOAO_LAPACK::geadd         lapack/compute/cee_cvv.hpp:22-23
//   intersample_prepare / _init / _free / _process
//                              common/tomo_struct/intersample.hpp:24-63
//   fitsExists, getFitsDims, readFits, writeFits
//                              common/io/fits.hpp:13-19
//
// Buffers are the caller's host memory, column-major, with the reference's
// in-place contracts. The work runs on the GPU through the C ABI
// (moao_b200.h) on one context per process (device from MOAO_B200_DEVICE,
// default 0). Observable error behaviour follows the reference: an unknown
// matcov type prints and exits(1), a failed Cholesky prints
// "An error occured in dpotrf: <col>" and returns with Ctm untouched.
//
// MOAO_B200_PRECISION=mixed selects the mixed-precision reconstructor for
// reconstructor<double> (FP64 otherwise); the LGS constant blocks of the tomo
// last used for a type-1 matcov_tile of the same size are declared as offsets,
// and a build whose estimated error of R exceeds MOAO_B200_ACCURACY (default
// 1e-5; 0 turns the check off) is redone on the FP64 path.
#ifndef MOAO_B200_COMPAT_HPP
#define MOAO_B200_COMPAT_HPP

#include "moao_b200_tomo.hpp"

namespace MOAO_COMMON {
template <typename T>
void matcov_tile(T* data, int nrows, int ncols, int xoffset, int yoffset, int lda,
                 Tomo_struct<T>* tomo, int part);
}  // namespace MOAO_COMMON

namespace MOAO_LAPACK {
template <typename T>
void reconstructor(long nmeas, long nmeasts, T* Cmm, long ldCmm, T* Ctm, long ldCtm, long ngal);
template <typename T>
void Cee_Cvv(long nmeas, long nmeasts, long nact, T* Cmm, long ldCmm, T* Cpp, long ldCpp, T* Cpm,
             long ldCpm, T* R, long ldR, T* Dx, long ldDx, T* Cee, long ldCee, T* Cvv, long ldCvv,
             T* Tmp, long ldTmp);
template <typename T>
void geadd(char trans, long M, long N, T alpha, T* A, long ldA, T beta, T* C, long ldC);
}  // namespace MOAO_LAPACK

// The reference's intersample state (intersample.hpp:24-44). The FFTW members
// are opaque pointers here (same size and position); `dphi` holds the PSF
// after intersample_process, as in the reference.
extern "C" {
struct isample_struct {
  long N;
  long np;
  long nidx;
  double lambda;
  double dactupix;

  long* idx;
  double* abs2fi;
  double* otf_tel;

  double* Map;
  double* div;

  double* map;
  void* tmp;
  double* dphi;

  void* plan_backward;  // this library's device state
  void* plan_forward;

  char filename_idx[256], filename_abs2fi[256], filename_otftel[256];
};

void intersample_prepare(struct isample_struct* isample, long nidx, long nsubap, float Dtel,
                         const char* path);
int intersample_init(struct isample_struct* isample);
void intersample_free(struct isample_struct* isample);
}

template <typename T>
int intersample_process(struct isample_struct* isample, T* data);

// FITS images (read as doubles and converted, written as BITPIX -64 2-D images).
int fitsExists(const char* fileName);
void getFitsDims(const char* fileName, long* naxes);  // naxes[0] = -1 if unreadable
template <typename T>
void readFits(const char* fileName, T* data);
template <typename T>
void writeFits(const char* file_name, int nx, int ny, T* data);

#endif  // MOAO_B200_COMPAT_HPP
