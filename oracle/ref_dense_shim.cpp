// TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// C entry points over the reference's own dense and PSF code, compiled
// unchanged from the reference tree by oracle/Makefile into
// oracle/_ref/libmoao_ref_dense.so:
//   MOAO_LAPACK::reconstructor<double>   lapack/compute/reconstructor.cpp:32-58
//   MOAO_LAPACK::Cee_Cvv<double>         lapack/compute/cee_cvv.cpp:50-125
//   MOAO_LAPACK::geadd<double>           lapack/compute/cee_cvv.cpp:144-160
//   intersample_prepare / _init / _process<double> / _free
//                                        common/tomo_struct/intersample.cpp:74-333
// Their third-party dependencies are absent from the image and are supplied
// here (headers in oracle/shim/):
//   * CBLAS / LAPACKE: scipy's bundled OpenBLAS (linked by the Makefile).
//   * FFTW 3.3.7 (the reference README's version): the 2-D real transforms
//     fftw_plan_dft_r2c_2d / fftw_plan_dft_c2r_2d restated from the DFT's
//     definition, X[k0][k1] = sum x[j0][j1] exp(-+2 pi i (j0 k0 / n0 + j1 k1 / n1)),
//     unnormalised, with FFTW's half-spectrum layout; computed as radix-2
//     Cooley-Tukey transforms over rows and columns (n0, n1 powers of two, as
//     intersample_prepare's N always is). c2r takes the half spectrum as the
//     Hermitian half of a full one: a full complex transform along dimension 0,
//     then a real output along dimension 1 from the real parts of its zero and
//     Nyquist columns.
//   * cfitsio 3.420: fits_open_file / fits_read_keys_lng / fits_read_img /
//     fits_close_file over in-memory images registered by ref_intersample().
#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "cee_cvv.hpp"
#include "fitsio.h"
#include "fftw3.h"
#include "intersample.hpp"
#include "reconstructor.hpp"

namespace {

using cplx = std::complex<double>;

// In-place radix-2 transform of n (a power of two) values spaced by stride,
// sign -1 forward, +1 backward, unnormalised.
void fft1d(cplx* a, int n, int stride, int sign) {
  for (int i = 1, j = 0; i < n; ++i) {  // bit reversal
    int bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[(long)i * stride], a[(long)j * stride]);
  }
  for (int len = 2; len <= n; len <<= 1) {
    const int half = len >> 1;
    for (int k = 0; k < half; ++k) {
      const double ang = sign * 2.0 * M_PI * k / len;
      const cplx w(std::cos(ang), std::sin(ang));
      for (int b = 0; b < n; b += len) {
        cplx& u = a[(long)(b + k) * stride];
        cplx& v = a[(long)(b + k + half) * stride];
        const cplx t = w * v;
        v = u - t;
        u = u + t;
      }
    }
  }
}

bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

}  // namespace

struct moao_shim_fftw_plan {
  int n0, n1;
  bool r2c;
  double* real;
  fftw_complex* cpx;
};

extern "C" {

void* fftw_malloc(size_t n) { return std::malloc(n); }
void fftw_free(void* p) { std::free(p); }

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double* in, fftw_complex* out, unsigned) {
  if (!pow2(n0) || !pow2(n1)) return nullptr;
  return new moao_shim_fftw_plan{n0, n1, true, in, out};
}

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex* in, double* out, unsigned) {
  if (!pow2(n0) || !pow2(n1)) return nullptr;
  return new moao_shim_fftw_plan{n0, n1, false, out, in};
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

void fftw_execute(const fftw_plan p) {
  const int n0 = p->n0, n1 = p->n1, h = n1 / 2 + 1;
  std::vector<cplx> row(n1), col((size_t)n0 * h);
  if (p->r2c) {
    for (int i = 0; i < n0; ++i) {  // rows: real -> half spectrum
      for (int j = 0; j < n1; ++j) row[j] = cplx(p->real[(long)i * n1 + j], 0.0);
      fft1d(row.data(), n1, 1, -1);
      for (int j = 0; j < h; ++j) col[(size_t)i * h + j] = row[j];
    }
    for (int j = 0; j < h; ++j) fft1d(col.data() + j, n0, h, -1);  // columns
    for (size_t e = 0; e < col.size(); ++e) {
      p->cpx[e][0] = col[e].real();
      p->cpx[e][1] = col[e].imag();
    }
  } else {
    for (size_t e = 0; e < col.size(); ++e) col[e] = cplx(p->cpx[e][0], p->cpx[e][1]);
    for (int j = 0; j < h; ++j) fft1d(col.data() + j, n0, h, +1);  // columns
    for (int i = 0; i < n0; ++i) {  // rows: Hermitian half -> real
      const cplx* c = col.data() + (size_t)i * h;
      row[0] = cplx(c[0].real(), 0.0);
      row[n1 / 2] = cplx(c[n1 / 2].real(), 0.0);
      for (int k = 1; k < n1 / 2; ++k) {
        row[k] = c[k];
        row[n1 - k] = std::conj(c[k]);
      }
      fft1d(row.data(), n1, 1, +1);
      for (int j = 0; j < n1; ++j) p->real[(long)i * n1 + j] = row[j].real();
    }
  }
}

}  // extern "C"

// ---- cfitsio over registered in-memory images
namespace {
struct Image {
  long n1 = 0, n2 = 0;
  std::vector<double> d;
  std::vector<long> l;
};
std::map<std::string, Image>& images() {
  static std::map<std::string, Image> m;
  return m;
}
std::string base_name(const char* path) {
  const char* s = std::strrchr(path, '/');
  return s ? s + 1 : path;
}
}  // namespace

struct moao_shim_fitsfile {
  Image* img;
};

extern "C" {

int fits_open_file(fitsfile** f, const char* name, int, int* status) {
  auto it = images().find(base_name(name));
  if (it == images().end()) {
    *status = 104;  // cfitsio's FILE_NOT_OPENED
    return *status;
  }
  *f = new moao_shim_fitsfile{&it->second};
  return 0;
}

int fits_read_keys_lng(fitsfile* f, const char*, int nstart, int nmax, long* value, int* nfound,
                       int*) {
  *nfound = 0;
  for (int k = nstart; k < nstart + nmax && k <= 2; ++k) value[(*nfound)++] = k == 1 ? f->img->n1 : f->img->n2;
  return 0;
}

int fits_read_img(fitsfile* f, int type, long first, long n, void*, void* out, int* anynul,
                  int* status) {
  const Image& im = *f->img;
  const long avail = im.n1 * im.n2 - (first - 1);
  if (n > avail) {
    *status = 107;  // END_OF_FILE
    return *status;
  }
  for (long i = 0; i < n; ++i) {
    const long k = first - 1 + i;
    const double v = im.l.empty() ? im.d[k] : (double)im.l[k];
    if (type == TLONG) static_cast<long*>(out)[i] = im.l.empty() ? (long)v : im.l[k];
    else static_cast<double*>(out)[i] = v;
  }
  if (anynul) *anynul = 0;
  return 0;
}

int fits_close_file(fitsfile* f, int*) {
  delete f;
  return 0;
}

void fits_report_error(FILE* stream, int status) {
  std::fprintf(stream, "fits shim: status %d\n", status);
}

// ---- entry points used by oracle/oracle.py

void ref_reconstructor(long nmeas, long nmeasts, double* Cmm, long ldCmm, double* Ctm, long ldCtm,
                       long ngal) {
  MOAO_LAPACK::reconstructor<double>(nmeas, nmeasts, Cmm, ldCmm, Ctm, ldCtm, ngal);
}

void ref_cee_cvv(long nmeas, long nmeasts, long nact, double* Cmm, long ldCmm, double* Cpp,
                 long ldCpp, double* Cpm, long ldCpm, double* R, long ldR, double* Dx, long ldDx,
                 double* Cee, long ldCee, double* Cvv, long ldCvv, double* Tmp, long ldTmp) {
  MOAO_LAPACK::Cee_Cvv<double>(nmeas, nmeasts, nact, Cmm, ldCmm, Cpp, ldCpp, Cpm, ldCpm, R, ldR,
                               Dx, ldDx, Cee, ldCee, Cvv, ldCvv, Tmp, ldTmp);
}

// PSF (N x N, into psf) of Cvv (nact^2 values, nidx = nact^2) through the
// reference's intersample_prepare / _init / _process / _free, with the three
// tables given as arrays in the order the reference reads them from its FITS
// files. Returns N, or -1 if N differs from the tables' size.
long ref_intersample(long nidx, long np, double Dtel, const long* idx, const double* abs2fi,
                     const double* otf, long N, const double* Cvv, double* psf) {
  Image a, b, c;
  a.n1 = nidx;
  a.n2 = 1;
  a.l.assign(idx, idx + nidx);
  b.n1 = b.n2 = c.n1 = c.n2 = N;
  b.d.assign(abs2fi, abs2fi + N * N);
  c.d.assign(otf, otf + N * N);
  images()["idx.fits"] = a;
  images()["abs2fi.fits"] = b;
  images()["otftel.fits"] = c;
  isample_struct is;
  std::memset(&is, 0, sizeof(is));
  intersample_prepare(&is, nidx, np, (float)Dtel, "memory");
  if (is.N != N) return -1;
  intersample_init(&is);
  intersample_process<double>(&is, const_cast<double*>(Cvv));
  std::memcpy(psf, is.dphi, sizeof(double) * N * N);
  intersample_free(&is);
  return N;
}

}  // extern "C"
