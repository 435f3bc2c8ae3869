// The reference's C++ entry points (include/moao_b200_compat.hpp) on top of
// the C ABI. Each call runs on the GPU; host buffers keep the reference's
// in-place contracts.
#include "moao_b200_compat.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "context.h"
#include "moao_b200.h"

namespace {

struct Compat {
  moao_ctx* ctx = nullptr;
  bool mixed = false;
  std::mutex mu;
  // Device-side copies of the callers' tomos, refreshed when their version changes.
  std::map<const void*, std::unique_ptr<moao_tomo>> tomos;
  const moao_tomo* last_cmm_tomo = nullptr;  // tomo of the last type-1 matcov_tile
  long last_cmm_n = 0;
};

Compat& compat() {
  static Compat c;
  static std::once_flag once;
  std::call_once(once, [] {
    const char* dev = std::getenv("MOAO_B200_DEVICE");
    const char* prec = std::getenv("MOAO_B200_PRECISION");
    if (moao_ctx_create(dev ? std::atoi(dev) : 0, &c.ctx) != MOAO_OK) {
      std::fprintf(stderr, "moao_b200: %s\n", moao_last_error());
      std::exit(1);
    }
    c.mixed = prec && std::string(prec) == "mixed";
    if (c.mixed) {
      moao_ctx_set_host_precision(c.ctx, MOAO_PREC_MIXED);
      // the accuracy guard: R's estimated error above the target (default
      // 1e-5, MOAO_B200_ACCURACY, 0 turns it off) falls back to FP64
      const char* acc = std::getenv("MOAO_B200_ACCURACY");
      moao_ctx_set_accuracy(c.ctx, acc ? std::atof(acc) : 1e-5);
    }
  });
  return c;
}

[[noreturn]] void die(const char* where) {
  std::fprintf(stderr, "moao_b200 %s: %s\n", where, moao_last_error());
  std::exit(1);
}

template <typename D, typename S>
std::vector<D> cvt(const std::vector<S>& v) {
  return std::vector<D>(v.begin(), v.end());
}

// Field-by-field copy of a Tomo_struct<float> into double.
void widen(const Tomo_struct<float>& f, Tomo_struct<double>& d) {
  d.sys_path = f.sys_path;
  d.atm_path = f.atm_path;
  const SysParams<float>& s = f.sys;
  SysParams<double>& o = d.sys;
  o.diam = s.diam; o.obs = s.obs; o.tFrame = s.tFrame;
  o.nW = s.nW; o.nLgs = s.nLgs; o.nNgs = s.nNgs; o.nTarget = s.nTarget; o.nssp = s.nssp;
  o.gsAlt = cvt<double>(s.gsAlt); o.gsType = s.gsType;
  o.alphaX_as = cvt<double>(s.alphaX_as); o.alphaY_as = cvt<double>(s.alphaY_as);
  o.XPup = cvt<double>(s.XPup); o.YPup = cvt<double>(s.YPup);
  o.thetaML = cvt<double>(s.thetaML); o.thetaCam = cvt<double>(s.thetaCam);
  o.sensibilite = cvt<double>(s.sensibilite); o.tracking = cvt<double>(s.tracking);
  o.pasDphi = s.pasDphi; o.ncpu = s.ncpu; o.mrNGS = cvt<double>(s.mrNGS);
  o.lgsFlux = s.lgsFlux; o.ngsPixSize = s.ngsPixSize; o.lgsPixSize = s.lgsPixSize;
  o.lambdaNGS = s.lambdaNGS; o.lambdaLGS = s.lambdaLGS; o.bdw_m = s.bdw_m;
  o.throughNGS = s.throughNGS; o.throughLGS = s.throughLGS; o.throughAtm = s.throughAtm;
  o.RON = s.RON; o.lgsCst = s.lgsCst; o.spotWidth = s.spotWidth; o.lgsAlt = s.lgsAlt;
  o.lgsDepth = s.lgsDepth;
  o.targetX_as = cvt<double>(s.targetX_as); o.targetY_as = cvt<double>(s.targetY_as);
  d.atm.nLayer = f.atm.nLayer; d.atm.r0 = f.atm.r0;
  d.atm.cn2 = cvt<double>(f.atm.cn2); d.atm.h = cvt<double>(f.atm.h); d.atm.L0 = cvt<double>(f.atm.L0);
  d.X = cvt<double>(f.X); d.Y = cvt<double>(f.Y);
  d.Nssp = f.Nssp; d.Nsubap = f.Nsubap;
  d.diamPup = cvt<double>(f.diamPup); d.sspSize = cvt<double>(f.sspSize);
  d.rmax = f.rmax; d.qr = f.qr; d.bdw = f.bdw;
  d.mr = cvt<double>(f.mr); d.throughput = cvt<double>(f.throughput);
  d.alphaX = cvt<double>(f.alphaX); d.alphaY = cvt<double>(f.alphaY);
  d.targetX = cvt<double>(f.targetX); d.targetY = cvt<double>(f.targetY);
  d.Nx = f.Nx; d.Nslopes = f.Nslopes; d.part = f.part;
  d.sNGS2 = f.sNGS2; d.sLGS2 = f.sLGS2;
  d.pixSize = cvt<double>(f.pixSize); d.lgsExt = cvt<double>(f.lgsExt);
  d.lgsTheta = cvt<double>(f.lgsTheta);
  d.noiseNGS = cvt<double>(f.noiseNGS); d.noiseLGSxx = cvt<double>(f.noiseLGSxx);
  d.noiseLGSyy = cvt<double>(f.noiseLGSyy); d.noiseLGSxy = cvt<double>(f.noiseLGSxy);
  d.indexL0 = f.indexL0; d.L0diff = cvt<double>(f.L0diff);
  d.u = cvt<double>(f.u); d.v = cvt<double>(f.v); d.sspSizeL = cvt<double>(f.sspSizeL);
  d.nsubaps_offaxis = f.nsubaps_offaxis;
  d.version = f.version;
}

const moao_tomo* device_tomo(Compat& c, const Tomo_struct<double>* t) {
  std::unique_ptr<moao_tomo>& e = c.tomos[t];
  if (!e) {
    e.reset(new moao_tomo);
    e->t.version = ~0ull;
  }
  if (e->t.version != t->version) e->t = *t;
  return e.get();
}

const moao_tomo* device_tomo(Compat& c, const Tomo_struct<float>* t) {
  std::unique_ptr<moao_tomo>& e = c.tomos[t];
  if (!e) {
    e.reset(new moao_tomo);
    e->t.version = ~0ull;
  }
  if (e->t.version != t->version) widen(*t, e->t);
  return e.get();
}

// Column-major copies between T and double buffers (m x n, leading dimension ld).
template <typename T>
std::vector<double> to_double(const T* a, long ld, long m, long n) {
  std::vector<double> d((size_t)ld * (n > 0 ? n - 1 : 0) + (size_t)m);
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) d[(size_t)j * ld + i] = (double)a[(size_t)j * ld + i];
  return d;
}

template <typename T>
void from_double(const std::vector<double>& d, T* a, long ld, long m, long n) {
  for (long j = 0; j < n; ++j)
    for (long i = 0; i < m; ++i) a[(size_t)j * ld + i] = (T)d[(size_t)j * ld + i];
}

template <typename T>
void matcov_impl(T* data, int nrows, int ncols, int xoffset, int yoffset, int lda,
                 Tomo_struct<T>* tomo, int part) {
  Compat& c = compat();
  std::lock_guard<std::mutex> lk(c.mu);
  if (part != 1 && part != 2 && part != 3 && part != 4) {
    // common/compute/matcov.cpp:55-56
    std::fprintf(stderr, "ERROR: unrecognized type_mat %d\n", part);
    std::exit(1);
  }
  const moao_tomo* t = device_tomo(c, tomo);
  if (part == 1) {
    c.last_cmm_tomo = t;
    c.last_cmm_n = tomo->getNMeas();
  }
  moao_status st;
  if (std::is_same<T, double>::value) {
    st = moao_matcov_tile_host(c.ctx, t, reinterpret_cast<double*>(data), nrows, ncols, xoffset,
                               yoffset, lda, part);
  } else {
    std::vector<double> d = to_double(data, lda, nrows, ncols);
    st = moao_matcov_tile_host(c.ctx, t, d.data(), nrows, ncols, xoffset, yoffset, lda, part);
    if (st == MOAO_OK) from_double(d, data, lda, nrows, ncols);
  }
  if (st != MOAO_OK) die("matcov_tile");
}

template <typename T>
void reconstructor_impl(long nmeas, long nmeasts, T* Cmm, long ldCmm, T* Ctm, long ldCtm,
                        long ngal) {
  Compat& c = compat();
  std::lock_guard<std::mutex> lk(c.mu);
  if (c.mixed) {
    if (c.last_cmm_tomo && c.last_cmm_n == nmeas) moao_ctx_set_offsets_from_tomo(c.ctx, c.last_cmm_tomo);
    else moao_ctx_set_offsets(c.ctx, 0, nullptr, nullptr, nullptr);
  }
  moao_solve_report rep;
  moao_status st;
  if (std::is_same<T, double>::value) {
    st = moao_reconstructor_host(c.ctx, nmeas, nmeasts, reinterpret_cast<double*>(Cmm), ldCmm,
                                 reinterpret_cast<double*>(Ctm), ldCtm, ngal, &rep);
  } else {
    std::vector<double> C = to_double(Cmm, ldCmm, nmeas, nmeas);
    const long tcols = nmeas * ngal;  // targets are nmeas*nmeasts apart (ldCtm == nmeasts)
    std::vector<double> R = to_double(Ctm, ldCtm, nmeasts, tcols);
    st = moao_reconstructor_host(c.ctx, nmeas, nmeasts, C.data(), ldCmm, R.data(), ldCtm, ngal,
                                 &rep);
    if (st == MOAO_OK || st == MOAO_ERR_NOT_SPD) from_double(C, Cmm, ldCmm, nmeas, nmeas);
    if (st == MOAO_OK) from_double(R, Ctm, ldCtm, nmeasts, tcols);
  }
  if (st == MOAO_ERR_NOT_SPD) {
    std::printf("An error occured in dpotrf: %d\n", rep.info);  // reconstructor.cpp:34-38
    return;
  }
  if (st != MOAO_OK) die("reconstructor");
}

template <typename T>
void cee_cvv_impl(long nmeas, long nmeasts, long nact, T* Cmm, long ldCmm, T* Cpp, long ldCpp,
                  T* Cpm, long ldCpm, T* R, long ldR, T* Dx, long ldDx, T* Cee, long ldCee,
                  T* Cvv, long ldCvv, T* Tmp, long ldTmp) {
  Compat& c = compat();
  std::lock_guard<std::mutex> lk(c.mu);
  moao_status st;
  if (std::is_same<T, double>::value) {
    st = moao_cee_cvv_host(c.ctx, nmeas, nmeasts, nact, (double*)Cmm, ldCmm, (double*)Cpp, ldCpp,
                           (double*)Cpm, ldCpm, (double*)R, ldR, (double*)Dx, ldDx,
                           (double*)Cee, ldCee, (double*)Cvv, ldCvv, (double*)Tmp, ldTmp);
  } else {
    std::vector<double> a = to_double(Cmm, ldCmm, nmeas, nmeas),
                        b = to_double(Cpp, ldCpp, nmeasts, nmeasts),
                        p = to_double(Cpm, ldCpm, nmeasts, nmeas),
                        r = to_double(R, ldR, nmeasts, nmeas),
                        x = to_double(Dx, ldDx, nact, nmeasts),
                        e = to_double(Cee, ldCee, nmeasts, nmeasts),
                        v = to_double(Cvv, ldCvv, nact, nact),
                        w = to_double(Tmp, ldTmp, nact, nmeasts);
    st = moao_cee_cvv_host(c.ctx, nmeas, nmeasts, nact, a.data(), ldCmm, b.data(), ldCpp,
                           p.data(), ldCpm, r.data(), ldR, x.data(), ldDx, e.data(), ldCee,
                           v.data(), ldCvv, w.data(), ldTmp);
    if (st == MOAO_OK) {
      from_double(b, Cpp, ldCpp, nmeasts, nmeasts);
      from_double(p, Cpm, ldCpm, nmeasts, nmeas);
      from_double(e, Cee, ldCee, nmeasts, nmeasts);
      from_double(v, Cvv, ldCvv, nact, nact);
      from_double(w, Tmp, ldTmp, nact, nmeasts);
    }
  }
  if (st != MOAO_OK) die("Cee_Cvv");
}

}  // namespace

namespace MOAO_COMMON {
template <typename T>
void matcov_tile(T* data, int nrows, int ncols, int xoffset, int yoffset, int lda,
                 Tomo_struct<T>* tomo, int part) {
  matcov_impl(data, nrows, ncols, xoffset, yoffset, lda, tomo, part);
}
template void matcov_tile(float*, int, int, int, int, int, Tomo_struct<float>*, int);
template void matcov_tile(double*, int, int, int, int, int, Tomo_struct<double>*, int);
}  // namespace MOAO_COMMON

namespace MOAO_LAPACK {
template <typename T>
void reconstructor(long nmeas, long nmeasts, T* Cmm, long ldCmm, T* Ctm, long ldCtm, long ngal) {
  reconstructor_impl(nmeas, nmeasts, Cmm, ldCmm, Ctm, ldCtm, ngal);
}
template void reconstructor(long, long, float*, long, float*, long, long);
template void reconstructor(long, long, double*, long, double*, long, long);

template <typename T>
void Cee_Cvv(long nmeas, long nmeasts, long nact, T* Cmm, long ldCmm, T* Cpp, long ldCpp, T* Cpm,
             long ldCpm, T* R, long ldR, T* Dx, long ldDx, T* Cee, long ldCee, T* Cvv, long ldCvv,
             T* Tmp, long ldTmp) {
  cee_cvv_impl(nmeas, nmeasts, nact, Cmm, ldCmm, Cpp, ldCpp, Cpm, ldCpm, R, ldR, Dx, ldDx, Cee,
               ldCee, Cvv, ldCvv, Tmp, ldTmp);
}
template void Cee_Cvv(long, long, long, float*, long, float*, long, float*, long, float*, long,
                      float*, long, float*, long, float*, long, float*, long);
template void Cee_Cvv(long, long, long, double*, long, double*, long, double*, long, double*,
                      long, double*, long, double*, long, double*, long, double*, long);

// B = beta op(B) + alpha A as the reference defines it (cee_cvv.cpp:144-166):
// 'N' elementwise; 'T' reads A and B transposed in place, element by element in
// the reference's loop order (so an in-place call with A == B mirrors as it
// does there).
template <typename T>
void geadd(char trans, long M, long N, T alpha, T* A, long ldA, T beta, T* C, long ldC) {
  if (trans == 'N') {
    for (long i = 0; i < M; ++i)
      for (long j = 0; j < N; ++j) C[i + j * ldC] = beta * C[i + j * ldC] + alpha * A[i + j * ldA];
  } else if (trans == 'T') {
    for (long i = 0; i < M; ++i)
      for (long j = 0; j < N; ++j) C[i * ldC + j] = beta * C[i + j * ldC] + alpha * A[i * ldA + j];
  }
}
template void geadd(char, long, long, float, float*, long, float, float*, long);
template void geadd(char, long, long, double, double*, long, double, double*, long);
}  // namespace MOAO_LAPACK

// ------------------------------------------------------------------ intersample
extern "C" {

void intersample_prepare(struct isample_struct* is, long nidx, long np, float Dtel,
                         const char* path) {
  std::memset(is, 0, sizeof(*is));
  // common/tomo_struct/intersample.cpp:190-205
  const long lg = (long)(std::log((double)np) + 0.5);
  is->np = np;
  is->N = std::max(512L, (long)(8 * std::pow(2.0, (double)lg)));
  is->nidx = nidx;
  is->lambda = 1.65e-06;
  is->dactupix = (double)(is->N / (3 * (np - 1)) + 1);
  std::snprintf(is->filename_idx, sizeof(is->filename_idx), "%s/idx.fits", path);
  std::snprintf(is->filename_abs2fi, sizeof(is->filename_abs2fi), "%s/abs2fi.fits", path);
  std::snprintf(is->filename_otftel, sizeof(is->filename_otftel), "%s/otftel.fits", path);
  is->plan_backward = nullptr;
  (void)Dtel;
}

int intersample_init(struct isample_struct* is) {
  Compat& c = compat();
  const long N = is->N;
  long n1 = 0, n2 = 0;
  std::vector<long long> idx(is->nidx);
  if (moao_fits_read_i64(is->filename_idx, &n1, &n2, nullptr, 0) != MOAO_OK || n1 != is->nidx ||
      moao_fits_read_i64(is->filename_idx, &n1, &n2, idx.data(), (long)idx.size()) != MOAO_OK)
    return 0;
  is->idx = (long*)std::malloc(sizeof(long) * is->nidx);
  is->abs2fi = (double*)std::malloc(sizeof(double) * N * N);
  is->otf_tel = (double*)std::malloc(sizeof(double) * N * N);
  const long nmap = (2 * is->np - 1) * (2 * is->np - 1);
  is->Map = (double*)std::calloc(nmap, sizeof(double));
  is->div = (double*)std::calloc(nmap, sizeof(double));
  is->map = (double*)std::calloc(N * N, sizeof(double));
  is->dphi = (double*)std::calloc(N * N, sizeof(double));
  if (!is->idx || !is->abs2fi || !is->otf_tel || !is->Map || !is->div || !is->map || !is->dphi)
    return 0;
  for (long i = 0; i < is->nidx; ++i) is->idx[i] = (long)idx[i];
  if (moao_fits_read_f64(is->filename_abs2fi, &n1, &n2, is->abs2fi, N * N) != MOAO_OK || n1 != N)
    return 0;
  if (moao_fits_read_f64(is->filename_otftel, &n1, &n2, is->otf_tel, N * N) != MOAO_OK || n1 != N)
    return 0;
  for (long i = 0; i < is->nidx; ++i) {
    const long k = is->idx[i] - 1;
    if (k >= 0 && k < nmap) is->div[k] += 1;
  }
  std::lock_guard<std::mutex> lk(c.mu);
  moao_isample* h = nullptr;
  if (moao_intersample_create(c.ctx, is->nidx, is->np, 0.0, is->idx, is->abs2fi, is->otf_tel, &h) !=
      MOAO_OK)
    return 0;
  is->plan_backward = h;
  return 1;
}

void intersample_free(struct isample_struct* is) {
  if (is->plan_backward) moao_intersample_destroy(static_cast<moao_isample*>(is->plan_backward));
  std::free(is->idx);
  std::free(is->abs2fi);
  std::free(is->otf_tel);
  std::free(is->Map);
  std::free(is->div);
  std::free(is->map);
  std::free(is->dphi);
  std::memset(is, 0, sizeof(*is));
}

}  // extern "C"

template <typename T>
int intersample_process(struct isample_struct* is, T* data) {
  if (!is->plan_backward) return 0;
  Compat& c = compat();
  std::vector<double> cvv(data, data + is->nidx);
  std::lock_guard<std::mutex> lk(c.mu);
  if (moao_intersample_process_host(static_cast<moao_isample*>(is->plan_backward), cvv.data(),
                                    is->dphi) != MOAO_OK)
    return 0;
  return 1;
}
template int intersample_process(struct isample_struct*, float*);
template int intersample_process(struct isample_struct*, double*);

// ------------------------------------------------------------------ FITS
int fitsExists(const char* fileName) {
  long n1 = 0, n2 = 0;
  return moao_fits_read_f64(fileName, &n1, &n2, nullptr, 0) == MOAO_OK ? 1 : 0;
}

void getFitsDims(const char* fileName, long* naxes) {
  long n1 = 0, n2 = 0;
  if (moao_fits_read_f64(fileName, &n1, &n2, nullptr, 0) != MOAO_OK) {
    naxes[0] = -1;
    std::fprintf(stderr, "%s\n", moao_last_error());
    return;
  }
  naxes[0] = n1;
  naxes[1] = n2;
}

template <typename T>
void readFits(const char* fileName, T* data) {
  long n1 = 0, n2 = 0;
  if (moao_fits_read_f64(fileName, &n1, &n2, nullptr, 0) != MOAO_OK) {
    std::fprintf(stderr, "%s\n", moao_last_error());
    return;
  }
  std::vector<double> buf((size_t)n1 * n2);
  if (moao_fits_read_f64(fileName, &n1, &n2, buf.data(), (long)buf.size()) != MOAO_OK) {
    std::fprintf(stderr, "%s\n", moao_last_error());
    return;
  }
  std::copy(buf.begin(), buf.end(), data);
}
template void readFits(const char*, float*);
template void readFits(const char*, double*);

template <typename T>
void writeFits(const char* file_name, int nx, int ny, T* data) {
  std::vector<double> buf(data, data + (size_t)nx * ny);
  if (moao_fits_write_f64(file_name, nx, ny, buf.data()) != MOAO_OK)
    std::fprintf(stderr, "%s\n", moao_last_error());
}
template void writeFits(const char*, int, int, float*);
template void writeFits(const char*, int, int, double*);
