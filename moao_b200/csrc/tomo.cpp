// Host system model: parameter files and per-WFS / per-layer geometry.
//
// Follows the reference's definitions step by step because the covariance
// values depend on every one of these numbers bit for bit:
//   getSysParams      common/tomo_struct/tomo_struct.cpp:90-133
//   validSubap        common/tomo_struct/tomo_struct.cpp:380-470
//   generateElongation common/tomo_struct/tomo_struct.cpp:478-495
//   updateAtm         common/tomo_struct/tomo_struct.cpp:213-262
//   projectedSubap    common/tomo_struct/tomo_struct.cpp:502-565
//   updateSeeing      common/tomo_struct/tomo_struct.cpp:314-332
//   updateNoise       common/tomo_struct/tomo_struct.cpp:339-374
//   flux / magnitudeFromFlux  common/tomo_struct/noise.cpp:15-52
#include "moao_b200_tomo.hpp"

#include <cmath>
#include <fstream>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <atomic>

namespace {

const double kRasc = 206265.0;  // arcsec per radian, as used by the reference

// Process-wide geometry version: every change of any model gets a fresh value,
// so device caches can never confuse two models.
std::atomic<unsigned long long> g_version{0};

// ---- positional text format ------------------------------------------------
struct LineReader {
  std::ifstream in;
  std::string path;
  explicit LineReader(const std::string& p) : in(p), path(p) {
    if (!in.is_open()) throw std::runtime_error("Could not open file '" + p + "'!");
  }
  // Skip the comment line, return the value line.
  std::string value_line(const char* what) {
    std::string comment, line;
    if (!std::getline(in, comment) || !std::getline(in, line))
      throw std::runtime_error(std::string("unexpected end of file while reading ") +
                               what + " in '" + path + "'");
    return line;
  }
  template <typename V>
  void scalar(V& v, const char* what) {
    std::istringstream ss(value_line(what));
    if (!(ss >> v))
      throw std::runtime_error(std::string("bad value for ") + what + " in '" + path + "'");
  }
  template <typename V>
  void vec(std::vector<V>& v, const char* what) {
    std::istringstream ss(value_line(what));
    v.clear();
    V x;
    while (ss >> x) v.push_back(x);
  }
};

template <typename V>
void need(const std::vector<V>& v, long n, const char* what) {
  if ((long)v.size() < n)
    throw std::runtime_error(std::string("vector ") + what + " has only " +
                             std::to_string(v.size()) + " elements, requires " +
                             std::to_string(n));
}

template <typename V>
void put_vec(std::ostream& os, const std::vector<V>& v) {
  for (size_t i = 0; i < v.size(); ++i) os << (i ? " " : "") << v[i];
  os << '\n';
}

template <typename T>
T flux(T qr, T mr, T throughput, T d, T t, T bdw) {
  return std::pow(10, qr - 0.4 * mr) * throughput * d * d * t * bdw * 1.e4;
}

template <typename T>
T magnitude_from_flux(T qr, T F, T throughput, T d, T t, T bdw) {
  return -(std::log10(F / (throughput * d * d * bdw * 1.e4 * t)) - qr) / 0.4;
}

}  // namespace

// ============================================================================
// Value lines of a positional parameter file (one comment line before each).
static long value_lines(const std::string& path) {
  std::ifstream in(path);
  if (!in.is_open()) throw std::runtime_error("Could not open file '" + path + "'!");
  long n = 0;
  std::string line;
  while (std::getline(in, line)) ++n;
  return n / 2;
}

template <typename T>
void SysParams<T>::read(const std::string& sf) {
  if (value_lines(sf) <= 24) {
    // Legacy benchmark layout (datafile/benchmark/*/sys-params.txt of the
    // reference, read by its PLASMA-era driver): 22 fields in another order
    // and a uniform noise variance instead of the photometry. The fields it
    // does not carry take the defaults of SysParams' constructor
    // (common/tomo_struct/sysParams.cpp:53-104), one target on axis.
    LineReader r(sf);
    r.scalar(diam, "diam");
    r.scalar(obs, "obs");
    r.scalar(nW, "nW");
    r.scalar(nssp, "Nssp");
    r.vec(gsAlt, "gsAlt");
    r.vec(gsType, "type");
    r.scalar(nLgs, "nLgs");
    r.vec(alphaX_as, "alphaX_as");
    r.vec(alphaY_as, "alphaY_as");
    r.vec(XPup, "XPup");
    r.vec(YPup, "YPup");
    r.vec(thetaML, "thetaML");
    r.vec(thetaCam, "thetaCam");
    r.vec(sensibilite, "sensibilite");
    r.vec(tracking, "tracking");
    r.scalar(pasDphi, "pasDphi");
    r.scalar(ncpu, "ncpu");
    r.scalar(lgsCst, "lgs_cst");
    r.scalar(noiseVar, "noise_var");
    r.scalar(spotWidth, "spot_width");
    r.scalar(lgsAlt, "lgs_alt");
    r.scalar(lgsDepth, "lgs_depth");
    legacy = 1;
    tFrame = 0.004;
    nTarget = 1;
    lgsFlux = 1.e7;
    ngsPixSize = 0.3;
    lgsPixSize = 1.0;
    lambdaNGS = 6.5e-07;
    lambdaLGS = 5.89e-07;
    bdw_m = 3.3e-07;
    throughNGS = 0.425;
    throughLGS = 0.382;
    throughAtm = 0.84;
    RON = 3;
    targetX_as.assign(1, 0);
    targetY_as.assign(1, 0);
    if (nW < 2 || nLgs < 0 || nLgs > nW - 1 || nssp < 1 || diam <= 0 || noiseVar < 0)
      throw std::runtime_error("invalid system sizes in '" + sf + "'");
    mrNGS.assign(nW - nLgs, 0.0);
  } else {
    read_current(sf);
  }
  nNgs = nW - nLgs - 1;
  need(gsAlt, nW, "gsAlt");
  need(gsType, nW, "type");
  need(alphaX_as, nW, "alphaX_as");
  need(alphaY_as, nW, "alphaY_as");
  need(XPup, nW, "XPup");
  need(YPup, nW, "YPup");
  need(thetaML, nW, "thetaML");
  need(thetaCam, nW, "thetaCam");
  need(sensibilite, nW, "sensibilite");
  need(tracking, 3, "tracking");
  need(mrNGS, nW - nLgs, "mrNGS");
  need(targetX_as, nTarget, "targetX_as");
  need(targetY_as, nTarget, "targetY_as");
}

template <typename T>
void SysParams<T>::read_current(const std::string& sf) {
  legacy = 0;
  noiseVar = 0;
  LineReader r(sf);
  r.scalar(diam, "diam");
  r.scalar(obs, "obs");
  r.scalar(tFrame, "tFrame");
  r.scalar(nW, "nW");
  r.scalar(nLgs, "nLgs");
  r.scalar(nTarget, "nTarget");
  r.scalar(nssp, "Nssp");
  r.vec(gsAlt, "gsAlt");
  r.vec(gsType, "type");
  r.vec(alphaX_as, "alphaX_as");
  r.vec(alphaY_as, "alphaY_as");
  r.vec(XPup, "XPup");
  r.vec(YPup, "YPup");
  r.vec(thetaML, "thetaML");
  r.vec(thetaCam, "thetaCam");
  r.vec(sensibilite, "sensibilite");
  r.vec(tracking, "tracking");
  r.scalar(pasDphi, "pasDphi");
  r.scalar(ncpu, "ncpu");
  r.vec(mrNGS, "mrNGS");
  r.scalar(lgsFlux, "lgsFlux");
  r.scalar(ngsPixSize, "ngsPixSize");
  r.scalar(lgsPixSize, "lgsPixSize");
  r.scalar(lambdaNGS, "lambdaNGS");
  r.scalar(lambdaLGS, "lambdaLGS");
  r.scalar(bdw_m, "bdw_m");
  r.scalar(throughNGS, "throughNGS");
  r.scalar(throughLGS, "throughLGS");
  r.scalar(throughAtm, "throughAtm");
  r.scalar(RON, "RON");
  r.scalar(lgsCst, "lgsCst");
  r.scalar(spotWidth, "spotWidth");
  r.scalar(lgsAlt, "lgsAlt");
  r.scalar(lgsDepth, "lgsDepth");
  r.vec(targetX_as, "targetX_as");
  r.vec(targetY_as, "targetY_as");
  if (nW < 2 || nLgs < 0 || nLgs > nW - 1 || nssp < 1 || nTarget < 1 || diam <= 0)
    throw std::runtime_error("invalid system sizes in '" + sf + "'");
}

template <typename T>
void SysParams<T>::write(const std::string& sf) const {
  std::ofstream os(sf);
  if (!os.is_open()) throw std::runtime_error("Could not open file '" + sf + "'!");
  os.precision(17);
  os << "diam\n" << diam << "\nobs\n" << obs << "\ntFrame\n" << tFrame << "\nnW\n" << nW
     << "\nnLgs\n" << nLgs << "\nnTarget\n" << nTarget << "\nNssp\n" << nssp << "\ngsAlt\n";
  put_vec(os, gsAlt);
  os << "type\n"; put_vec(os, gsType);
  os << "alphaX_as\n"; put_vec(os, alphaX_as);
  os << "alphaY_as\n"; put_vec(os, alphaY_as);
  os << "XPup\n"; put_vec(os, XPup);
  os << "YPup\n"; put_vec(os, YPup);
  os << "thetaML\n"; put_vec(os, thetaML);
  os << "thetaCam\n"; put_vec(os, thetaCam);
  os << "sensibility\n"; put_vec(os, sensibilite);
  os << "tracking\n"; put_vec(os, tracking);
  os << "pasDPHI\n" << pasDphi << "\nncpu\n" << ncpu << "\nmrNGS\n";
  put_vec(os, mrNGS);
  os << "lgsFlux\n" << lgsFlux << "\nngsPixSize\n" << ngsPixSize << "\nlgsPixSize\n"
     << lgsPixSize << "\nlambdaNGS\n" << lambdaNGS << "\nlambdaLGS\n" << lambdaLGS
     << "\nbdw_m\n" << bdw_m << "\nthroughNGS\n" << throughNGS << "\nthroughLGS\n"
     << throughLGS << "\nthroughAtm\n" << throughAtm << "\nRON\n" << RON << "\nlgsCst\n"
     << lgsCst << "\nspotWidth\n" << spotWidth << "\nlgsAlt\n" << lgsAlt << "\nlgsDepth\n"
     << lgsDepth << "\ntargetX_as\n";
  put_vec(os, targetX_as);
  os << "targetY_as\n"; put_vec(os, targetY_as);
}

template <typename T>
void AtmParams<T>::read(const std::string& af) {
  LineReader r(af);
  r.scalar(nLayer, "nLayer");
  r.scalar(r0, "r0");
  r.vec(cn2, "cn2");
  r.vec(h, "h");
  r.vec(L0, "L0");
  if (nLayer < 1) throw std::runtime_error("nLayer must be >= 1 in '" + af + "'");
  need(cn2, nLayer, "cn2");
  need(h, nLayer, "h");
  need(L0, nLayer, "L0");
}

template <typename T>
void AtmParams<T>::write(const std::string& af) const {
  std::ofstream os(af);
  if (!os.is_open()) throw std::runtime_error("Could not open file '" + af + "'!");
  os.precision(17);
  os << "nLayer\n" << nLayer << "\nr0\n" << r0 << "\ncn2\n";
  put_vec(os, cn2);
  os << "h\n"; put_vec(os, h);
  os << "L0\n"; put_vec(os, L0);
}

// ============================================================================
template <typename T>
Tomo_struct<T>::Tomo_struct(const std::string& sf, const std::string& af) {
  sys_path = sf;
  initSys();
  atm_path = af;
  initAtm();
}

template <typename T>
void Tomo_struct<T>::initSys() {
  sys = SysParams<T>(sys_path);
  getSysParams();
  validSubap();
  generateElongation();
}

template <typename T>
void Tomo_struct<T>::initAtm() {
  atm = AtmParams<T>();
  updateAtm(atm_path);
}

template <typename T>
void Tomo_struct<T>::getSysParams() {
  const int nW = sys.nW, nL = sys.nLgs;
  qr = 2.9;
  bdw = sys.bdw_m * 1.e10;
  Nssp.assign(nW, sys.nssp);
  pixSize.assign(nW, sys.ngsPixSize);
  throughput.assign(nW, sys.throughNGS);
  for (int w = 0; w < nL; ++w) {
    pixSize[w] = sys.lgsPixSize;
    throughput[w] = sys.throughLGS;
  }
  diamPup.assign(Nssp.begin(), Nssp.end());
  const T inv_rasc = 1 / kRasc;
  alphaX.resize(nW);
  alphaY.resize(nW);
  for (int w = 0; w < nW; ++w) {
    alphaX[w] = inv_rasc * sys.alphaX_as[w];
    alphaY[w] = inv_rasc * sys.alphaY_as[w];
  }
  targetX.assign(nW, 0);
  targetY.assign(nW, 0);
  for (int g = 0; g < sys.nTarget && g < nW; ++g) {
    targetX[g] = inv_rasc * sys.targetX_as[g];
    targetY[g] = inv_rasc * sys.targetY_as[g];
  }
  sspSize.resize(nW);
  for (int w = 0; w < nW; ++w) sspSize[w] = sys.diam / (int)Nssp[w];
  mr.assign(nW, 0);
  for (int k = 0; k < nW - nL; ++k) mr[nL + k] = sys.mrNGS[k];
  const T fluxPerSubapPerFrame = sys.lgsFlux * sys.tFrame *
                                 std::pow(sys.diam / Nssp[0], 2.) * throughput[0] /
                                 sys.throughAtm;
  for (int w = 0; w < nL; ++w)
    mr[w] = magnitude_from_flux<T>(qr, fluxPerSubapPerFrame, throughput[w], sspSize[w],
                                   sys.tFrame, bdw);
}

template <typename T>
void Tomo_struct<T>::validSubap() {
  const int nW = sys.nW;
  Nsubap.assign(nW, 0);
  const T bornemin = -sys.diam / 2.;
  const T Rtel2 = (sys.diam * sys.diam) / 4.;
  X.clear();
  Y.clear();
  for (int n = 0; n < nW; ++n) {
    const long ns = Nssp[n];
    if (ns == 1) {  // single subaperture: the pupil centre
      X.push_back(0.);
      Y.push_back(0.);
      Nsubap[n] = 1;
      continue;
    }
    const T pas = sys.diam / (1. * ns);
    // The reference narrows the obscuration for Nssp == 7 at obs ~ 0.286
    // (common/tomo_struct/tomo_struct.cpp:404-409).
    T Robs2;
    if (ns != 7 || (sys.obs <= 0.285 || sys.obs >= 0.29))
      Robs2 = sys.diam * sys.obs / 2. * sys.diam * sys.obs / 2.;
    else
      Robs2 = sys.diam * 0.285 / 2. * sys.diam * 0.285 / 2.;
    long count = 0;
    for (long i = 0; i < ns; ++i) {
      const T yc = bornemin + pas / 2. * (2. * i + 1.);
      for (long j = 0; j < ns; ++j) {
        const T xc = bornemin + pas / 2. * (2. * j + 1.);
        const T r2 = xc * xc + yc * yc;
        if (!(r2 < Robs2 || r2 >= Rtel2)) {
          X.push_back(xc);
          Y.push_back(yc);
          ++count;
        }
      }
    }
    Nsubap[n] = count;
  }
  Nx = (int)X.size();
}

template <typename T>
void Tomo_struct<T>::generateElongation() {
  lgsExt.assign(Nx, 0);
  lgsTheta.assign(Nx, 0);
  const T toFwhm = kRasc * sys.lgsDepth / (sys.lgsAlt * sys.lgsAlt);
  int k = 0;
  for (int w = 0; w < sys.nLgs; ++w) {
    const T nrm = std::sqrt(alphaX[w] * alphaX[w] + alphaY[w] * alphaY[w]);
    const T lltx = alphaX[w] * (sys.diam / 2. / nrm);
    const T llty = alphaY[w] * (sys.diam / 2. / nrm);
    for (long i = 0; i < Nsubap[w]; ++i, ++k) {
      lgsExt[k] = std::sqrt((std::pow(X[k] - lltx, 2) + std::pow(Y[k] - llty, 2))) * toFwhm;
      lgsTheta[k] = std::atan2((Y[k] - llty) * toFwhm, (X[k] - lltx) * toFwhm);
    }
  }
}

template <typename T>
void Tomo_struct<T>::allocAtm() {
  indexL0.assign(atm.nLayer, 0);
  L0diff.assign((size_t)atm.nLayer * Nx, 0);
  u.assign((size_t)atm.nLayer * Nx, 0);
  v.assign((size_t)atm.nLayer * Nx, 0);
  sspSizeL.assign((size_t)sys.nW * atm.nLayer, 0);
}

template <typename T>
void Tomo_struct<T>::updateAtm(const std::string& af) {
  if (!af.empty()) {
    const int old = atm.nLayer;
    atm_path = af;
    atm.read(atm_path);
    if (old != atm.nLayer) allocAtm();
  }
  recomputeAtm();
}

template <typename T>
void Tomo_struct<T>::setProfile(int nLayer, const T* cn2, const T* h, const T* L0) {
  if (nLayer < 1) throw std::runtime_error("nLayer must be >= 1");
  const int old = atm.nLayer;
  atm.nLayer = nLayer;
  atm.cn2.assign(cn2, cn2 + nLayer);
  atm.h.assign(h, h + nLayer);
  atm.L0.assign(L0, L0 + nLayer);
  if (old != nLayer) allocAtm();
  recomputeAtm();
}

template <typename T>
void Tomo_struct<T>::recomputeAtm() {
  const int nL = atm.nLayer;
  for (int cc = 0; cc < sys.nW * nL; ++cc) {
    const int n = cc / nL, l = cc - n * nL;
    sspSizeL[cc] = sspSize[n] * (1. - sys.gsAlt[n] * atm.h[l]);
  }
  // indexL0: index of each layer's L0 among the distinct values (kept for layout
  // compatibility; the covariance reads L0diff directly).
  std::vector<T> distinct;
  for (int i = 0; i < nL; ++i) {
    size_t j = 0;
    while (j < distinct.size() && distinct[j] != atm.L0[i]) ++j;
    if (j == distinct.size()) distinct.push_back(atm.L0[i]);
    indexL0[i] = (long)j;
  }
  for (int i = 0; i < nL; ++i) L0diff[i] = atm.L0[i];
  projectedSubap();
  updateNoise();
}

template <typename T>
void Tomo_struct<T>::setTarget(int tarInd) {
  if (tarInd < 0 || tarInd >= sys.nTarget) throw std::runtime_error("target index out of range");
  setTargetCoord(targetX[tarInd], targetY[tarInd], 0);
}

template <typename T>
void Tomo_struct<T>::setTargetCoord(T aX, T aY, int toRad) {
  if (toRad) {
    aX /= kRasc;
    aY /= kRasc;
  }
  alphaX[sys.nW - 1] = aX;
  alphaY[sys.nW - 1] = aY;
  projectedSubap();
  updateNoise();
}

template <typename T>
void Tomo_struct<T>::updateSeeing() {
  const T lambda_m = 500. * 1.e-9;
  T r0 = std::accumulate(atm.cn2.begin(), atm.cn2.end(), 0.);
  r0 = std::pow(r0, -3. / 5.);
  sNGS2 = lambda_m / r0 * std::pow(lambda_m / sys.lambdaNGS, 0.2) * kRasc;
  sNGS2 *= sNGS2;
  sLGS2 = lambda_m / r0 * std::pow(lambda_m / sys.lambdaLGS, 0.2) * kRasc;
  sLGS2 *= sLGS2;
}

template <typename T>
void Tomo_struct<T>::updateNoise() {
  noiseNGS.assign(sys.nNgs + 1, 0);
  noiseLGSxx.assign(Nx, 0);
  noiseLGSyy.assign(Nx, 0);
  noiseLGSxy.assign(Nx, 0);
  updateSeeing();
  int k = 0;
  if (sys.legacy) {
    // Legacy noise model of the benchmark files (the PLASMA-era covariance
    // kernels of the reference, plasma/matcov_gpu/matcov_gpu_gb.cu:1265-1297):
    // every NGS slope has variance noise_var; an LGS slope has noise_var across
    // its spot elongation and noise_var (ext^2 + w^2) / w^2 along it (w the spot
    // width, ext the elongation).
    const T v = sys.noiseVar, w2 = sys.spotWidth * sys.spotWidth;
    for (int i = 0; i < sys.nW; ++i) {
      if (i < sys.nLgs) {
        for (long j = 0; j < Nsubap[i]; ++j, ++k) {
          const T longAxis = v * (lgsExt[k] * lgsExt[k] + w2) / w2;
          const T c = std::cos(lgsTheta[k]), s = std::sin(lgsTheta[k]);
          noiseLGSxx[k] = longAxis * c * c + v * s * s;
          noiseLGSyy[k] = longAxis * s * s + v * c * c;
          noiseLGSxy[k] = (longAxis - v) * s * c;
        }
      } else {
        noiseNGS[i - sys.nLgs] = v;
      }
    }
    return;
  }
  for (int i = 0; i < sys.nW; ++i) {
    const T d = (sys.diam / Nssp[i]);
    const T F = flux<T>(qr, mr[i], throughput[i], d, sys.tFrame, bdw);
    const T fact1 = 0.32 / F;
    const T fact2 = 0.82 * std::pow(sys.RON / (F * pixSize[i]), 2);
    if (i < sys.nLgs) {
      const T pe = sLGS2 + (sys.spotWidth * sys.spotWidth);
      const T shortAxis = (fact1 * pe + fact2 * std::pow((pe), 1.5) * std::pow(pe, 0.5));
      for (long j = 0; j < Nsubap[i]; ++j, ++k) {
        const T e2 = lgsExt[k] * lgsExt[k];
        const T longAxis = (fact1 * (pe + e2) + fact2 * std::pow((pe + e2), 1.5) * std::pow(pe, 0.5));
        const T c = std::cos(lgsTheta[k]), s = std::sin(lgsTheta[k]);
        noiseLGSxx[k] = longAxis * std::pow(c, 2) + shortAxis * std::pow(s, 2);
        noiseLGSyy[k] = longAxis * std::pow(s, 2) + shortAxis * std::pow(c, 2);
        noiseLGSxy[k] = (longAxis - shortAxis) * s * c;
      }
    } else {
      noiseNGS[i - sys.nLgs] = (fact1 * sNGS2 + fact2 * sNGS2 * sNGS2);
    }
  }
}

template <typename T>
void Tomo_struct<T>::projectedSubap() {
  const T rad = 3.14159265358979323846 / 180.;
  const int nW = sys.nW;
  std::vector<long> ioff(nW, 0);
  for (int i = 1; i < nW; ++i) ioff[i] = ioff[i - 1] + Nsubap[i - 1];
  for (int l = 0; l < atm.nLayer; ++l) {
    const T hl = atm.h[l];
    for (int n = 0; n < nW; ++n) {
      const T dX = alphaX[n] * hl;
      const T dY = alphaY[n] * hl;
      const T rr = 1. - hl * sys.gsAlt[n];
      const T G = diamPup[n] / (T)(Nssp[n]);
      const T th = sys.thetaML[n] * rad;
      const T ct = std::cos(th), st = std::sin(th);
      for (long i = 0; i < Nsubap[n]; ++i) {
        const long pos = ioff[n] + i;
        const T xtp = X[pos] * G;
        const T ytp = Y[pos] * G;
        T uu = xtp * ct - ytp * st;
        T vv = xtp * st + ytp * ct;
        uu += sys.XPup[n];
        vv += sys.YPup[n];
        u[(size_t)l * Nx + pos] = uu * rr + dX;
        v[(size_t)l * Nx + pos] = vv * rr + dY;
      }
    }
  }
  version = ++g_version;
}

template <typename T>
long Tomo_struct<T>::getNMeas() const {
  return 2 * (Nx - Nsubap[sys.nW - 1]);
}

template <typename T>
long Tomo_struct<T>::getNMeasTS() const {
  return 2 * Nsubap[sys.nLgs + sys.nNgs];
}

template class SysParams<double>;
template class AtmParams<double>;
template class Tomo_struct<double>;
template class SysParams<float>;
template class AtmParams<float>;
template class Tomo_struct<float>;
