// Host-side system model with the public layout of the reference's Tomo_struct
// (common/tomo_struct/tomo_struct.hpp:9-94), SysParams
// (common/tomo_struct/sysParams.hpp:8-59) and AtmParams
// (common/tomo_struct/atmParams.hpp:8-28), so driver code written against the
// reference (lapack/moao_lapack.cpp) compiles unchanged against this library.
//
// The geometry is computed in double on the host; it is O(Nx * nLayer) and is
// uploaded to the device by the covariance entry points.
#ifndef MOAO_B200_TOMO_HPP
#define MOAO_B200_TOMO_HPP

#include <string>
#include <vector>

template <typename T>
class SysParams {
 public:
  T diam = 0, obs = 0, tFrame = 0;
  int nW = 0, nLgs = 0, nNgs = 0, nTarget = 0, nssp = 0;
  std::vector<T> gsAlt;
  std::vector<int> gsType;
  std::vector<T> alphaX_as, alphaY_as, XPup, YPup, thetaML, thetaCam, sensibilite,
      tracking;
  T pasDphi = 0;
  int ncpu = 1;
  std::vector<T> mrNGS;
  T lgsFlux = 0, ngsPixSize = 0, lgsPixSize = 0, lambdaNGS = 0, lambdaLGS = 0,
    bdw_m = 0, throughNGS = 0, throughLGS = 0, throughAtm = 0;
  int RON = 0;
  T lgsCst = 0, spotWidth = 0, lgsAlt = 0, lgsDepth = 0;
  std::vector<T> targetX_as, targetY_as;
  // Read from a legacy benchmark file (datafile/benchmark/*/sys-params.txt):
  // its uniform noise variance replaces the photometric noise model.
  int legacy = 0;
  T noiseVar = 0;

  SysParams() = default;
  explicit SysParams(const std::string& sf) { read(sf); }
  // Positional reader of sys-params.txt: one comment line before every value
  // line (SysParams::getParams, common/tomo_struct/sysParams.cpp:166-204).
  // A file of at most 24 value lines is read in the legacy benchmark layout
  // instead (22 fields: diam, obs, nW, Nssp, gsAlt, type, nLgs, alphaX,
  // alphaY, XPup, YPup, thetaML, thetaCam, sensibilite, tracking, pasDphi,
  // ncpu, lgs_cst, noise_var, spot_width, lgs_alt, lgs_depth), the fields it
  // lacks taking the reference constructor's defaults (one on-axis target).
  // Throws std::runtime_error on a missing file or a short vector.
  void read(const std::string& sf);
  void write(const std::string& sf) const;

 private:
  void read_current(const std::string& sf);
};

template <typename T>
class AtmParams {
 public:
  int nLayer = 0;
  T r0 = 0;
  std::vector<T> cn2, h, L0;

  AtmParams() = default;
  explicit AtmParams(const std::string& af) { read(af); }
  void read(const std::string& af);
  void write(const std::string& af) const;
};

template <typename T>
class Tomo_struct {
 public:
  std::string sys_path, atm_path;
  SysParams<T> sys;
  AtmParams<T> atm;

  std::vector<T> X, Y;          // valid subaperture centres on the pupil [Nx]
  std::vector<long> Nssp;       // subapertures across the diameter, per WFS
  std::vector<long> Nsubap;     // valid subapertures per WFS
  std::vector<T> diamPup, sspSize;
  T rmax = 0;
  T qr = 0, bdw = 0;
  std::vector<T> mr, throughput, alphaX, alphaY, targetX, targetY;
  int Nx = 0;
  int Nslopes = 0;
  int part = 0;
  T sNGS2 = 0, sLGS2 = 0;
  std::vector<T> pixSize, lgsExt, lgsTheta;
  std::vector<T> noiseNGS, noiseLGSxx, noiseLGSyy, noiseLGSxy;
  std::vector<long> indexL0;
  std::vector<T> L0diff;
  std::vector<T> u, v;          // subapertures projected on each layer [nLayer*Nx]
  std::vector<T> sspSizeL;      // subaperture size on each layer [nW*nLayer]
  long nsubaps_offaxis = 0;

  // Incremented whenever the geometry tables change (atmosphere or target);
  // device caches compare it to decide whether to re-upload.
  unsigned long long version = 0;

  Tomo_struct() = default;
  Tomo_struct(const std::string& sf, const std::string& af);

  void initSys();
  void initAtm();
  void updateAtm(const std::string& af = "");
  // Replace the profile from arrays (no file); recomputes like updateAtm.
  void setProfile(int nLayer, const T* cn2, const T* h, const T* L0);
  void setTarget(int tarInd);
  void setTargetCoord(T aX, T aY, int toRad = 0);
  void updateSeeing();
  void updateNoise();
  void validSubap();
  void generateElongation();
  void projectedSubap();
  long getNMeas() const;
  long getNMeasTS() const;

 private:
  void getSysParams();
  void allocAtm();
  void recomputeAtm();
};

#endif  // MOAO_B200_TOMO_HPP
