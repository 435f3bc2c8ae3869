// A driver written against the reference's C++ interface only (the call
// sequence of its lapack driver: one refinement step building R for every
// target, then one observation computing Cee, Cvv and the PSF per target),
// linked against libmoao_b200 through include/moao_b200_compat.hpp.
//
//   lapack_driver <sys_dir> <atm_file> <out_dir>
//
// sys_dir holds sys-params.txt, Dx.fits, idx.fits, abs2fi.fits, otftel.fits;
// out_dir receives R_g<k>.fits, Cee_g<k>.fits, Cvv_g<k>.fits, psf_g<k>.fits.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "moao_b200_compat.hpp"

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s sys_dir atm_file out_dir\n", argv[0]);
    return 2;
  }
  const std::string sys_dir = argv[1], atm = argv[2], out = argv[3];
  Tomo_struct<double> tomo(sys_dir + "/sys-params.txt", atm);

  long naxes[2] = {0, 0};
  const std::string dx_file = sys_dir + "/Dx.fits";
  getFitsDims(dx_file.c_str(), naxes);
  if (naxes[0] <= 0) return 3;
  const long nact = naxes[0];
  isample_struct isample;
  intersample_prepare(&isample, nact * nact, tomo.Nssp[tomo.sys.nW - 1] + 1, tomo.sys.diam,
                      sys_dir.c_str());
  if (!intersample_init(&isample)) return 4;

  const long nmeas = tomo.getNMeas(), nmeasts = tomo.getNMeasTS();
  const int ntarget = tomo.sys.nTarget;
  std::vector<double> Cmm(nmeas * nmeas), R(nmeasts * nmeas * ntarget), Ctm(nmeasts * nmeas),
      Ctt(nmeasts * nmeasts), Cee(nmeasts * nmeasts), Cvv(nact * nact), Dx(nact * nmeasts),
      Tmp(nact * nmeasts);
  readFits(dx_file.c_str(), Dx.data());

  // refinement step: R for every target from one factorisation
  tomo.updateAtm(atm);
  MOAO_COMMON::matcov_tile(Cmm.data(), nmeas, nmeas, 0, 0, nmeas, &tomo, 1);
  for (int g = 0; g < ntarget; ++g) {
    tomo.setTarget(g);
    MOAO_COMMON::matcov_tile(&R[nmeas * nmeasts * g], nmeasts, nmeas, 0, 0, nmeasts, &tomo, 3);
  }
  MOAO_LAPACK::reconstructor(nmeas, nmeasts, Cmm.data(), nmeas, R.data(), nmeasts, ntarget);

  // one observation: Cee, Cvv and the PSF for every target
  MOAO_COMMON::matcov_tile(Cmm.data(), nmeas, nmeas, 0, 0, nmeas, &tomo, 1);
  for (int g = 0; g < ntarget; ++g) {
    double* Rg = &R[nmeas * nmeasts * g];
    tomo.setTarget(g);
    MOAO_COMMON::matcov_tile(Ctm.data(), nmeasts, nmeas, 0, 0, nmeasts, &tomo, 3);
    MOAO_COMMON::matcov_tile(Ctt.data(), nmeasts, nmeasts, 0, 0, nmeasts, &tomo, 4);
    const std::string k = std::to_string(g);
    writeFits((out + "/R_g" + k + ".fits").c_str(), nmeasts, nmeas, Rg);
    MOAO_LAPACK::Cee_Cvv(nmeas, nmeasts, nact, Cmm.data(), nmeas, Ctt.data(), nmeasts, Ctm.data(),
                         nmeasts, Rg, nmeasts, Dx.data(), nact, Cee.data(), nmeasts, Cvv.data(),
                         nact, Tmp.data(), nact);
    if (!intersample_process(&isample, Cvv.data())) return 5;
    writeFits((out + "/Cee_g" + k + ".fits").c_str(), nmeasts, nmeasts, Cee.data());
    writeFits((out + "/Cvv_g" + k + ".fits").c_str(), nact, nact, Cvv.data());
    writeFits((out + "/psf_g" + k + ".fits").c_str(), isample.N, isample.N, isample.dphi);
  }
  intersample_free(&isample);
  std::printf("nmeas %ld nmeasts %ld nact %ld targets %d\n", nmeas, nmeasts, nact, ntarget);
  return 0;
}
