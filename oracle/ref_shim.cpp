// TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// C entry points over the reference's own common/ code (Tomo_struct,
// SysParams/AtmParams readers, MOAO_COMMON::matcov_tile), compiled unchanged
// from the reference tree by oracle/Makefile into oracle/_ref/libmoao_ref.so.
// The parity tests use it to pin the oracle restatement and the product's
// host geometry against the reference itself.
//
// Reference interfaces wrapped:
//   Tomo_struct<double>(sys, atm)      common/tomo_struct/tomo_struct.cpp:11
//   Tomo_struct::updateAtm             common/tomo_struct/tomo_struct.cpp:213
//   Tomo_struct::setTarget             common/tomo_struct/tomo_struct.cpp:278
//   MOAO_COMMON::matcov_tile           common/compute/matcov.cpp:17
#include <cstring>
#include <cstdio>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "tomo_struct/tomo_struct.hpp"
#include "compute/matcov.hpp"

namespace {
// The reference prints progress to std::cout; keep test output quiet.
struct Mute {
  std::streambuf* old;
  std::ostringstream sink;
  Mute() : old(std::cout.rdbuf(sink.rdbuf())) {}
  ~Mute() { std::cout.rdbuf(old); }
};

template <typename V>
long copy_out(const V& v, double* out, long cap) {
  long n = (long)v.size();
  if (out) {
    for (long i = 0; i < n && i < cap; ++i) out[i] = (double)v[i];
  }
  return n;
}
}  // namespace

extern "C" {

void* ref_tomo_create(const char* sys_file, const char* atm_file) {
  Mute m;
  try {
    return new Tomo_struct<double>(std::string(sys_file), std::string(atm_file));
  } catch (...) {
    return nullptr;
  }
}

void ref_tomo_destroy(void* h) { delete static_cast<Tomo_struct<double>*>(h); }

int ref_tomo_update_atm(void* h, const char* atm_file) {
  Mute m;
  try {
    static_cast<Tomo_struct<double>*>(h)->updateAtm(std::string(atm_file));
  } catch (...) {
    return 1;
  }
  return 0;
}

void ref_tomo_set_target(void* h, int idx) {
  Mute m;
  static_cast<Tomo_struct<double>*>(h)->setTarget(idx);
}

// info[0..7] = nW, nLgs, nNgs, nLayer, Nx, nmeas, nmeasts, nTarget
void ref_tomo_info(void* h, long* info) {
  auto* t = static_cast<Tomo_struct<double>*>(h);
  info[0] = t->sys.nW;
  info[1] = t->sys.nLgs;
  info[2] = t->sys.nNgs;
  info[3] = t->atm.nLayer;
  info[4] = t->Nx;
  info[5] = t->getNMeas();
  info[6] = t->getNMeasTS();
  info[7] = t->sys.nTarget;
}

// Copies one named geometry table into out (capacity cap); returns its length.
long ref_tomo_table(void* h, const char* name, double* out, long cap) {
  auto* t = static_cast<Tomo_struct<double>*>(h);
  std::string n(name);
  if (n == "u") return copy_out(t->u, out, cap);
  if (n == "v") return copy_out(t->v, out, cap);
  if (n == "X") return copy_out(t->X, out, cap);
  if (n == "Y") return copy_out(t->Y, out, cap);
  if (n == "sspSizeL") return copy_out(t->sspSizeL, out, cap);
  if (n == "L0diff") return copy_out(t->L0diff, out, cap);
  if (n == "cn2") return copy_out(t->atm.cn2, out, cap);
  if (n == "h") return copy_out(t->atm.h, out, cap);
  if (n == "Nsubap") return copy_out(t->Nsubap, out, cap);
  if (n == "Nssp") return copy_out(t->Nssp, out, cap);
  if (n == "noiseNGS") return copy_out(t->noiseNGS, out, cap);
  if (n == "noiseLGSxx") return copy_out(t->noiseLGSxx, out, cap);
  if (n == "noiseLGSyy") return copy_out(t->noiseLGSyy, out, cap);
  if (n == "noiseLGSxy") return copy_out(t->noiseLGSxy, out, cap);
  if (n == "alphaX") return copy_out(t->alphaX, out, cap);
  if (n == "alphaY") return copy_out(t->alphaY, out, cap);
  if (n == "lgsExt") return copy_out(t->lgsExt, out, cap);
  if (n == "lgsTheta") return copy_out(t->lgsTheta, out, cap);
  if (n == "mr") return copy_out(t->mr, out, cap);
  if (n == "scalars") {
    std::vector<double> s = {t->sys.diam, t->sys.lgsCst, t->sNGS2, t->sLGS2,
                             t->sys.obs, t->sys.lgsAlt, t->sys.lambdaNGS,
                             t->sys.lambdaLGS};
    return copy_out(s, out, cap);
  }
  return -1;
}

void ref_matcov_tile(void* h, double* data, int nrows, int ncols, int xoffset,
                     int yoffset, int lda, int type_mat) {
  MOAO_COMMON::matcov_tile(data, nrows, ncols, xoffset, yoffset, lda,
                           static_cast<Tomo_struct<double>*>(h), type_mat);
}

}  // extern "C"

#include <thread>
#include <atomic>

extern "C" {
// Multi-threaded driver over the reference's own tile entry point: the matrix
// is cut into ts x ts tiles and each worker calls MOAO_COMMON::matcov_tile on
// whole tiles (tiles above the diagonal of a type-1 matrix compute nothing,
// exactly as in the reference's uplo='l' handling).
void ref_matcov_tiled_mt(void* h, double* data, int nrows, int ncols, int lda,
                         int type_mat, int ts, int nthreads) {
  auto* t = static_cast<Tomo_struct<double>*>(h);
  const int mt = (nrows + ts - 1) / ts, nt = (ncols + ts - 1) / ts;
  const long ntiles = (long)mt * nt;
  std::atomic<long> next(0);
  auto work = [&]() {
    for (;;) {
      long k = next.fetch_add(1);
      if (k >= ntiles) break;
      int tm = (int)(k % mt), tn = (int)(k / mt);
      int r0 = tm * ts, c0 = tn * ts;
      int nr = std::min(ts, nrows - r0), nc = std::min(ts, ncols - c0);
      if (type_mat == 1 && c0 > r0 + nr - 1) continue;  // strictly upper tile
      MOAO_COMMON::matcov_tile(data + (long)c0 * lda + r0, nr, nc, r0, c0, lda,
                               t, type_mat);
    }
  };
  if (nthreads < 1) nthreads = 1;
  std::vector<std::thread> pool;
  for (int i = 1; i < nthreads; ++i) pool.emplace_back(work);
  work();
  for (auto& th : pool) th.join();
}
}  // extern "C"
