// Covariance generation on sm_100a: Cmm, Ctm, Ctt tiles from the von Karman
// phase structure function.
//
// Model (restated from the reference, common/kernels/matcov_kernels.cpp):
//   DPHI(r) = k1 L0^(5/3) f(2 pi r / L0)                          rodconan :92
//   f(x) = -x^(5/6) K_5/6(x) series (x <= Xlim)                   macdo_x56 :38
//   f(x) = k2 - k3 e^-x x^(1/3) (1 + a1/x + a2/x^2 + a3/x^3)      asymp_macdo :65
//   slope covariances are 4-point DPHI stencils                    cov_XX_gb.. :147-193
//   element = sum over layers of 0.5 cov kk cn2 (+ WFS noise)      compute_element_tiled_4 :206
//   Ctt uses the unprojected truth-sensor positions                compute_element_ts_tile :423
//
// Work decomposition (B200): one thread owns one subaperture pair (i, j) and
// produces the 2x2 slope block {x_i, y_i} x {x_j, y_j} of that pair, so the
// geometry decode, the per-layer loads and the separation are shared by the
// four covariances. When the two WFS have the same subaperture size on a layer
// (every NGS/NGS and equal-altitude LGS/LGS pair) the 16 stencil points of the
// block collapse to 9 distinct DPHI evaluations. Per-layer constants
// (2 pi / L0, k1 L0^(5/3), 0.5 kk cn2) are hoisted to shared memory. The
// kernel is bound by FP64 pipe throughput (cbrt / exp / an 11-term polynomial
// per DPHI), not by HBM: each 8-byte store costs ~10^3 FP64 operations.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "moao_internal.h"

namespace moao {
namespace {

// Constants of the reference model (common/moao_defs.h:15-38).
__constant__ double c_Ga[11] = {0,
                                12.067619015983075,
                                5.17183672113560444,
                                0.795667187867016068,
                                0.0628158306210802181,
                                0.00301515986981185091,
                                9.72632216068338833e-05,
                                2.25320204494595251e-06,
                                3.93000356676612095e-08,
                                5.34694362825451923e-10,
                                5.83302941264329804e-12};
__constant__ double c_Gma[11] = {-3.74878707653729304,   -2.04479295083852408,
                                 -0.360845814853857083,  -0.0313778969438136685,
                                 -0.001622994669507603,  -5.56455315259749673e-05,
                                 -1.35720808599938951e-06, -2.47515152461894642e-08,
                                 -3.50257291219662472e-10, -3.95770950530691961e-12,
                                 -3.65327031259100284e-14};
constexpr double kPi = 3.1415926535897932384626433;
constexpr double kK1 = 0.1716613621245709486;
constexpr double kK2 = 1.00563491799858928388289314170833;
constexpr double kK3 = 1.25331413731550012081;
constexpr double kA1 = 0.22222222222222222222;
constexpr double kA2 = -0.08641975308641974829;
constexpr double kA3 = 0.08001828989483310284;
constexpr double kXlim = 0.75 * 2 * kPi;
constexpr double kLambda2 = 0.00026942094446267851;  // (lambda/(2 pi) rasc)^2

// f(x) / (k1 L0^(5/3)) for x = 2 pi r / L0 >= 0 (so that DPHI = amp * f).
__device__ __forceinline__ double dphi_unit(double x) {
  if (x > kXlim) {
    const double xi = 1.0 / x;
    return kK2 - kK3 * exp(-x) * cbrt(x) * (1.0 + xi * (kA1 + xi * (kA2 + xi * kA3)));
  }
  const double c = cbrt(x);
  const double x2a = x * c * c;  // x^(5/3)
  const double z = 0.25 * x * x;  // (x/2)^2
  double pg = c_Gma[10];
#pragma unroll
  for (int n = 9; n >= 0; --n) pg = fma(pg, z, c_Gma[n]);
  double pa = c_Ga[10];
#pragma unroll
  for (int n = 9; n >= 1; --n) pa = fma(pa, z, c_Ga[n]);
  return -0.5 * (x2a * pg + z * pa);
}

// The same function of s = x^2, without the square root and cube root:
// y = s^(-1/6) = x^(-1/3) by Newton's iteration for y^-6 = s,
//   y <- y (7 - s y^6) / 6        (quadratic convergence, no division),
// started from a single-precision seed 2^(-log2(s) / 6) (relative error
// ~1e-6, so two steps reach double precision). Then x^(5/3) = s y, x = s y^3,
// 1/x = y^3 and x^(1/3) = x y^2. Below s = 1e-30 (a float seed would lose
// range) the direct form is used. The per-pair kernels call the non-inlined
// copy below: their 9 or 16 stencil points per layer then share one body,
// which keeps them inside the instruction cache (inlined, they stalled on
// instruction fetch; ~8% slower). The shared-point kernel inlines it at its
// four call sites (two evaluations per loop iteration, two loops).
// The two uncommon branches are separate functions, so that the series path,
// the one most points take, issues none of their instructions (inlined, the
// compiler predicates them into every evaluation).
__device__ __noinline__ double dphi_tiny_s(double s) { return s > 0 ? dphi_unit(sqrt(s)) : 0.0; }
__device__ __noinline__ double dphi_asym_y(double s, double y) {
  const double xi = y * y * y;  // 1/x
  const double x = s * xi;
  return kK2 - kK3 * exp(-x) * (x * y * y) * (1.0 + xi * (kA1 + xi * (kA2 + xi * kA3)));
}

// The branch is taken on s = x^2 against xlim^2, so the series path never forms
// x (points within an ulp of the boundary may take either form, as they may in
// the reference's own rounding of x).
constexpr double kXlim2 = kXlim * kXlim;

__device__ __forceinline__ double dphi_unit_s_inl(double s) {
  if (!(s > 1e-30)) return dphi_tiny_s(s);
  // seed 2^(-log2(s)/6) from the PTX approximations (flush-to-zero forms: s is
  // a normal float here, and so is the seed), then y <- y (7/6 - (s/6) y^6)
  float l2, y0;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(l2) : "f"((float)s));
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(l2 * (-1.0f / 6.0f)));
  double y = (double)y0;
  const double s6 = s * (1.0 / 6.0);
#pragma unroll
  for (int it = 0; it < 2; ++it) {
    const double y2 = y * y;
    y = y * fma(-s6, y2 * y2 * y2, 7.0 / 6.0);
  }
  if (s > kXlim2) return dphi_asym_y(s, y);
  const double x53 = s * y;        // x^(5/3)
  const double z = 0.25 * s;       // (x/2)^2
  double pg = c_Gma[10];
#pragma unroll
  for (int n = 9; n >= 0; --n) pg = fma(pg, z, c_Gma[n]);
  double pa = c_Ga[10];
#pragma unroll
  for (int n = 9; n >= 1; --n) pa = fma(pa, z, c_Ga[n]);
  return -0.5 * (x53 * pg + z * pa);
}

__device__ __noinline__ double dphi_unit_s(double s) { return dphi_unit_s_inl(s); }

__device__ __forceinline__ double D(double x, double y, double tpl) {
  return dphi_unit_s((tpl * tpl) * (x * x + y * y));
}

constexpr int kMaxJobs = 160;
constexpr int kTileI = 32;
constexpr int kTileJ = 8;

struct Job {
  int m, n;        // row WFS, column WFS
  int i0, ni;      // subaperture range of the row WFS
  int j0, nj;      // subaperture range of the column WFS
  int rb, cb;      // global row / column of the first slope of each WFS
  int tiles_i, tile_base;
};

struct LaunchDesc {
  int njobs, total_tiles, type;
  int r0, c0, nrows, ncols;
  long long ld;
  Job jobs[kMaxJobs];
};

// Element bits: 1 = (x_i, x_j), 2 = (x_i, y_j), 4 = (y_i, x_j), 8 = (y_i, y_j).
template <typename OutT>
__global__ void __launch_bounds__(kTileI* kTileJ)
    matcov_block_kernel(const __grid_constant__ LaunchDesc d, const DevGeometry g,
                        OutT* __restrict__ out) {
  __shared__ double s_tpl[kMaxLayers], s_amp[kMaxLayers], s_w[kMaxLayers];
  __shared__ double s_sm[kMaxLayers], s_sn[kMaxLayers];
  __shared__ int s_job;

  if (threadIdx.x == 0 && threadIdx.y == 0) {
    int k = 0;
    while (k + 1 < d.njobs && d.jobs[k + 1].tile_base <= (int)blockIdx.x) ++k;
    s_job = k;
  }
  __syncthreads();
  const Job& jb = d.jobs[s_job];
  const int nL = g.nLayer;
  const int m = jb.m, n = jb.n;
  const double sspm = g.diam / g.Nssp[m], sspn = g.diam / g.Nssp[n];
  const double kk = kLambda2 / (sspm * sspn);
  for (int l = threadIdx.y * kTileI + threadIdx.x; l < nL; l += kTileI * kTileJ) {
    s_tpl[l] = g.layer[l];
    s_amp[l] = g.layer[nL + l];
    s_w[l] = 0.5 * kk * g.layer[2 * nL + l];
    s_sm[l] = g.layer[3 * nL + m * nL + l];
    s_sn[l] = g.layer[3 * nL + n * nL + l];
  }
  __syncthreads();

  const int t = blockIdx.x - jb.tile_base;
  const int ti = t % jb.tiles_i, tj = t / jb.tiles_i;
  const int i = jb.i0 + ti * kTileI + threadIdx.x;
  const int j = jb.j0 + tj * kTileJ + threadIdx.y;
  if (i >= jb.i0 + jb.ni || j >= jb.j0 + jb.nj) return;

  const int Nm = g.Nsubap[m], Nn = g.Nsubap[n];
  const int rx = jb.rb + i, ry = jb.rb + Nm + i;
  const int cx = jb.cb + j, cy = jb.cb + Nn + j;
  const int r1 = d.r0 + d.nrows, c1 = d.c0 + d.ncols;
  const bool lower = (d.type == 1 || d.type == 5);
  auto want = [&](int r, int c) {
    return r >= d.r0 && r < r1 && c >= d.c0 && c < c1 && (!lower || r >= c);
  };
  unsigned mask = (want(rx, cx) ? 1u : 0u) | (want(rx, cy) ? 2u : 0u) |
                  (want(ry, cx) ? 4u : 0u) | (want(ry, cy) ? 8u : 0u);
  if (!mask) return;

  const int pi = g.off[m] + i, pj = g.off[n] + j;
  double cxx = 0, cxy = 0, cyx = 0, cyy = 0;
  const int tab = g.ttab ? g.tpair[m][n] : -1;
  if (tab >= 0) {
    const int N = g.nssp_grid, W = 2 * N - 1;
    const int2 a = reinterpret_cast<const int2*>(g.grid_cr)[i];
    const int2 b = reinterpret_cast<const int2*>(g.grid_cr)[j];
    const long off = ((long)tab * W * W + (long)(a.y - b.y + N - 1) * W + (a.x - b.x + N - 1)) * 4;
    const double4 t4 = *reinterpret_cast<const double4*>(g.ttab + off);
    cxx = t4.x;
    cxy = t4.y;
    cyx = t4.z;
    cyy = t4.w;
  }
  for (int l = 0; l < nL && tab < 0; ++l) {
    const double sml = s_sm[l], snl = s_sn[l];
    if (!(sml > 0 && snl > 0)) continue;
    const double* ul = g.u + (size_t)l * g.Nx;
    const double* vl = g.v + (size_t)l * g.Nx;
    const double du = __ldg(ul + pi) - __ldg(ul + pj);
    const double dv = __ldg(vl + pi) - __ldg(vl + pj);
    const double s1 = sml * 0.5, s2 = snl * 0.5;
    const double tpl = s_tpl[l];
    const double w = s_w[l] * s_amp[l];
    if (s1 == s2) {
      // Equal subaperture sizes: ac = 0, ad = 2 s; XY and YX share 4 points.
      const double ad = s1 + s2;
      const double d0 = (mask & 9u) ? D(du, dv, tpl) : 0.0;
      if (mask & 1u) {
        const double xx = -d0 + D(du + ad, dv, tpl) + D(du - ad, dv, tpl) - d0;
        cxx += xx * w;
      }
      if (mask & 8u) {
        const double yy = -d0 + D(du, dv + ad, tpl) + D(du, dv - ad, tpl) - d0;
        cyy += yy * w;
      }
      if (mask & 6u) {
        const double pp = D(du + s1, dv + s2, tpl), pm = D(du + s1, dv - s2, tpl);
        const double mp = D(du - s1, dv + s2, tpl), mm = D(du - s1, dv - s2, tpl);
        cxy += (-pm + pp + mm - mp) * w;
        cyx += (-mp + pp + mm - pm) * w;
      }
    } else {
      const double ac = s1 - s2, ad = s1 + s2, bc = -ad, bd = -ac;
      if (mask & 1u)
        cxx += (-D(du + ac, dv, tpl) + D(du + ad, dv, tpl) + D(du + bc, dv, tpl) -
                D(du + bd, dv, tpl)) * w;
      if (mask & 8u)
        cyy += (-D(du, dv + ac, tpl) + D(du, dv + ad, tpl) + D(du, dv + bc, tpl) -
                D(du, dv + bd, tpl)) * w;
      if (mask & 2u)
        cxy += (-D(du + s1, dv - s2, tpl) + D(du + s1, dv + s2, tpl) +
                D(du - s1, dv - s2, tpl) - D(du - s1, dv + s2, tpl)) * w;
      if (mask & 4u)
        cyx += (-D(du - s2, dv + s1, tpl) + D(du + s2, dv + s1, tpl) +
                D(du - s2, dv - s1, tpl) - D(du + s2, dv - s1, tpl)) * w;
    }
  }

  // WFS noise on same-WFS blocks (compute_element_tiled_4 :310-330).
  if (m == n && d.type != 3) {
    if (m < g.nLgs) {
      if (i == j) {
        const int p = g.off[m] + i;
        cxx += g.noiseLGSxx[p];
        cyy += g.noiseLGSyy[p];
        cxy += g.noiseLGSxy[p];
        cyx += g.noiseLGSxy[p];
      }
      cxx += g.lgsCst;
      cyy += g.lgsCst;
    } else if (i == j) {
      cxx += g.noiseNGS[m - g.nLgs];
      cyy += g.noiseNGS[m - g.nLgs];
    }
  }

  const long long ld = d.ld;
  auto store = [&](int r, int c, double val) {
    out[(size_t)(c - d.c0) * ld + (r - d.r0)] = (OutT)val;
    if (d.type == 5 && r != c) out[(size_t)(r - d.c0) * ld + (c - d.r0)] = (OutT)val;
  };
  if (mask & 1u) store(rx, cx, cxx);
  if (mask & 2u) store(rx, cy, cxy);
  if (mask & 4u) store(ry, cx, cyx);
  if (mask & 8u) store(ry, cy, cyy);
}

// ---- Edge-aligned WFS pairs without an offset table (an LGS against an NGS or
// the truth sensor): shared stencil points.
//
// On every layer the projected subaperture of such a WFS spans [centre - s,
// centre + s] with 2 s the projected grid spacing, so its edges are the grid
// lines between neighbouring centres. The 4-point stencils then only ever
// evaluate DPHI at (edge or centre of i) - (edge or centre of j): XX at
// (x-edges, y-centres), YY at (x-centres, y-edges), XY at (x-edge of i minus
// x-centre of j, y-centre of i minus y-edge of j), YX the reverse. A block
// handles a 4x4-cell tile of WFS m against an 8x8-cell tile of WFS n: it
// evaluates the 4 x 1,440 distinct points of a layer once into shared memory
// and each of its 1,024 pairs gathers its 16 values, 5.6 evaluations per pair
// instead of 16.
//
// Each covariance's points form an outer sum s = a[r] + b[c] of two short
// arrays of scaled squared 1-D separations (x part and y part), so a layer
// first fills the 306 entries of those arrays and each point then costs one
// addition before DPHI. Point tables are row-major [r][c]; the i-cell indices
// (a = column, b = row of the i tile) enter rows and columns with strides that
// map the 16 lanes of a half-warp (a, b in 0..3) onto 16 distinct banks, and
// every stencil value of a pair sits at a compile-time offset from one of
// three per-thread bases:
//   XX [ix = 5 ej + ei][iy = 4 rj + ri]      stride 36, base A = (5c + a) 36 + 4e + b
//   YY [iy = 5 fj + fi][ix = 4 cj + ci]      stride 36, base Y = (5e + b) 36 + 4c + a
//   XY [ix = 5 cj + ei][iy = 4 fj + ri]      stride 36, base A
//   YX [ix = 4 ej + ci][iy = 5 rj + fi]      stride 44, base X = (4c + a) 44 + 5e + b
// (e* edge, c* centre index along x; f* edge, r* centre index along y; i
// indices run over the 4x4 tile, j indices over the 8x8 tile.)
constexpr int kEA = 4, kEB = 8;                              // cells per tile side
constexpr int kEThreads = 256;
constexpr int kEPairs = kEA * kEA * kEB * kEB / kEThreads;   // pairs per thread (4)
constexpr int kEKind = (kEA + 1) * kEA * (kEB + 1) * kEB;    // points per covariance (1,440)
constexpr int kEOffYY = 45 * 36, kEOffXY = kEOffYY + 45 * 36, kEOffYX = kEOffXY + 40 * 36;
constexpr int kEPtsTotal = kEOffYX + 36 * 44;                // 6,264 doubles
// scaled squared separations: row array then column array of each covariance
constexpr int kESqXXr = 0, kESqXXc = 45, kESqYYr = 77, kESqYYc = 122, kESqXYr = 154,
              kESqXYc = 194, kESqYXr = 230, kESqYXc = 266, kESqTotal = 306;
constexpr size_t kESmem = (size_t)(kEPtsTotal + kESqTotal) * sizeof(double);
static_assert(kEKind == 45 * 32 && kEKind == 40 * 36 && kEKind % 32 == 0,
              "a covariance's points must fill whole warps");

struct EdgeJob {
  int m, n;        // row WFS, column WFS
  int rb, cb;      // global row / column of the first slope of each WFS
  int tile_base;
};

struct EdgeLaunch {
  int njobs, total_tiles, type;
  int r0, c0, nrows, ncols;
  long long ld;
  EdgeJob jobs[kMaxJobs];
};

// Projected centre of grid column (or row) c of WFS w on a layer:
// ((bornemin + pitch (c + 1/2)) + pup) (1 - h gsAlt) + alpha h, the same
// expression as the host projection (tomo.cpp projectedSubap) with no rotation
// and unit magnification.
__device__ __forceinline__ double grid_centre(const DevGeometry& g, int c, double pup,
                                              double rr, double shift) {
  const double x = g.bornemin + g.pitch / 2. * (2. * c + 1.);
  return (x + pup) * rr + shift;
}

template <typename OutT>
__global__ void __launch_bounds__(kEThreads, 3)
    matcov_edge_kernel(const __grid_constant__ EdgeLaunch d, const DevGeometry g,
                       OutT* __restrict__ out) {
  extern __shared__ double esm[];
  double* pts = esm;                 // XX | YY | XY | YX point tables of the current layer
  double* sq = esm + kEPtsTotal;     // the 8 separation arrays
  __shared__ int s_job;
  const int tid = threadIdx.x;
  if (tid == 0) {
    int k = 0;
    while (k + 1 < d.njobs && d.jobs[k + 1].tile_base <= (int)blockIdx.x) ++k;
    s_job = k;
  }
  __syncthreads();
  const EdgeJob& jb = d.jobs[s_job];
  const int t = blockIdx.x - jb.tile_base;
  const int ta = t % g.ntiles_a, tb = t / g.ntiles_a;
  const int ci0 = g.tiles_a[2 * ta], ri0 = g.tiles_a[2 * ta + 1];
  const int cj0 = g.tiles_b[2 * tb], rj0 = g.tiles_b[2 * tb + 1];
  const int N = g.nssp_grid, m = jb.m, n = jb.n;
  const int Nm = g.Nsubap[m], Nn = g.Nsubap[n];

  // this thread's pairs: i cell (a, b) = tid % 16 of the 4x4 tile, j cells
  // (c, e + 2 q) of the 8x8 tile with c = tid / 16 % 8, e = tid / 128
  const int a = tid % kEA, b = tid / kEA % kEA;
  const int c = tid / (kEA * kEA) % kEB, e = tid / (kEA * kEA * kEB);
  const int ci = ci0 + a, ri = ri0 + b;
  const int vi = (ci < N && ri < N) ? g.cell_idx[ri * N + ci] : -1;
  const int r1 = d.r0 + d.nrows, c1 = d.c0 + d.ncols;
  const bool lower = (d.type == 1 || d.type == 5);
  auto want = [&](int r, int cc) {
    return r >= d.r0 && r < r1 && cc >= d.c0 && cc < c1 && (!lower || r >= cc);
  };
  unsigned mask[kEPairs];
  int vj[kEPairs];
  bool any = false;
#pragma unroll
  for (int q = 0; q < kEPairs; ++q) {
    const int cj = cj0 + c, rj = rj0 + e + 2 * q;
    vj[q] = (cj < N && rj < N) ? g.cell_idx[rj * N + cj] : -1;
    mask[q] = 0;
    if (vi >= 0 && vj[q] >= 0) {
      const int rx = jb.rb + vi, ry = jb.rb + Nm + vi;
      const int cx = jb.cb + vj[q], cy = jb.cb + Nn + vj[q];
      mask[q] = (want(rx, cx) ? 1u : 0u) | (want(rx, cy) ? 2u : 0u) | (want(ry, cx) ? 4u : 0u) |
                (want(ry, cy) ? 8u : 0u);
    }
    any |= mask[q] != 0;
  }
  if (!__syncthreads_or(any)) return;  // the whole block: nothing to write
  const int bA = (5 * c + a) * 36 + 4 * e + b;
  const int bY = kEOffYY + (5 * e + b) * 36 + 4 * c + a;
  const int bX = kEOffYX + (4 * c + a) * 44 + 5 * e + b;

  double acc[kEPairs][4];
#pragma unroll
  for (int q = 0; q < kEPairs; ++q) acc[q][0] = acc[q][1] = acc[q][2] = acc[q][3] = 0.0;
  const int nL = g.nLayer;
  const double sspm = g.diam / g.Nssp[m], sspn = g.diam / g.Nssp[n];
  const double kk = kLambda2 / (sspm * sspn);
  for (int l = 0; l < nL; ++l) {
    const double sml = g.layer[3 * nL + m * nL + l], snl = g.layer[3 * nL + n * nL + l];
    if (!(sml > 0 && snl > 0)) continue;
    const double h = g.layer[3 * nL + g.nW * nL + l];
    const double tpl = g.layer[l];
    const double t2 = tpl * tpl;
    const double w = 0.5 * kk * g.layer[2 * nL + l] * g.layer[nL + l];
    // 1. separations: value = t2 ((C_m(o_m + u) - [edge] s_m/2) - (C_n(o_n + v) - [edge] s_n/2))^2
    for (int k = tid; k < kESqTotal; k += kEThreads) {
      int arr, u0;
      if (k < kESqXXc) { arr = 0; u0 = kESqXXr; }
      else if (k < kESqYYr) { arr = 1; u0 = kESqXXc; }
      else if (k < kESqYYc) { arr = 2; u0 = kESqYYr; }
      else if (k < kESqXYr) { arr = 3; u0 = kESqYYc; }
      else if (k < kESqXYc) { arr = 4; u0 = kESqXYr; }
      else if (k < kESqYXr) { arr = 5; u0 = kESqXYc; }
      else if (k < kESqYXc) { arr = 6; u0 = kESqYXr; }
      else { arr = 7; u0 = kESqYXc; }
      // axis (x = 0), i edge, j edge of each array: XXr XXc YYr YYc XYr XYc YXr YXc
      const bool yax = (0xA6u >> arr) & 1u;     // XXc, YYr, XYc, YXc
      const bool iedge = (0x95u >> arr) & 1u;   // XXr, YYr, XYr, YXc
      const bool jedge = (0x65u >> arr) & 1u;   // XXr, YYr, XYc, YXr
      const int nu = iedge ? kEA + 1 : kEA;
      const int idx = k - u0, u = idx % nu, v = idx / nu;
      const double rm = 1. - h * g.gsAlt[m], rn = 1. - h * g.gsAlt[n];
      const double xm = yax ? grid_centre(g, ri0 + u, g.YPup[m], rm, g.alphaY[m] * h)
                            : grid_centre(g, ci0 + u, g.XPup[m], rm, g.alphaX[m] * h);
      const double xn = yax ? grid_centre(g, rj0 + v, g.YPup[n], rn, g.alphaY[n] * h)
                            : grid_centre(g, cj0 + v, g.XPup[n], rn, g.alphaX[n] * h);
      const double dv = (iedge ? xm - sml * 0.5 : xm) - (jedge ? xn - snl * 0.5 : xn);
      sq[k] = t2 * (dv * dv);
    }
    __syncthreads();
    // 2. points: 4 x 1,440, two independent evaluations per iteration (twice the
    // FP64 chains in flight) with the table indices stepped, not divided out
    {
      // XX and YY (45 x 32 each, row stride 36): column tid % 32, rows tid / 32 + 8 k
      const int cc = tid & 31;
      const double scx = sq[kESqXXc + cc], scy = sq[kESqYYc + cc];
      for (int r = tid >> 5; r < 45; r += kEThreads / 32) {
        const double vx = dphi_unit_s_inl(sq[kESqXXr + r] + scx);
        const double vy = dphi_unit_s_inl(sq[kESqYYr + r] + scy);
        pts[r * 36 + cc] = vx;
        pts[kEOffYY + r * 36 + cc] = vy;
      }
      // XY (40 x 36, stride 36) and YX (36 x 40, stride 44) by flat index
      for (int f = tid; f < kEKind; f += kEThreads) {
        const int r1 = f / 36, c1 = f - 36 * r1;
        const int r2 = f / 40, c2 = f - 40 * r2;
        const double v1 = dphi_unit_s_inl(sq[kESqXYr + r1] + sq[kESqXYc + c1]);
        const double v2 = dphi_unit_s_inl(sq[kESqYXr + r2] + sq[kESqYXc + c2]);
        pts[kEOffXY + r1 * 36 + c1] = v1;
        pts[kEOffYX + r2 * 44 + c2] = v2;
      }
    }
    __syncthreads();
    // 3. the reference's stencils (cov_XX/YY/XY/YX, matcov_kernels.cpp:147-193), in its
    // order: right/top edges are index + 1, left/bottom edges index + 0
#pragma unroll
    for (int q = 0; q < kEPairs; ++q) {
      if (!mask[q]) continue;
      const double* XX = pts + bA + 8 * q;             // XX(a + di, c + dj) at 36 di + 180 dj
      const double* XY = pts + kEOffXY + bA + 8 * q;   // XY(a + di, e + dj) at 36 di + 4 dj
      const double* YX = pts + bX + 10 * q;            // YX(b + di, c + dj) at di + 176 dj
      const double* YY = pts + bY + 360 * q;           // YY(b + di, e + dj) at 36 di + 180 dj
      if (mask[q] & 1u) acc[q][0] += (-XX[216] + XX[36] + XX[180] - XX[0]) * w;
      if (mask[q] & 2u) acc[q][1] += (-XY[40] + XY[36] + XY[4] - XY[0]) * w;
      if (mask[q] & 4u) acc[q][2] += (-YX[177] + YX[1] + YX[176] - YX[0]) * w;
      if (mask[q] & 8u) acc[q][3] += (-YY[216] + YY[36] + YY[180] - YY[0]) * w;
    }
    __syncthreads();
  }
  const long long ld = d.ld;
#pragma unroll
  for (int q = 0; q < kEPairs; ++q) {
    if (!mask[q]) continue;
    const int rx = jb.rb + vi, ry = jb.rb + Nm + vi;
    const int cx = jb.cb + vj[q], cy = jb.cb + Nn + vj[q];
    auto store = [&](int r, int cc, double val) {
      out[(size_t)(cc - d.c0) * ld + (r - d.r0)] = (OutT)val;
      if (d.type == 5 && r != cc) out[(size_t)(r - d.c0) * ld + (cc - d.r0)] = (OutT)val;
    };
    if (mask[q] & 1u) store(rx, cx, acc[q][0]);
    if (mask[q] & 2u) store(rx, cy, acc[q][1]);
    if (mask[q] & 4u) store(ry, cx, acc[q][2]);
    if (mask[q] & 8u) store(ry, cy, acc[q][3]);
  }
}

// Ctt (type 4): truth-sensor auto-covariance from the unprojected positions,
// compute_element_ts_tile (common/kernels/matcov_kernels.cpp:423-483). The
// reference indexes the truth sensor at Nsubap_ts * (nW - 1), which assumes
// every WFS has the same number of valid subapertures; kept as is.
template <typename OutT>
__global__ void __launch_bounds__(kTileI* kTileJ)
    matcov_ts_kernel(const DevGeometry g, int r0, int c0, int nrows, int ncols,
                     long long ld, OutT* __restrict__ out) {
  __shared__ double s_tpl[kMaxLayers], s_w[kMaxLayers];
  const int nL = g.nLayer;
  const int ts = g.nW - 1;
  const int Nt = g.Nsubap[ts];
  const double ssp = g.diam / g.Nssp[ts];
  const double kk = kLambda2 / (ssp * ssp);
  for (int l = threadIdx.y * kTileI + threadIdx.x; l < nL; l += kTileI * kTileJ) {
    s_tpl[l] = g.layer[l];
    s_w[l] = 0.5 * kk * g.layer[2 * nL + l] * g.layer[nL + l];
  }
  __syncthreads();
  // Pair grid covers the subaperture bounding range of the window.
  const int i = blockIdx.x * kTileI + threadIdx.x;
  const int j = blockIdx.y * kTileJ + threadIdx.y;
  if (i >= Nt || j >= Nt) return;
  const int r1 = r0 + nrows, c1 = c0 + ncols;
  auto want = [&](int r, int c) { return r >= r0 && r < r1 && c >= c0 && c < c1; };
  const unsigned mask = (want(i, j) ? 1u : 0u) | (want(i, Nt + j) ? 2u : 0u) |
                        (want(Nt + i, j) ? 4u : 0u) | (want(Nt + i, Nt + j) ? 8u : 0u);
  if (!mask) return;
  const int base = Nt * (g.nW - 1);
  const double du = g.X[base + i] - g.X[base + j];
  const double dv = g.Y[base + i] - g.Y[base + j];
  const double s = ssp * 0.5, ad = 2.0 * s;
  double cxx = 0, cxy = 0, cyx = 0, cyy = 0;
  for (int l = 0; l < nL; ++l) {
    const double tpl = s_tpl[l], w = s_w[l];
    const double d0 = (mask & 9u) ? D(du, dv, tpl) : 0.0;
    if (mask & 1u) cxx += (-d0 + D(du + ad, dv, tpl) + D(du - ad, dv, tpl) - d0) * w;
    if (mask & 8u) cyy += (-d0 + D(du, dv + ad, tpl) + D(du, dv - ad, tpl) - d0) * w;
    if (mask & 6u) {
      const double pp = D(du + s, dv + s, tpl), pm = D(du + s, dv - s, tpl);
      const double mp = D(du - s, dv + s, tpl), mm = D(du - s, dv - s, tpl);
      cxy += (-pm + pp + mm - mp) * w;
      cyx += (-mp + pp + mm - pm) * w;
    }
  }
  auto store = [&](int r, int c, double val) {
    out[(size_t)(c - c0) * ld + (r - r0)] = (OutT)val;
  };
  if (mask & 1u) store(i, j, cxx);
  if (mask & 2u) store(i, Nt + j, cxy);
  if (mask & 4u) store(Nt + i, j, cyx);
  if (mask & 8u) store(Nt + i, Nt + j, cyy);
}

// Offset tables of the equal-projection WFS pairs. Two WFS with the same guide
// star altitude, grid, magnification and rotation see every layer through the
// same affine map up to a constant shift, so the separation of subapertures i
// and j depends only on their grid offset (dc, dr):
//   du = G rr (dx cos - dy sin) + rr (XPup_m - XPup_n) + (alphaX_m - alphaX_n) h
//   dv = G rr (dx sin + dy cos) + rr (YPup_m - YPup_n) + (alphaY_m - alphaY_n) h
// with dx = dc pitch, dy = dr pitch and rr = 1 - h gsAlt. One thread per
// (pair, offset) evaluates the 2x2 slope block over all layers; the matrix
// kernel then gathers from the table. The separation is formed from the grid
// offset instead of from two projected positions, which changes it by rounding
// only (a few ulp of a position).
__global__ void toeplitz_table_kernel(const DevGeometry g, const int2* __restrict__ pairs,
                                      int npairs, double* __restrict__ out) {
  const int N = g.nssp_grid, W = 2 * N - 1;
  const long total = (long)npairs * W * W;
  const int nL = g.nLayer;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const int pidx = (int)(e / ((long)W * W));
    const int off = (int)(e % ((long)W * W));
    const int dr = off / W - (N - 1), dc = off % W - (N - 1);
    const int m = pairs[pidx].x, n = pairs[pidx].y;
    const double dx = dc * g.pitch, dy = dr * g.pitch;
    const double sspm = g.diam / g.Nssp[m], sspn = g.diam / g.Nssp[n];
    const double kk = kLambda2 / (sspm * sspn);
    const double bx = g.G[m] * (dx * g.cth[m] - dy * g.sth[m]);
    const double by = g.G[m] * (dx * g.sth[m] + dy * g.cth[m]);
    double cxx = 0, cxy = 0, cyx = 0, cyy = 0;
    for (int l = 0; l < nL; ++l) {
      const double sml = g.layer[3 * nL + m * nL + l];
      if (!(sml > 0)) continue;
      const double h = g.layer[3 * nL + g.nW * nL + l];
      const double rr = 1. - h * g.gsAlt[m];
      const double du = (bx + (g.XPup[m] - g.XPup[n])) * rr + (g.alphaX[m] - g.alphaX[n]) * h;
      const double dv = (by + (g.YPup[m] - g.YPup[n])) * rr + (g.alphaY[m] - g.alphaY[n]) * h;
      const double s = sml * 0.5, ad = s + s, tpl = g.layer[l];
      const double w = 0.5 * kk * g.layer[2 * nL + l] * g.layer[nL + l];
      const double d0 = D(du, dv, tpl);
      cxx += (-d0 + D(du + ad, dv, tpl) + D(du - ad, dv, tpl) - d0) * w;
      cyy += (-d0 + D(du, dv + ad, tpl) + D(du, dv - ad, tpl) - d0) * w;
      const double pp = D(du + s, dv + s, tpl), pm = D(du + s, dv - s, tpl);
      const double mp = D(du - s, dv + s, tpl), mm = D(du - s, dv - s, tpl);
      cxy += (-pm + pp + mm - mp) * w;
      cyx += (-mp + pp + mm - pm) * w;
    }
    double* o = out + 4 * e;
    o[0] = cxx;
    o[1] = cxy;
    o[2] = cyx;
    o[3] = cyy;
  }
}

// Bounding subaperture range [lo, hi) of a WFS whose x slopes start at global
// index base and y slopes at base + N, intersected with the window [w0, w1).
void subap_range(int base, int N, int w0, int w1, int* lo, int* hi) {
  int a = std::max(w0 - base, 0), b = std::min(w1 - base, N);          // x part
  int c = std::max(w0 - base - N, 0), e = std::min(w1 - base - N, N);  // y part
  int l = N, h = 0;
  if (a < b) { l = std::min(l, a); h = std::max(h, b); }
  if (c < e) { l = std::min(l, c); h = std::max(h, e); }
  *lo = l;
  *hi = h;
}

template <typename OutT>
moao_status launch_impl(const DevGeometry& g, OutT* data, int nrows, int ncols, int xoffset,
                        int yoffset, int lda, int type_mat, cudaStream_t s,
                        long long* launches) {
  if (nrows < 0 || ncols < 0 || xoffset < 0 || yoffset < 0)
    return set_error(MOAO_ERR_BAD_ARG, "matcov: negative size or offset");
  if (nrows == 0 || ncols == 0) return MOAO_OK;
  if (lda < nrows) return set_error(MOAO_ERR_BAD_ARG, "matcov: lda < nrows");
  if (!data) return set_error(MOAO_ERR_BAD_ARG, "matcov: null data");
  if (g.nLayer > kMaxLayers || g.nW > kMaxWfs)
    return set_error(MOAO_ERR_UNSUPPORTED, "matcov: too many layers or WFS");
  const int ts = g.nW - 1;
  long nmeas = 0;
  for (int w = 0; w < ts; ++w) nmeas += 2L * g.Nsubap[w];
  const long nts = 2L * g.Nsubap[ts];

  if (type_mat == 4) {
    if (xoffset + (long)nrows > nts || yoffset + (long)ncols > nts)
      return set_error(MOAO_ERR_BAD_ARG, "matcov: Ctt tile outside nmeasts x nmeasts");
    const int Nt = g.Nsubap[ts];
    if ((long)Nt * g.nW > g.Nx)  // the reference's uniform-Nsubap indexing would overrun X, Y
      return set_error(MOAO_ERR_UNSUPPORTED, "matcov: Ctt needs equal subaperture counts per WFS");
    dim3 grid((Nt + kTileI - 1) / kTileI, (Nt + kTileJ - 1) / kTileJ);
    matcov_ts_kernel<OutT><<<grid, dim3(kTileI, kTileJ), 0, s>>>(g, xoffset, yoffset, nrows,
                                                                 ncols, lda, data);
    if (launches) ++*launches;
    MOAO_CUDA_TRY(cudaGetLastError());
    return MOAO_OK;
  }
  if (type_mat != 1 && type_mat != 2 && type_mat != 3 && type_mat != 5)
    return set_error(MOAO_ERR_BAD_ARG, "matcov: unrecognized type_mat " + std::to_string(type_mat));
  const long rows_total = (type_mat == 3) ? nts : nmeas;
  const long cols_total = (type_mat == 2) ? nts : nmeas;
  if (xoffset + (long)nrows > rows_total || yoffset + (long)ncols > cols_total)
    return set_error(MOAO_ERR_BAD_ARG, "matcov: tile outside the matrix");
  if (type_mat == 5 && (xoffset != yoffset || nrows != ncols))
    return set_error(MOAO_ERR_BAD_ARG, "matcov: type 5 needs a square diagonal tile");

  // Row / column WFS lists and their slope bases.
  std::vector<int> rw, cw, rbase, cbase;
  if (type_mat == 3) { rw.push_back(ts); rbase.push_back(0); }
  else { int b = 0; for (int w = 0; w < ts; ++w) { rw.push_back(w); rbase.push_back(b); b += 2 * g.Nsubap[w]; } }
  if (type_mat == 2) { cw.push_back(ts); cbase.push_back(0); }
  else { int b = 0; for (int w = 0; w < ts; ++w) { cw.push_back(w); cbase.push_back(b); b += 2 * g.Nsubap[w]; } }

  const bool lower = (type_mat == 1 || type_mat == 5);
  std::vector<Job> jobs;
  for (size_t a = 0; a < rw.size(); ++a) {
    for (size_t b = 0; b < cw.size(); ++b) {
      const int m = rw[a], n = cw[b];
      if (lower && m < n) continue;  // entirely above the diagonal
      Job jb{};
      jb.m = m; jb.n = n; jb.rb = rbase[a]; jb.cb = cbase[b];
      int ilo, ihi, jlo, jhi;
      subap_range(jb.rb, g.Nsubap[m], xoffset, xoffset + nrows, &ilo, &ihi);
      subap_range(jb.cb, g.Nsubap[n], yoffset, yoffset + ncols, &jlo, &jhi);
      if (ilo >= ihi || jlo >= jhi) continue;
      jb.i0 = ilo; jb.ni = ihi - ilo; jb.j0 = jlo; jb.nj = jhi - jlo;
      jb.tiles_i = (jb.ni + kTileI - 1) / kTileI;
      jobs.push_back(jb);
    }
  }
  // Edge-aligned pairs without an offset table go to the shared-point kernel.
  std::vector<Job> plain;
  std::vector<EdgeJob> edge;
  for (const Job& jb : jobs) {
    const bool tab = g.ttab && g.tpair[jb.m][jb.n] >= 0;
    if (!tab && jb.m != jb.n && g.aligned[jb.m] && g.aligned[jb.n] && g.cell_idx &&
        g.ntiles_a > 0 && g.ntiles_b > 0) {
      EdgeJob e{};
      e.m = jb.m; e.n = jb.n; e.rb = jb.rb; e.cb = jb.cb;
      edge.push_back(e);
    } else {
      plain.push_back(jb);
    }
  }
  jobs.swap(plain);
  const int per_job = g.ntiles_a * g.ntiles_b;
  for (size_t base = 0; base < edge.size(); base += kMaxJobs) {
    EdgeLaunch d{};
    d.type = type_mat;
    d.r0 = xoffset; d.c0 = yoffset; d.nrows = nrows; d.ncols = ncols; d.ld = lda;
    int tiles = 0;
    for (size_t k = base; k < edge.size() && k < base + kMaxJobs; ++k) {
      EdgeJob e = edge[k];
      e.tile_base = tiles;
      tiles += per_job;
      d.jobs[d.njobs++] = e;
    }
    d.total_tiles = tiles;
    if (tiles == 0) continue;
    static std::atomic<unsigned long long> configured{0};
    MOAO_CUDA_TRY(set_smem_limit(matcov_edge_kernel<OutT>, (int)kESmem, configured));
    matcov_edge_kernel<OutT><<<tiles, kEThreads, kESmem, s>>>(d, g, data);
    if (launches) ++*launches;
    MOAO_CUDA_TRY(cudaGetLastError());
  }
  // Launch in chunks of kMaxJobs jobs.
  for (size_t base = 0; base < jobs.size(); base += kMaxJobs) {
    LaunchDesc d{};
    d.type = type_mat;
    d.r0 = xoffset; d.c0 = yoffset; d.nrows = nrows; d.ncols = ncols; d.ld = lda;
    int tiles = 0;
    for (size_t k = base; k < jobs.size() && k < base + kMaxJobs; ++k) {
      Job jb = jobs[k];
      jb.tile_base = tiles;
      tiles += jb.tiles_i * ((jb.nj + kTileJ - 1) / kTileJ);
      d.jobs[d.njobs++] = jb;
    }
    d.total_tiles = tiles;
    if (tiles == 0) continue;
    matcov_block_kernel<OutT><<<tiles, dim3(kTileI, kTileJ), 0, s>>>(d, g, data);
    if (launches) ++*launches;
    MOAO_CUDA_TRY(cudaGetLastError());
  }
  return MOAO_OK;
}

// Ordered WFS pairs that get an offset table: Cmm pairs (m >= n) and the truth
// sensor against each WFS, in both orders, when their projections match.
void table_pairs(const DevGeometry& g, int2* pairs, int* npairs) {
  *npairs = 0;
  const int ts = g.nW - 1;
  auto same = [&](int m, int n) {
    return g.gsAlt[m] == g.gsAlt[n] && g.G[m] == g.G[n] && g.cth[m] == g.cth[n] &&
           g.sth[m] == g.sth[n] && g.Nssp[m] == g.nssp_grid && g.Nssp[n] == g.nssp_grid &&
           g.Nsubap[m] == g.Nsubap[0] && g.Nsubap[n] == g.Nsubap[0];
  };
  for (int m = 0; m < g.nW; ++m)
    for (int n = 0; n < g.nW; ++n) {
      const bool needed = (m < ts && n < ts && m >= n) || (m == ts && n < ts) || (n == ts && m < ts);
      if (needed && same(m, n)) pairs[(*npairs)++] = make_int2(m, n);
    }
}

}  // namespace

long toeplitz_table_doubles(const DevGeometry& g, int* npairs) {
  int2 pairs[kMaxWfs * kMaxWfs];
  table_pairs(g, pairs, npairs);
  const long W = 2L * g.nssp_grid - 1;
  return (long)*npairs * W * W * 4;
}

moao_status build_toeplitz_tables(DevGeometry& g, cudaStream_t s, long long* launches) {
  int2 pairs[kMaxWfs * kMaxWfs];
  int np = 0;
  table_pairs(g, pairs, &np);
  for (int m = 0; m < kMaxWfs; ++m)
    for (int n = 0; n < kMaxWfs; ++n) g.tpair[m][n] = -1;
  if (np == 0 || !g.ttab) {
    g.ttab = nullptr;
    return MOAO_OK;
  }
  for (int k = 0; k < np; ++k) g.tpair[pairs[k].x][pairs[k].y] = k;
  // the pair list travels in the table's tail (4 doubles per offset before it)
  const long W = 2L * g.nssp_grid - 1;
  int2* d_pairs = reinterpret_cast<int2*>(g.ttab + (long)np * W * W * 4);
  MOAO_CUDA_TRY(cudaMemcpyAsync(d_pairs, pairs, np * sizeof(int2), cudaMemcpyHostToDevice, s));
  const long total = (long)np * W * W;
  const unsigned blocks = (unsigned)std::min<long>((total + 127) / 128, 148L * 64);
  toeplitz_table_kernel<<<blocks, 128, 0, s>>>(g, d_pairs, np, g.ttab);
  if (launches) ++*launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status launch_matcov(const DevGeometry& g, double* data, int nrows, int ncols,
                          int xoffset, int yoffset, int lda, int type_mat, cudaStream_t s,
                          long long* launches) {
  return launch_impl<double>(g, data, nrows, ncols, xoffset, yoffset, lda, type_mat, s,
                             launches);
}

moao_status launch_matcov_f32(const DevGeometry& g, float* data, int nrows, int ncols,
                              int xoffset, int yoffset, int lda, int type_mat, cudaStream_t s,
                              long long* launches) {
  return launch_impl<float>(g, data, nrows, ncols, xoffset, yoffset, lda, type_mat, s,
                            launches);
}

}  // namespace moao
