/*
 * TEST INFRASTRUCTURE — CPU oracle of the covariance generation (see
 * moao_oracle.h). Restates, element by element and in the reference's order of
 * operations, the von Karman slope-covariance model:
 *
 *   series_f        macdo_x56     common/kernels/matcov_kernels.cpp:38-62
 *   asymptotic_f    asymp_macdo   common/kernels/matcov_kernels.cpp:65-89
 *   dphi_r          rodconan      common/kernels/matcov_kernels.cpp:92-116
 *   oracle_dphi     DPHI_gb       common/kernels/matcov_kernels.cpp:135-140
 *   cov_*           cov_XX/YY/XY/YX_gb  common/kernels/matcov_kernels.cpp:147-193
 *   element         compute_element_tiled_4  :206-333 (noise :310-330)
 *   element_ts      compute_element_ts_tile  :423-483
 *   tile driver     MOAO_COMMON::matcov_tile common/compute/matcov.cpp:17-99
 *                   + matcov_kernel_4 uplo handling :355-400
 *
 * Model constants are the published ones of common/moao_defs.h:15-38.
 */
#include "moao_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>

static const double GA[11] = {0, 12.067619015983075, 5.17183672113560444, 0.795667187867016068,
                              0.0628158306210802181, 0.00301515986981185091,
                              9.72632216068338833e-05, 2.25320204494595251e-06,
                              3.93000356676612095e-08, 5.34694362825451923e-10,
                              5.83302941264329804e-12};
static const double GMA[11] = {-3.74878707653729304, -2.04479295083852408,
                               -0.360845814853857083, -0.0313778969438136685,
                               -0.001622994669507603, -5.56455315259749673e-05,
                               -1.35720808599938951e-06, -2.47515152461894642e-08,
                               -3.50257291219662472e-10, -3.95770950530691961e-12,
                               -3.65327031259100284e-14};
static const double PI_ = 3.1415926535897932384626433;
static const double K1 = 0.1716613621245709486;
static const double K2 = 1.00563491799858928388289314170833;
static const double K3 = 1.25331413731550012081;
static const double A1 = 0.22222222222222222222;
static const double A2 = -0.08641975308641974829;
static const double A3 = 0.08001828989483310284;
#define XLIM (0.75 * 2 * PI_)
#define LAMBDA2 0.00026942094446267851

/* x^(5/6) K_5/6(x) series without its constant term, accumulated upward in n. */
static double series_f(double x) {
  const double x2a = pow(x, 2.0 * (5. / 6.));
  const double x22 = x * x / 4.;
  double x2n = 0.5;
  double s = GMA[0] * x2a * x2n;
  x2n *= x22;
  for (int n = 1; n <= 10; ++n) {
    s += (GMA[n] * x2a + GA[n]) * x2n;
    x2n *= x22;
  }
  return s;
}

static double asymptotic_f(double x) {
  const double xi = 1. / x;
  return K2 - K3 * exp(-x) * pow(x, 1 / 3.) * (1.0 + xi * (A1 + xi * (A2 + xi * A3)));
}

static double dphi_r(double r, double L0) {
  const double x = (2 * PI_ / L0) * r;
  double f = (x > XLIM) ? asymptotic_f(x) : -series_f(x);
  return f * (K1 * pow(L0, 5. / 3.0));
}

double oracle_dphi(double x, double y, double L0) { return dphi_r(sqrt(x * x + y * y), L0); }

static double cov_xx(double du, double dv, double ac, double ad, double bc, double bd, double L0) {
  return -oracle_dphi(du + ac, dv, L0) + oracle_dphi(du + ad, dv, L0) +
         oracle_dphi(du + bc, dv, L0) - oracle_dphi(du + bd, dv, L0);
}
static double cov_yy(double du, double dv, double ac, double ad, double bc, double bd, double L0) {
  return -oracle_dphi(du, dv + ac, L0) + oracle_dphi(du, dv + ad, L0) +
         oracle_dphi(du, dv + bc, L0) - oracle_dphi(du, dv + bd, L0);
}
static double cov_xy(double du, double dv, double s1, double s2, double L0) {
  return -oracle_dphi(du + s1, dv - s2, L0) + oracle_dphi(du + s1, dv + s2, L0) +
         oracle_dphi(du - s1, dv - s2, L0) - oracle_dphi(du - s1, dv + s2, L0);
}
static double cov_yx(double du, double dv, double s1, double s2, double L0) {
  return -oracle_dphi(du - s2, dv + s1, L0) + oracle_dphi(du + s2, dv + s1, L0) +
         oracle_dphi(du - s2, dv - s1, L0) - oracle_dphi(du + s2, dv - s1, L0);
}

/* Slope index -> (WFS, subaperture, x/y); base = first slope of that WFS. */
static void decode(long pos, const oracle_geom* g, int* w, long* sub, int* xy, long* off) {
  long first = 0, o = 0;
  int k = 0;
  while (k < g->nW - 1 && pos >= first + 2 * g->Nsubap[k]) {
    first += 2 * g->Nsubap[k];
    o += g->Nsubap[k];
    ++k;
  }
  long i = pos - first;
  *xy = (i >= g->Nsubap[k]) ? 1 : 0;
  if (*xy) i -= g->Nsubap[k];
  *w = k;
  *sub = i;
  *off = o;
}

/* Element (row, col) of Cmm (type 1) or Ctm (type 3, row in the truth sensor). */
static double element(long row, long col, const oracle_geom* g, int type_mat) {
  int m, n, xyi, xyj;
  long i, j, offm, offn;
  if (type_mat == 3) {
    m = g->nW - 1;
    offm = 0;
    for (int w = 0; w < m; ++w) offm += g->Nsubap[w];
    i = row;
    xyi = (i >= g->Nsubap[m]) ? 1 : 0;
    if (xyi) i -= g->Nsubap[m];
  } else {
    decode(row, g, &m, &i, &xyi, &offm);
  }
  decode(col, g, &n, &j, &xyj, &offn);
  const double sm = g->diam / g->Nssp[m], sn = g->diam / g->Nssp[n];
  const double kk = LAMBDA2 / (sm * sn);
  const int type = xyi * 2 + xyj;
  double c = 0.0;
  for (int l = 0; l < g->nLayer; ++l) {
    const double sml = g->sspSizeL[m * g->nLayer + l], snl = g->sspSizeL[n * g->nLayer + l];
    if (!(sml > 0 && snl > 0)) continue;
    const long p1 = i + offm + (long)l * g->Nx, p2 = j + offn + (long)l * g->Nx;
    const double du = g->u[p1] - g->u[p2], dv = g->v[p1] - g->v[p2];
    const double s1 = sml * 0.5, s2 = snl * 0.5;
    const double ac = s1 - s2, ad = s1 + s2, bc = -ad, bd = -ac;
    double cv;
    if (type == 0) cv = cov_xx(du, dv, ac, ad, bc, bd, g->L0[l]);
    else if (type == 3) cv = cov_yy(du, dv, ac, ad, bc, bd, g->L0[l]);
    else if (type == 1) cv = cov_xy(du, dv, s1, s2, g->L0[l]);
    else cv = cov_yx(du, dv, s1, s2, g->L0[l]);
    c += 0.5 * cv * kk * g->cn2[l];
  }
  if (m == n) {
    if (m < g->nLgs) {
      if (i == j) {
        const long p = i + offm;
        c += (type == 0) ? g->noiseLGSxx[p] : (type == 3) ? g->noiseLGSyy[p] : g->noiseLGSxy[p];
      }
      if (type == 0 || type == 3) c += g->lgsCst;
    } else if (i == j && (type == 0 || type == 3)) {
      c += g->noiseNGS[m - g->nLgs];
    }
  }
  return c;
}

/* Ctt element from the unprojected truth-sensor positions; the truth sensor is
 * indexed at Nsubap_ts * (nW - 1) exactly as the reference does. */
static double element_ts(long row, long col, const oracle_geom* g) {
  const int ts = g->nW - 1;
  const long N = g->Nsubap[ts];
  const long i = row < N ? row : row - N, j = col < N ? col : col - N;
  const int type = (row < N ? 0 : 2) + (col < N ? 0 : 1);
  const double ssp = g->diam / g->Nssp[ts];
  const double kk = LAMBDA2 / (ssp * ssp);
  const double s = ssp * 0.5;
  const double ac = 0.0, ad = 2.0 * s, bc = -ad, bd = 0.0;
  const double du = g->X[N * ts + i] - g->X[N * ts + j];
  const double dv = g->Y[N * ts + i] - g->Y[N * ts + j];
  double c = 0.0;
  for (int l = 0; l < g->nLayer; ++l) {
    double cv;
    if (type == 0) cv = cov_xx(du, dv, ac, ad, bc, bd, g->L0[l]);
    else if (type == 3) cv = cov_yy(du, dv, ac, ad, bc, bd, g->L0[l]);
    else if (type == 1) cv = cov_xy(du, dv, s, s, g->L0[l]);
    else cv = cov_yx(du, dv, s, s, g->L0[l]);
    c += 0.5 * cv * kk * g->cn2[l];
  }
  return c;
}

int oracle_matcov_tile(double* data, int nrows, int ncols, int xoffset, int yoffset, int lda,
                       const oracle_geom* g, int type_mat) {
  if (type_mat != 1 && type_mat != 3 && type_mat != 4) return 1;
  for (long ly = 0; ly < ncols; ++ly) {
    for (long lx = 0; lx < nrows; ++lx) {
      const long gx = lx + xoffset, gy = ly + yoffset;
      if (type_mat == 1 && gy > gx) continue; /* uplo = 'l' */
      data[ly * lda + lx] = (type_mat == 4) ? element_ts(gx, gy, g) : element(gx, gy, g, type_mat);
    }
  }
  return 0;
}

typedef struct {
  double* data;
  int r0, r1, ncols, xoffset, yoffset, lda, type_mat;
  const oracle_geom* g;
} band_t;

static void* band_main(void* arg) {
  band_t* b = (band_t*)arg;
  oracle_matcov_tile(b->data + b->r0, b->r1 - b->r0, b->ncols, b->xoffset + b->r0, b->yoffset,
                     b->lda, b->g, b->type_mat);
  return NULL;
}

int oracle_matcov_tile_mt(double* data, int nrows, int ncols, int xoffset, int yoffset, int lda,
                          const oracle_geom* g, int type_mat, int nthreads) {
  if (type_mat != 1 && type_mat != 3 && type_mat != 4) return 1;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  pthread_t th[256];
  band_t bands[256];
  /* Rows split so that lower-triangle work is balanced. */
  int prev = 0;
  for (int t = 0; t < nthreads; ++t) {
    int r1 = (int)((double)nrows * sqrt((double)(t + 1) / nthreads));
    if (type_mat != 1) r1 = (int)((long)nrows * (t + 1) / nthreads);
    if (t == nthreads - 1) r1 = nrows;
    bands[t] = (band_t){data, prev, r1, ncols, xoffset, yoffset, lda, type_mat, g};
    prev = r1;
  }
  for (int t = 1; t < nthreads; ++t) pthread_create(&th[t], NULL, band_main, &bands[t]);
  band_main(&bands[0]);
  for (int t = 1; t < nthreads; ++t) pthread_join(th[t], NULL);
  return 0;
}
