/*
 * TEST INFRASTRUCTURE — the CPU oracle of the covariance generation.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it, and only as the checker. The product library never links it.
 *
 * A plain-C restatement, one element at a time, of the reference's
 * covariance model (common/kernels/matcov_kernels.cpp) driven by the geometry
 * tables of a system (u, v, sspSizeL, L0, cn2, noise, ...).
 */
#ifndef MOAO_ORACLE_H
#define MOAO_ORACLE_H

typedef struct {
  int nW, nLgs, nLayer, Nx;
  const long* Nsubap;      /* [nW] */
  const long* Nssp;        /* [nW] */
  const double* u;         /* [nLayer*Nx] */
  const double* v;         /* [nLayer*Nx] */
  const double* sspSizeL;  /* [nW*nLayer] */
  const double* L0;        /* [nLayer] */
  const double* cn2;       /* [nLayer] */
  const double* X;         /* [Nx] */
  const double* Y;         /* [Nx] */
  const double* noiseNGS;  /* [nW-nLgs] */
  const double* noiseLGSxx;
  const double* noiseLGSyy;
  const double* noiseLGSxy;
  double lgsCst, diam;
} oracle_geom;

/* Same contract as MOAO_COMMON::matcov_tile (common/compute/matcov.cpp:17):
 * type 1 Cmm (lower only), 3 Ctm, 4 Ctt; returns nonzero on a bad type. */
int oracle_matcov_tile(double* data, int nrows, int ncols, int xoffset, int yoffset, int lda,
                       const oracle_geom* g, int type_mat);
/* The same over nthreads POSIX threads (rows split into contiguous bands). */
int oracle_matcov_tile_mt(double* data, int nrows, int ncols, int xoffset, int yoffset, int lda,
                          const oracle_geom* g, int type_mat, int nthreads);
/* DPHI for one separation, exposed for the model's sanity tests. */
double oracle_dphi(double x, double y, double L0);

#endif
