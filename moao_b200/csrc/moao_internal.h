// Internal declarations shared by the host library and the CUDA kernels.
#ifndef MOAO_INTERNAL_H
#define MOAO_INTERNAL_H

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>

#include "moao_b200.h"

namespace moao {

// Records a message for moao_last_error() and returns the status.
moao_status set_error(moao_status s, const std::string& msg);

#define MOAO_CUDA_TRY(expr)                                                        \
  do {                                                                             \
    cudaError_t _e = (expr);                                                       \
    if (_e != cudaSuccess)                                                         \
      return ::moao::set_error(MOAO_ERR_CUDA, std::string(#expr) + ": " +          \
                                                  cudaGetErrorString(_e));         \
  } while (0)

#define MOAO_TRY(expr)                 \
  do {                                 \
    moao_status _s = (expr);           \
    if (_s != MOAO_OK) return _s;      \
  } while (0)

// Raises a kernel's dynamic shared-memory limit once per device (the attribute
// belongs to the current device's copy of the kernel; devices past 63 set it on
// every call).
template <typename Kernel>
cudaError_t set_smem_limit(Kernel kern, int bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (bit && (done.load() & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done.fetch_or(bit);
  return e;
}

// ---------------------------------------------------------------------------
// Geometry tables resident on the device (uploaded from a Tomo_struct).
// ---------------------------------------------------------------------------
constexpr int kMaxWfs = 16;
constexpr int kMaxLayers = 128;

struct DevGeometry {
  int nW = 0, nLgs = 0, nLayer = 0, Nx = 0;
  double diam = 0, lgsCst = 0;
  int Nsubap[kMaxWfs];       // valid subapertures per WFS
  int off[kMaxWfs];          // first subaperture of each WFS in the Nx tables
  int Nssp[kMaxWfs];
  // device arrays
  double* u = nullptr;       // [nLayer*Nx]
  double* v = nullptr;       // [nLayer*Nx]
  double* X = nullptr;       // [Nx]
  double* Y = nullptr;       // [Nx]
  double* noiseLGSxx = nullptr;  // [Nx]
  double* noiseLGSyy = nullptr;
  double* noiseLGSxy = nullptr;
  double* noiseNGS = nullptr;    // [nW - nLgs]
  // per-layer tables: [0,nL) 2*pi/L0, [nL,2nL) k1*L0^(5/3), [2nL,3nL) cn2,
  // [3nL, 3nL + nW*nL) sspSizeL, then h [nL]
  double* layer = nullptr;

  // Projection of each WFS onto a layer at altitude h (projectedSubap):
  //   u = (G (X cos - Y sin) + XPup) (1 - h gsAlt) + alphaX h
  //   v = (G (X sin + Y cos) + YPup) (1 - h gsAlt) + alphaY h
  double gsAlt[kMaxWfs], G[kMaxWfs], cth[kMaxWfs], sth[kMaxWfs];
  double XPup[kMaxWfs], YPup[kMaxWfs], alphaX[kMaxWfs], alphaY[kMaxWfs];
  // Subaperture grid: pitch and the (column, row) of every valid subaperture
  // of a WFS (all WFS share one grid when their Nssp are equal).
  double pitch = 0;
  int nssp_grid = 0;
  int* grid_cr = nullptr;    // [2 * Nsubap of WFS 0]: column, row
  // Offset tables of the equal-projection WFS pairs (see matcov.cu), or null.
  double* ttab = nullptr;
  int tpair[kMaxWfs][kMaxWfs];  // table index of the pair (m, n), or -1
  // Edge-aligned WFS (unrotated, unit magnification, the common grid): on every
  // layer the projected subaperture edges are the midlines between neighbouring
  // centres, so neighbouring subapertures share stencil points (matcov.cu).
  int aligned[kMaxWfs];
  double bornemin = 0;          // pupil coordinate of the grid's first edge
  int* cell_idx = nullptr;      // [nssp_grid^2]: valid index of grid cell (row * N + col), or -1
  int* tiles_a = nullptr;       // 4x4-cell tiles holding a valid cell: (col0, row0) pairs
  int* tiles_b = nullptr;       // 8x8-cell tiles likewise
  int ntiles_a = 0, ntiles_b = 0;
};

// Builds the offset tables of g's equal-projection WFS pairs into g.ttab (device
// memory provided by the caller, toeplitz_table_doubles(g) doubles).
long toeplitz_table_doubles(const DevGeometry& g, int* npairs);
moao_status build_toeplitz_tables(DevGeometry& g, cudaStream_t s, long long* launches);

// Matcov launch (device pointers). type_mat: 1 Cmm lower, 3 Ctm, 4 Ctt,
// 5 Cmm full symmetric. The tile covers rows [xoffset, xoffset+nrows) and
// columns [yoffset, yoffset+ncols) of the global matrix; data points at the
// tile's first element.
moao_status launch_matcov(const DevGeometry& g, double* data, int nrows, int ncols,
                          int xoffset, int yoffset, int lda, int type_mat,
                          cudaStream_t s, long long* launches);
// FP32 output variant (mixed path); same geometry, FP64 evaluation.
moao_status launch_matcov_f32(const DevGeometry& g, float* data, int nrows, int ncols,
                              int xoffset, int yoffset, int lda, int type_mat,
                              cudaStream_t s, long long* launches);

}  // namespace moao

#endif  // MOAO_INTERNAL_H
