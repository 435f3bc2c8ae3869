// Intersample PSF: Cvv -> averaged covariance map -> phase structure function
// -> long-exposure PSF (common/tomo_struct/intersample.cpp:74-170).
//
// Device pipeline (N = 512 for every supported system), the reference's FFTW
// real-to-complex / complex-to-real steps done as full complex transforms
// (fft.cu) whose spectra are built Hermitian from the half spectrum the real
// transforms keep, so the results are those of the half-spectrum pipeline:
//   gather_place   Map cell c = sum of Cvv[i] over idx[i]-1 == c, in increasing i
//                  (the reference's sequential scatter order, so the sum is
//                  bit-identical), divided by its hit count, written straight
//                  onto the N x N lattice with pitch dactupix; other pixels 0.
//   forward FFT    N x N (real input)
//   filter         half spectrum (columns 0..N/2): re *= abs2fi[j*N+i]
//                  (transposed index, as in the reference), im = 0; the other
//                  columns the Hermitian mirror of it
//   inverse FFT    (its real part is the complex-to-real result)
//   to_dphi        exp(-0.5 (norm - dphi fact / fact2)) with the reference's
//                  truncated pi in fact, written through the quadrant swap
//                  (_eclat_double) so no separate shift pass runs
//   otf            half spectrum re = otf_tel[j*N+i] * dphi[j*N+i], im = 0,
//                  mirrored the same way
//   inverse FFT, then a final quadrant swap of its real part into the output.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "context.h"
#include "fft.h"

struct moao_isample {
  moao_ctx* ctx = nullptr;
  moao_isample_info info{};
  long nmap = 0, ncov = 0;
  // device
  double* abs2fi = nullptr;   // N*N
  double* otf = nullptr;      // N*N
  int* cell_start = nullptr;  // nmap+1 (CSR over Cvv indices)
  int* cell_idx = nullptr;    // nidx
  double* inv_div = nullptr;  // nmap (1/div, or 1 when div == 0)
  double* div = nullptr;      // nmap
  double* dphi = nullptr;     // N*N real
  moao::Cplx* spec = nullptr;   // N*N: the map, then spectra
  moao::Cplx* spec2 = nullptr;  // N*N
  double* in_host_cvv = nullptr;
  moao::Fft2d fft;
  double fact = 0, fact2 = 0;
  long idx_norm = 0;
};

namespace moao {
namespace {

__global__ void gather_place_kernel(const double* __restrict__ cvv, const int* __restrict__ start,
                                    const int* __restrict__ cidx, const double* __restrict__ div,
                                    Cplx* __restrict__ map, long N, long ncov, long a,
                                    long pitch) {
  const long total = N * N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    // map[j + i*N]: i is the slow index
    const long i = e / N, j = e % N;
    double v = 0.0;
    const long di = i - a, dj = j - a;
    if (di >= 0 && dj >= 0 && di % pitch == 0 && dj % pitch == 0) {
      const long ii = di / pitch, jj = dj / pitch;
      if (ii < ncov && jj < ncov) {
        const long c = ii * ncov + jj;
        double s = 0.0;
        for (int k = start[c]; k < start[c + 1]; ++k) s += cvv[cidx[k]];
        if (div[c] > 0) s /= div[c];
        v = s;
      }
    }
    map[e] = {v, 0.0};
  }
}

// Element (i, j) of the full spectrum whose half j <= N/2 is the real value
// f(i, j) and whose other columns mirror it, f((N - i) mod N, N - j): what a
// complex-to-real transform reads from a half spectrum.
template <class F>
__device__ __forceinline__ double hermitian_real(long i, long j, long N, F f) {
  return j <= N / 2 ? f(i, j) : f((N - i) % N, N - j);
}

// out = re(spec) * abs2fi[j*N+i] on the half spectrum (transposed index), im 0
__global__ void filter_kernel(const Cplx* __restrict__ spec, const double* __restrict__ abs2fi,
                              Cplx* __restrict__ out, long N) {
  const long total = N * N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e / N, j = e % N;
    const double v = hermitian_real(i, j, N, [&](long a, long b) {
      return spec[a * N + b].x * abs2fi[b * N + a];
    });
    out[e] = {v, 0.0};
  }
}

// dst[swap(e)] = exp(-0.5 * (norm - re(src[e]) / fact2 * fact))
__global__ void to_dphi_kernel(const Cplx* __restrict__ src, double* __restrict__ dst, long N,
                               long idx_norm, double fact, double fact2) {
  const double norm = src[idx_norm].x / fact2 * fact;
  const long total = N * N, h = N / 2;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long x = e % N, y = e / N;
    const long d = ((x + h) % N) + ((y + h) % N) * N;
    dst[d] = exp(-0.5 * (norm - src[e].x / fact2 * fact));
  }
}

// spec = otf[j*N+i] * dphi[j*N+i] on the half spectrum, im 0
__global__ void otf_kernel(Cplx* __restrict__ spec, const double* __restrict__ otf,
                           const double* __restrict__ dphi, long N) {
  const long total = N * N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e / N, j = e % N;
    const double v = hermitian_real(i, j, N, [&](long a, long b) {
      return otf[b * N + a] * dphi[b * N + a];
    });
    spec[e] = {v, 0.0};
  }
}

__global__ void swap_quadrants_kernel(const Cplx* __restrict__ src, double* __restrict__ dst,
                                      long N) {
  const long total = N * N, h = N / 2;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long x = e % N, y = e / N;
    dst[((x + h) % N) + ((y + h) % N) * N] = src[e].x;
  }
}

unsigned grid_for(long total) {
  return (unsigned)std::max(1L, std::min((total + 255) / 256, 148L * 8));
}

void free_isample(moao_isample* is) {
  if (!is) return;
  fft2d_free(&is->fft);
  void* ptrs[] = {is->abs2fi, is->otf, is->cell_start, is->cell_idx, is->inv_div,
                  is->div, is->dphi, is->spec, is->spec2};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  delete is;
}

}  // namespace
}  // namespace moao

using namespace moao;

extern "C" {

moao_status moao_intersample_create(moao_ctx* ctx, long nidx, long np, double Dtel,
                                    const long* idx, const double* abs2fi, const double* otf_tel,
                                    moao_isample** out) {
  (void)Dtel;
  if (!ctx || !idx || !abs2fi || !otf_tel || !out || nidx <= 0 || np < 2)
    return set_error(MOAO_ERR_BAD_ARG, "intersample_create: bad arguments");
  if (nidx > 0x7fffffffL) return set_error(MOAO_ERR_UNSUPPORTED, "intersample: nidx too large");
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  moao_isample* is = new moao_isample;
  is->ctx = ctx;
  // intersample_prepare (intersample.cpp:176-207)
  const long N = std::max(512L, (long)(8 * std::pow(2, (long)(std::log((double)np) + 0.5))));
  is->info.N = N;
  is->info.np = np;
  is->info.nidx = nidx;
  is->info.lambda = 1.65e-06;
  is->info.dactupix = (double)(N / (3 * (np - 1)) + 1);
  is->ncov = 2 * np - 1;
  is->nmap = is->ncov * is->ncov;
  // Hit counts and the CSR gather lists; indices are validated here instead of
  // being written out of bounds.
  std::vector<int> count(is->nmap + 1, 0);
  for (long i = 0; i < nidx; ++i) {
    const long c = idx[i] - 1;
    if (c < 0 || c >= is->nmap) {
      delete is;
      return set_error(MOAO_ERR_BAD_ARG, "intersample_create: idx[" + std::to_string(i) +
                                             "] outside the covariance map");
    }
    ++count[c + 1];
  }
  std::vector<double> div(is->nmap);
  for (long c = 0; c < is->nmap; ++c) div[c] = (double)count[c + 1];
  for (long c = 0; c < is->nmap; ++c) count[c + 1] += count[c];
  std::vector<int> cidx(nidx), fill(count.begin(), count.end() - 1);
  for (long i = 0; i < nidx; ++i) cidx[fill[idx[i] - 1]++] = (int)i;

  const double dp = is->info.dactupix;
  is->fact = 2 * std::pow(2 * 3.14159 / is->info.lambda, 2);
  is->fact2 = N * N * dp * dp;
  const long ncmap = N / 2 + 1;
  is->idx_norm = N * (ncmap - 1) + ncmap - 1;

  const size_t NN = (size_t)N * N;
  moao_status st = MOAO_OK;
  auto alloc = [&](void** p, size_t bytes) {
    if (st == MOAO_OK && cudaMalloc(p, bytes) != cudaSuccess)
      st = set_error(MOAO_ERR_OOM, "intersample_create: device allocation");
  };
  alloc((void**)&is->abs2fi, NN * 8);
  alloc((void**)&is->otf, NN * 8);
  alloc((void**)&is->cell_start, (is->nmap + 1) * sizeof(int));
  alloc((void**)&is->cell_idx, nidx * sizeof(int));
  alloc((void**)&is->div, is->nmap * 8);
  alloc((void**)&is->dphi, NN * 8);
  alloc((void**)&is->spec, NN * sizeof(Cplx));
  alloc((void**)&is->spec2, NN * sizeof(Cplx));
  if (st == MOAO_OK) {
    cudaMemcpy(is->abs2fi, abs2fi, NN * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(is->otf, otf_tel, NN * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(is->cell_start, count.data(), (is->nmap + 1) * sizeof(int), cudaMemcpyHostToDevice);
    cudaMemcpy(is->cell_idx, cidx.data(), nidx * sizeof(int), cudaMemcpyHostToDevice);
    if (cudaMemcpy(is->div, div.data(), is->nmap * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      st = set_error(MOAO_ERR_CUDA, "intersample_create: upload");
  }
  if (st == MOAO_OK) st = fft2d_plan(&is->fft, N);
  if (st != MOAO_OK) {
    free_isample(is);
    return st;
  }
  *out = is;
  return MOAO_OK;
}

moao_status moao_intersample_get_info(const moao_isample* is, moao_isample_info* out) {
  if (!is || !out) return set_error(MOAO_ERR_BAD_ARG, "intersample_get_info: null");
  *out = is->info;
  return MOAO_OK;
}

moao_status moao_intersample_process(moao_isample* is, const double* d_Cvv, double* d_psf) {
  if (!is || !d_Cvv || !d_psf) return set_error(MOAO_ERR_BAD_ARG, "intersample_process: null");
  moao_ctx* ctx = is->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const long N = is->info.N, NN = N * N;
  const long ncmap = N / 2 + 1, nelem = (is->ncov - 1) / 2;
  const long pitch = (long)is->info.dactupix;
  const long a = ncmap - nelem * pitch - 1;
  if (a < 0) return set_error(MOAO_ERR_BAD_ARG, "intersample: map does not fit the FFT support");
  gather_place_kernel<<<grid_for(NN), 256, 0, s>>>(d_Cvv, is->cell_start, is->cell_idx, is->div,
                                                    is->spec, N, is->ncov, a, pitch);
  MOAO_TRY(fft2d(is->fft, is->spec, -1, s, &ctx->launches));
  filter_kernel<<<grid_for(NN), 256, 0, s>>>(is->spec, is->abs2fi, is->spec2, N);
  MOAO_TRY(fft2d(is->fft, is->spec2, +1, s, &ctx->launches));
  to_dphi_kernel<<<grid_for(NN), 256, 0, s>>>(is->spec2, is->dphi, N, is->idx_norm, is->fact,
                                               is->fact2);
  otf_kernel<<<grid_for(NN), 256, 0, s>>>(is->spec, is->otf, is->dphi, N);
  MOAO_TRY(fft2d(is->fft, is->spec, +1, s, &ctx->launches));
  swap_quadrants_kernel<<<grid_for(NN), 256, 0, s>>>(is->spec, d_psf, N);
  ctx->launches += 5;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status moao_intersample_process_host(moao_isample* is, const double* Cvv, double* psf) {
  if (!is || !Cvv || !psf) return set_error(MOAO_ERR_BAD_ARG, "intersample_process_host: null");
  moao_ctx* ctx = is->ctx;
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  const long N = is->info.N;
  double *dc = nullptr, *dp = nullptr;
  if (cudaMalloc(&dc, is->info.nidx * 8) != cudaSuccess)
    return set_error(MOAO_ERR_OOM, "intersample_process_host: Cvv");
  if (cudaMalloc(&dp, N * N * 8) != cudaSuccess) {
    cudaFree(dc);
    return set_error(MOAO_ERR_OOM, "intersample_process_host: psf");
  }
  moao_status st = MOAO_OK;
  if (cudaMemcpyAsync(dc, Cvv, is->info.nidx * 8, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
    st = set_error(MOAO_ERR_CUDA, "intersample_process_host: H2D");
  if (st == MOAO_OK) st = moao_intersample_process(is, dc, dp);
  if (st == MOAO_OK &&
      cudaMemcpyAsync(psf, dp, N * N * 8, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess)
    st = set_error(MOAO_ERR_CUDA, "intersample_process_host: D2H");
  cudaStreamSynchronize(ctx->stream);
  cudaFree(dc);
  cudaFree(dp);
  return st;
}

void moao_intersample_destroy(moao_isample* is) {
  if (!is) return;
  cudaSetDevice(is->ctx->device);
  cudaStreamSynchronize(is->ctx->stream);
  free_isample(is);
}

}  // extern "C"
