// 2-D complex FFT (FP64) as row transforms, a transpose, row transforms and a
// transpose back. A row transform is one CTA of N/2 threads: the row is read
// into shared memory in bit-reversed order, then log2(N) radix-2
// decimation-in-time stages run with one butterfly per thread and a barrier
// between stages (Cooley-Tukey). Twiddles come from a table computed on the
// host in long double, so every factor is the correctly rounded double of
// exp(-2 pi i k / N). The transposes move 32 x 32 tiles through shared memory
// so that reads and writes are both coalesced.
#include "fft.h"

#include <cmath>
#include <vector>

namespace moao {
namespace {

__device__ __forceinline__ unsigned bitrev(unsigned v, int bits) { return __brev(v) >> (32 - bits); }

__global__ void fft_rows_kernel(Cplx* __restrict__ data, int N, int logN,
                                const Cplx* __restrict__ tw, int dir) {
  extern __shared__ Cplx row[];
  Cplx* g = data + (long)blockIdx.x * N;
  for (int c = threadIdx.x; c < N; c += blockDim.x) row[bitrev((unsigned)c, logN)] = g[c];
  __syncthreads();
  const int t = threadIdx.x;  // one butterfly per thread and stage (N / 2 threads)
  for (int s = 0; s < logN; ++s) {
    const int half = 1 << s;
    const int pos = t & (half - 1);
    const int i0 = ((t >> s) << (s + 1)) + pos, i1 = i0 + half;
    Cplx w = tw[pos << (logN - 1 - s)];
    if (dir > 0) w.y = -w.y;
    const Cplx u = row[i0], v = row[i1];
    const Cplx vw = {v.x * w.x - v.y * w.y, v.x * w.y + v.y * w.x};
    row[i0] = {u.x + vw.x, u.y + vw.y};
    row[i1] = {u.x - vw.x, u.y - vw.y};
    __syncthreads();
  }
  for (int c = threadIdx.x; c < N; c += blockDim.x) g[c] = row[c];
}

// dst[c * N + r] = src[r * N + c]
__global__ void transpose_kernel(const Cplx* __restrict__ src, Cplx* __restrict__ dst, int N) {
  __shared__ Cplx tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = by + k, c = bx + threadIdx.x;
    if (r < N && c < N) tile[k][threadIdx.x] = src[(long)r * N + c];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int c = bx + k, r = by + threadIdx.x;
    if (r < N && c < N) dst[(long)c * N + r] = tile[threadIdx.x][k];
  }
}

}  // namespace

moao_status fft2d_plan(Fft2d* f, long N) {
  int logN = 0;
  while ((1L << logN) < N) ++logN;
  if (N < 2 || N > 2048 || (1L << logN) != N)
    return set_error(MOAO_ERR_UNSUPPORTED, "fft2d: N must be a power of two in [2, 2048]");
  std::vector<Cplx> tw(N / 2);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (long k = 0; k < N / 2; ++k) {
    const long double a = -2.0L * pi * (long double)k / (long double)N;
    tw[k] = {(double)std::cos(a), (double)std::sin(a)};
  }
  f->N = N;
  f->logN = logN;
  if (cudaMalloc(&f->tw, sizeof(Cplx) * (N / 2)) != cudaSuccess ||
      cudaMalloc(&f->tmp, sizeof(Cplx) * N * N) != cudaSuccess) {
    fft2d_free(f);
    return set_error(MOAO_ERR_OOM, "fft2d: device buffers");
  }
  MOAO_CUDA_TRY(cudaMemcpy(f->tw, tw.data(), sizeof(Cplx) * (N / 2), cudaMemcpyHostToDevice));
  return MOAO_OK;
}

void fft2d_free(Fft2d* f) {
  if (f->tw) cudaFree(f->tw);
  if (f->tmp) cudaFree(f->tmp);
  f->tw = f->tmp = nullptr;
  f->N = 0;
}

moao_status fft2d(const Fft2d& f, Cplx* data, int dir, cudaStream_t s, long long* launches) {
  const int N = (int)f.N;
  if (N < 2 || !f.tw || !f.tmp) return set_error(MOAO_ERR_BAD_ARG, "fft2d: no plan");
  const size_t smem = sizeof(Cplx) * N;
  const dim3 tgrid((N + 31) / 32, (N + 31) / 32), tblock(32, 8);
  fft_rows_kernel<<<N, N / 2, smem, s>>>(data, N, f.logN, f.tw, dir);
  transpose_kernel<<<tgrid, tblock, 0, s>>>(data, f.tmp, N);
  fft_rows_kernel<<<N, N / 2, smem, s>>>(f.tmp, N, f.logN, f.tw, dir);
  transpose_kernel<<<tgrid, tblock, 0, s>>>(f.tmp, data, N);
  if (launches) *launches += 4;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

}  // namespace moao
