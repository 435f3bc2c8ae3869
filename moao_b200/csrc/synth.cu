// Synthesis of the intersample inputs without the reference's Python tooling.
//
// The reference reads idx.fits, abs2fi.fits and otftel.fits, written by its
// Python pipeline; the formulas restated here:
//   DM actuators     cython/pipeline/commande.py:57-79 (makeDM): the
//                    (nssp+1)^2 grid on [-1, 1]^2, actuators with
//                    obs - 1/nssp < r < 1 + 1.4/nssp, influence width
//                    x0 = sqrt(-2 / ln(coupling)) / nssp
//   idx              cython/pipeline/generate_file.py:57-76: the 1-based index
//                    of actuator pair (i, j) (column-major Cvv element
//                    i + j nact) in the (2 Np - 1)^2 covariance map,
//                    (xx_i - xx_j + Np) + (2 Np - 1)(yy_i - yy_j + Np - 1)
//   Fourier support  cython/pipeline/intersample.pyx:3-39: N, pixel ud
//   abs2fi           generate_file.py:79-86 with the influence function of
//                    commande.py:160-174: |FFT2 of 1e-6 exp(-(x^2 + y^2) / (2 x0^2))|^2
//   otf_tel          intersample.pyx:151-200: inverse FFT2 of |FFT2(pupil)|^2
//                    over the squared pupil area in pixels
// The DM geometry and idx are exact integer work on the host; abs2fi and the
// OTF are N^2 complex FFTs (fft.cu), like the tooling's numpy.fft.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "context.h"
#include "fft.h"

namespace moao {
namespace {

struct Dm {
  long np = 0;                  // actuators across (nssp + 1)
  std::vector<long> ix, iy;     // grid column / row of each actuator
  double x0 = 0;                // influence-function width (pupil radius units)
};

Dm make_dm(long nssp, double coupling, double obs) {
  Dm d;
  d.np = nssp + 1;
  for (long k = 0; k < d.np * d.np; ++k) {
    const long row = k / d.np, col = k % d.np;
    // linspace(-1, 1, np) as numpy computes it: i * (2 / (np - 1)) - 1, the
    // last point exactly 1
    const double step = 2.0 / (double)(d.np - 1);
    const double x = col == d.np - 1 ? 1.0 : col * step + -1.0;
    const double y = row == d.np - 1 ? 1.0 : row * step + -1.0;
    const double r = std::sqrt(x * x + y * y);
    if (r < 1.0 + 1.4 / nssp && r > obs - 1.0 / nssp) {
      d.ix.push_back(col);
      d.iy.push_back(row);
    }
  }
  d.x0 = std::sqrt(-2.0 / std::log(coupling)) / nssp;
  return d;
}

// N, pixel size ud of the Fourier support (intersample.pyx:3-39).
void fourier(long np, double dtel, long* N, double* ud) {
  const double dactu = dtel / (double)(np - 1);
  *N = std::max(8L * (1L << (long)(std::log2((double)np) + 0.5)), 512L);
  const double ud0 = 3.0 * dtel / (double)(*N);
  const long km = (long)(dactu / ud0 + 1);
  *ud = dactu / (double)km;
}

// Coordinate of pixel i of the support in pupil-radius units, in the two
// evaluation orders of the tooling: (k ud) / (dtel / 2) for the influence
// function, (ud / (dtel / 2)) k for the pupil.
__device__ __forceinline__ double coord_fi(long i, long N, double ud, double half) {
  return ((double)(i + 1 - (N / 2 + 1)) * ud) / half;
}
__device__ __forceinline__ double coord(long i, long N, double scale) {
  return scale * (double)(i + 1 - (N / 2 + 1));
}

__global__ void influence_kernel(Cplx* out, long N, double ud, double half,
                                 double x0) {
  const long total = N * N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e / N, j = e % N;
    const double x = coord_fi(j, N, ud, half), y = coord_fi(i, N, ud, half);
    out[e] = Cplx{1.e-6 * exp(-(x * x + y * y) / (2 * x0 * x0)), 0.0};
  }
}

__global__ void pupil_kernel(Cplx* out, long N, double scale, double obs) {
  const long total = N * N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e / N, j = e % N;
    const double xi = coord(i, N, scale), xj = coord(j, N, scale);
    const double r = sqrt(xj * xj + xi * xi);
    out[e] = Cplx{(r <= 1.0 && r > obs) ? 1.0 : 0.0, 0.0};
  }
}

// out[e] = |z[e]|^2 (real), or z[e] <- |z[e]|^2 + 0i
__global__ void abs2_kernel(Cplx* z, double* out, long total) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const double m = sqrt(z[e].x * z[e].x + z[e].y * z[e].y);  // |F|, then squared as b * b
    const double v = m * m;
    if (out) out[e] = v;
    else z[e] = Cplx{v, 0.0};
  }
}

// otf[i][j] = Re(z[j][i]) / N^2 / surface^2  (numpy's ifft2 normalisation, then .T)
__global__ void otf_out_kernel(const Cplx* z, double* out, long N, double scale) {
  const long total = N * N;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e / N, j = e % N;
    out[e] = z[j * N + i].x * scale;
  }
}

unsigned grid_of(long total) { return (unsigned)std::min<long>((total + 255) / 256, 148L * 16); }

}  // namespace
}  // namespace moao

using namespace moao;

extern "C" moao_status moao_intersample_inputs(moao_ctx* ctx, long nssp, double Dtel, double obs,
                                               double coupling, long* nact, long* N_out,
                                               long* idx, double* abs2fi, double* otf_tel) {
  if (nssp < 1 || !(Dtel > 0) || !(coupling > 0 && coupling < 1) || !(obs >= 0 && obs < 1))
    return set_error(MOAO_ERR_BAD_ARG, "intersample_inputs: nssp >= 1, Dtel > 0, 0 < coupling < 1");
  const Dm dm = make_dm(nssp, coupling, obs);
  const long na = (long)dm.ix.size(), np = dm.np;
  long N = 0;
  double ud = 0;
  fourier(np, Dtel, &N, &ud);
  if (nact) *nact = na;
  if (N_out) *N_out = N;
  if (idx) {
    for (long j = 0; j < na; ++j)
      for (long i = 0; i < na; ++i)
        idx[i + j * na] = (dm.ix[i] - dm.ix[j] + np) + (2 * np - 1) * (dm.iy[i] - dm.iy[j] + np - 1);
  }
  if (!abs2fi && !otf_tel) return MOAO_OK;
  if (!ctx) return set_error(MOAO_ERR_BAD_ARG, "intersample_inputs: the FFT tables need a context");
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  const long NN = N * N;
  const double scale = ud / (Dtel / 2.0);
  Cplx* z = nullptr;
  double* d = nullptr;
  if (cudaMalloc(&z, sizeof(Cplx) * NN) != cudaSuccess)
    return set_error(MOAO_ERR_OOM, "intersample_inputs: device buffer");
  if (cudaMalloc(&d, sizeof(double) * NN) != cudaSuccess) {
    cudaFree(z);
    return set_error(MOAO_ERR_OOM, "intersample_inputs: device buffer");
  }
  Fft2d plan;
  moao_status st = MOAO_OK;
  cudaStream_t s = ctx->stream;
  auto fft = [&](int dir) {
    if (st == MOAO_OK) st = fft2d(plan, z, dir, s, &ctx->launches);
  };
  st = fft2d_plan(&plan, N);
  if (st == MOAO_OK && abs2fi) {
    influence_kernel<<<grid_of(NN), 256, 0, s>>>(z, N, ud, Dtel / 2.0, dm.x0);
    fft(-1);
    abs2_kernel<<<grid_of(NN), 256, 0, s>>>(z, d, NN);
    if (st == MOAO_OK && cudaMemcpyAsync(abs2fi, d, sizeof(double) * NN, cudaMemcpyDeviceToHost,
                                         s) != cudaSuccess)
      st = set_error(MOAO_ERR_CUDA, "intersample_inputs: D2H");
    ctx->launches += 2;
  }
  if (st == MOAO_OK && otf_tel) {
    const double pi = 3.14159265358979323846;
    const double surface = Dtel * Dtel * (1 - obs * obs) * pi / 4. / (ud * ud);
    pupil_kernel<<<grid_of(NN), 256, 0, s>>>(z, N, scale, obs);
    fft(-1);
    abs2_kernel<<<grid_of(NN), 256, 0, s>>>(z, nullptr, NN);
    fft(+1);
    otf_out_kernel<<<grid_of(NN), 256, 0, s>>>(z, d, N, 1.0 / ((double)NN * surface * surface));
    if (st == MOAO_OK && cudaMemcpyAsync(otf_tel, d, sizeof(double) * NN, cudaMemcpyDeviceToHost,
                                         s) != cudaSuccess)
      st = set_error(MOAO_ERR_CUDA, "intersample_inputs: D2H");
    ctx->launches += 3;
  }
  if (st == MOAO_OK && cudaGetLastError() != cudaSuccess)
    st = set_error(MOAO_ERR_CUDA, "intersample_inputs: kernel launch");
  if (cudaStreamSynchronize(s) != cudaSuccess && st == MOAO_OK)
    st = set_error(MOAO_ERR_CUDA, "intersample_inputs: synchronize");
  fft2d_free(&plan);
  cudaFree(z);
  cudaFree(d);
  return st;
}

extern "C" moao_status moao_intersample_create_synth(moao_ctx* ctx, long nssp, double Dtel,
                                                     double obs, double coupling,
                                                     moao_isample** out) {
  if (!ctx || !out) return set_error(MOAO_ERR_BAD_ARG, "intersample_create_synth: null");
  long na = 0, N = 0;
  MOAO_TRY(moao_intersample_inputs(ctx, nssp, Dtel, obs, coupling, &na, &N, nullptr, nullptr,
                                   nullptr));
  std::vector<long> idx((size_t)na * na);
  std::vector<double> a((size_t)N * N), o((size_t)N * N);
  MOAO_TRY(moao_intersample_inputs(ctx, nssp, Dtel, obs, coupling, &na, &N, idx.data(), a.data(),
                                   o.data()));
  return moao_intersample_create(ctx, na * na, nssp + 1, Dtel, idx.data(), a.data(), o.data(), out);
}
