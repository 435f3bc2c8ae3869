// Square 2-D complex FFTs in FP64 (fft.cu) for the intersample PSF and the
// synthesis of its input tables.
#ifndef MOAO_FFT_H
#define MOAO_FFT_H

#include <cuda_runtime.h>

#include "moao_internal.h"

namespace moao {

struct Cplx {
  double x, y;
};

// An N x N transform (N a power of two, 2 <= N <= 2048): twiddle table and a
// scratch array of N * N values on the device.
struct Fft2d {
  long N = 0;
  int logN = 0;
  Cplx* tw = nullptr;    // exp(-2 pi i k / N), k < N / 2
  Cplx* tmp = nullptr;   // N * N
};

moao_status fft2d_plan(Fft2d* f, long N);
void fft2d_free(Fft2d* f);
// In place on data (row-major N x N: data[r * N + c]), unnormalised:
// dir = -1 forward (exp(-2 pi i ...)), +1 inverse (exp(+2 pi i ...)), the
// conventions of FFTW and numpy.fft. Four launches on s.
moao_status fft2d(const Fft2d& f, Cplx* data, int dir, cudaStream_t s, long long* launches);

}  // namespace moao

#endif  // MOAO_FFT_H
