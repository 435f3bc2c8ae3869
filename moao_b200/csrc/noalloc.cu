// FP64 reconstructor that allocates no device memory.
//
// Some callers cannot call cudaMalloc while they run: a real-time controller
// of an adaptive-optics system, which recomputes its reconstructor between
// frames under a fixed time budget and cannot risk an allocation blocking in
// the driver; or a host application that has already handed all of the GPU's
// memory to its own pool. For them this entry point keeps its scratch (the
// inverse diagonal blocks, one panel and the pivot flag) in one file-scope
// __device__ array of fixed size, which every GPU that loads the library holds
// until the process exits. The caller passes the inputs and outputs.
#include <cuda_runtime.h>

#include <algorithm>

#include "context.h"
#include "dense.h"

namespace {

constexpr long kNoAllocMaxN = 2048;  // limit on nmeas and on nmeasts
constexpr long kNoAllocNb = 256;     // panel width used by this entry point
constexpr size_t kDinvDoubles = (size_t)kNoAllocMaxN * kNoAllocNb;
constexpr size_t kPanelDoubles = (size_t)kNoAllocMaxN * kNoAllocNb;
constexpr size_t kScratchDoubles = kDinvDoubles + kPanelDoubles + 32;  // + pivot flag

// 8 MiB + 256 bytes of device memory per GPU, shared by every call.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of the scratch array in the current context. A __device__
// symbol's address belongs to the CUDA context that loaded the module, not to
// the device: after cudaDeviceReset the module is loaded again, and a caller
// driving its own driver-API context gets a different copy. So the address is
// looked up on every call (a host-side table lookup once the module is loaded;
// it allocates nothing). The first call in a context loads the module.
moao_status scratch_for_current_context(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return moao::set_error(MOAO_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
                                              cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  return MOAO_OK;
}

}  // namespace

extern "C" moao_status moao_reconstructor_noalloc(long nmeas, long nmeasts, double* d_Cmm,
                                                  long ldCmm, double* d_Ctm, long ldCtm, long ngal,
                                                  void* stream, int* info) {
  using namespace moao;
  if (nmeas < 0 || nmeasts < 0 || ngal < 0 || ldCmm < std::max(1L, nmeas) ||
      ldCtm < std::max(1L, nmeasts) || (nmeas > 0 && (!d_Cmm || !d_Ctm)))
    return set_error(MOAO_ERR_BAD_ARG,
                     "reconstructor_noalloc: bad sizes, pointers or leading dimensions");
  if (nmeas > kNoAllocMaxN || nmeasts > kNoAllocMaxN)
    return set_error(MOAO_ERR_BAD_ARG,
                     "reconstructor_noalloc: nmeas and nmeasts must be at most 2048 (the size "
                     "of its fixed device scratch); use moao_reconstructor for larger systems");
  if (info) *info = 0;
  if (nmeas == 0) return MOAO_OK;  // nothing to factor, as moao_reconstructor
  int cur = 0, sdev = 0;
  MOAO_CUDA_TRY(cudaGetDevice(&cur));
  MOAO_CUDA_TRY(cudaStreamGetDevice(static_cast<cudaStream_t>(stream), &sdev));
  if (sdev != cur)
    return set_error(MOAO_ERR_BAD_ARG,
                     "reconstructor_noalloc: the stream belongs to device " + std::to_string(sdev) +
                         " but the current device is " + std::to_string(cur));
  double* scratch = nullptr;
  MOAO_TRY(scratch_for_current_context(&scratch));
  double* dinv = scratch;                 // nmeas x 256, leading dimension nmeas
  double* W = scratch + kDinvDoubles;     // one panel
  int* d_info = reinterpret_cast<int*>(W + kPanelDoubles);

  moao_ctx c;  // host-side bookkeeping only; owns no device memory
  c.device = cur;
  c.stream = static_cast<cudaStream_t>(stream);
  c.nb = (int)kNoAllocNb;
  const long n = nmeas, nb = kNoAllocNb;
  // The array keeps the previous call's contents; the pivot flag must start at 0.
  MOAO_CUDA_TRY(cudaMemsetAsync(d_info, 0, 2 * sizeof(int), c.stream));
  for (long k0 = 0; k0 < n; k0 += nb) {
    const long kb = std::min(nb, n - k0);
    double* Akk = d_Cmm + k0 + k0 * ldCmm;
    MOAO_TRY(potrf_inv_block(&c, Akk, ldCmm, dinv + k0, n, kb, k0, d_info, W));
    const long rest = n - k0 - kb;
    if (rest <= 0) break;
    double* P = d_Cmm + (k0 + kb) + k0 * ldCmm;
    MOAO_TRY(gemm(&c, rest, kb, kb, 1.0, P, ldCmm, dinv + k0, n, true, 0.0, W, rest));
    MOAO_TRY(copy_matrix(W, rest, P, ldCmm, rest, kb, c.stream));
    double* A22 = d_Cmm + (k0 + kb) + (k0 + kb) * ldCmm;
    MOAO_TRY(gemm(&c, rest, rest, kb, -1.0, P, ldCmm, P, ldCmm, true, 1.0, A22, ldCmm, true));
  }
  int h_info = 0;
  MOAO_CUDA_TRY(cudaMemcpyAsync(&h_info, d_info, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
  MOAO_CUDA_TRY(cudaStreamSynchronize(c.stream));
  if (info) *info = h_info;
  if (h_info) return set_error(MOAO_ERR_NOT_SPD, "reconstructor_noalloc: non-positive pivot at column " +
                                                     std::to_string(h_info));
  for (long g = 0; g < ngal && nmeasts > 0; ++g) {  // ngal 0: factor only
    double* B = d_Ctm + nmeas * nmeasts * g;
    const long m = nmeasts;
    for (long k0 = 0; k0 < n; k0 += nb) {  // X L^T = B
      const long kb = std::min(nb, n - k0);
      double* Bk = B + k0 * ldCtm;
      MOAO_TRY(gemm(&c, m, kb, kb, 1.0, Bk, ldCtm, dinv + k0, n, true, 0.0, W, m));
      MOAO_TRY(copy_matrix(W, m, Bk, ldCtm, m, kb, c.stream));
      const long rest = n - k0 - kb;
      if (rest > 0)
        MOAO_TRY(gemm(&c, m, rest, kb, -1.0, Bk, ldCtm, d_Cmm + (k0 + kb) + k0 * ldCmm, ldCmm,
                      true, 1.0, B + (k0 + kb) * ldCtm, ldCtm));
    }
    for (long b = (n + nb - 1) / nb - 1; b >= 0; --b) {  // R L = X
      const long k0 = b * nb, kb = std::min(nb, n - k0);
      double* Bk = B + k0 * ldCtm;
      MOAO_TRY(gemm(&c, m, kb, kb, 1.0, Bk, ldCtm, dinv + k0, n, false, 0.0, W, m));
      MOAO_TRY(copy_matrix(W, m, Bk, ldCtm, m, kb, c.stream));
      if (k0 > 0)
        MOAO_TRY(gemm(&c, m, k0, kb, -1.0, Bk, ldCtm, d_Cmm + k0, ldCmm, false, 1.0, B, ldCtm));
    }
  }
  MOAO_CUDA_TRY(cudaStreamSynchronize(c.stream));
  return MOAO_OK;
}
