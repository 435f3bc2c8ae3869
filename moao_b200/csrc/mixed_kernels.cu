// Conversion and slicing kernels of the mixed-precision reconstructor.
//
//   cvt_*            FP32 <-> FP64 copies of column-major blocks
//   split_bf16       FP64 block -> bf16 hi + lo (hi = bf16(x), lo = bf16(x - hi)),
//                    written row-major (K-major operand of the tensor-core GEMM,
//                    via a shared-memory transpose) and/or column-major
//   ozaki_*          int8 slices for the exact-accumulation residual: every row of
//                    R (and every column of the symmetric Cmm) gets a power-of-two
//                    exponent e with max |x| < 2^e; then
//                      x 2^-e = sum_p q_p 2^-(6 + 7(p-1)),  q_p in [-64, 64],
//                    each q_p the rounded remainder of the previous slice, so the
//                    products of slices accumulate exactly in int32.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <type_traits>

#include "mixed.h"

namespace moao {

// Kernels launched by the helpers below on the calling thread (the driver adds
// the difference over a call to its context's launch count).
static thread_local long long tl_launches = 0;
long long helper_launches() { return tl_launches; }

namespace {

unsigned blocks_for(long total, long per = 256) {
  return (unsigned)std::max(1L, std::min((total + per - 1) / per, 148L * 16));
}

__global__ void cvt_f32_f64_kernel(const float* __restrict__ s, long lds, double* __restrict__ d,
                                   long ldd, long m, long n, int lower) {
  const long total = m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    if (lower && i < j) continue;
    d[j * ldd + i] = (double)s[j * lds + i];
  }
}

__global__ void cvt_f64_f32_kernel(const double* __restrict__ s, long lds, float* __restrict__ d,
                                   long ldd, long m, long n, int lower) {
  const long total = m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    if (lower && i < j) continue;
    d[j * ldd + i] = (float)s[j * lds + i];
  }
}

__global__ void add_f32_to_f64_kernel(const float* __restrict__ s, long lds, double* __restrict__ d,
                                      long ldd, long m, long n) {
  const long total = m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    d[j * ldd + i] += (double)s[j * lds + i];
  }
}

// 32x32 tiles, 32x8 threads. Slice k = bf16(x - sum of the previous slices),
// computed in FP64: two slices carry ~16 significant bits, three ~24.
__global__ void split_bf16_kernel(const double* __restrict__ src, long lds, long m, long n,
                                  int ns, BfSlices rmaj, long ldr, BfSlices cmaj, long ldc) {
  __shared__ __nv_bfloat16 t[kMaxBfSlices][32][34];
  const long r0 = (long)blockIdx.x * 32, c0 = (long)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int jj = ty; jj < 32; jj += 8) {
    const long r = r0 + tx, c = c0 + jj;
    double rem = 0;
    if (r < m && c < n) rem = src[c * lds + r];
    for (int k = 0; k < ns; ++k) {
      const __nv_bfloat16 h = __double2bfloat16(rem);
      rem -= (double)__bfloat162float(h);
      t[k][tx][jj] = h;
      if (cmaj.p[0] && r < m && c < n)
        static_cast<__nv_bfloat16*>(cmaj.p[k])[c * ldc + r] = h;
    }
  }
  if (!rmaj.p[0]) return;
  __syncthreads();
  for (int ii = ty; ii < 32; ii += 8) {
    const long r = r0 + ii, c = c0 + tx;
    if (r < m && c < n)
      for (int k = 0; k < ns; ++k)
        static_cast<__nv_bfloat16*>(rmaj.p[k])[r * ldr + c] = t[k][ii][tx];
  }
}

__device__ __forceinline__ int exponent_of(double mx) {
  // smallest e with mx < 2^e (0 for an all-zero row)
  if (!(mx > 0)) return 0;
  return ilogb(mx) + 1;
}

// 2^k for an exponent in the normal range (exact), ldexp otherwise.
__device__ __forceinline__ double pow2i(int k) {
  return (k >= -1022 && k <= 1023) ? __longlong_as_double((long long)(k + 1023) << 52)
                                   : ldexp(1.0, k);
}

// 2^k in FP32 for an exponent in the normal range (exact), ldexpf otherwise.
__device__ __forceinline__ float pow2f(int k) {
  return (k >= -126 && k <= 127) ? __int_as_float((k + 127) << 23) : ldexpf(1.f, k);
}

// Row maxima of a column-major m x n block (FP64 or FP32 values): 32 rows per
// block, blockDim.y (<= 32) column strides, 4 loads in flight per thread.
template <typename T>
__global__ void row_exponent_kernel(const T* __restrict__ A, long lda, long m, long n,
                                    int* __restrict__ e, int bias) {
  __shared__ double red[32][33];
  const int ny = blockDim.y;
  const long r = (long)blockIdx.x * 32 + threadIdx.x;
  double mx = 0;
  if (r < m) {
    long c = threadIdx.y;
    for (; c + 3 * ny < n; c += 4 * ny) {
      const double a0 = fabs((double)A[c * lda + r]), a1 = fabs((double)A[(c + ny) * lda + r]);
      const double a2 = fabs((double)A[(c + 2 * ny) * lda + r]);
      const double a3 = fabs((double)A[(c + 3 * ny) * lda + r]);
      mx = fmax(mx, fmax(fmax(a0, a1), fmax(a2, a3)));
    }
    for (; c < n; c += ny) mx = fmax(mx, fabs((double)A[c * lda + r]));
  }
  red[threadIdx.y][threadIdx.x] = mx;
  __syncthreads();
  if (threadIdx.y == 0 && r < m) {
    for (int k = 1; k < ny; ++k) mx = fmax(mx, red[k][threadIdx.x]);
    e[r] = exponent_of(mx) - bias;
  }
}

// Column maxima of a column-major m x n block: one block per column.
template <typename T>
__global__ void col_exponent_kernel(const T* __restrict__ A, long lda, long m, long n,
                                    int* __restrict__ e, int bias) {
  __shared__ double red[32];
  const long c = blockIdx.x;
  double mx = 0;
  for (long r = threadIdx.x; r < m; r += blockDim.x) mx = fmax(mx, fabs((double)A[c * lda + r]));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) mx = fmax(mx, red[w]);
    e[c] = exponent_of(mx) - bias;
  }
}

// 32x32 tiles, 32x8 threads. fp16 slices of x * 2^-e: slice k = fp16 of what
// the previous slices left (in FP64), e = erow[r] for the row-major copy and
// ecol[c] for the column-major one, so either copy can be scaled back exactly
// by a power of two per row of the operand it feeds. x is FP64 or FP32 (an
// FP32 x is exact in FP64, so both give the same slices).
template <typename T>
__global__ void split_f16_kernel(const T* __restrict__ src, long lds, long m, long n, int ns,
                                 BfSlices rmaj, long ldr, const int* __restrict__ erow,
                                 BfSlices cmaj, long ldc, const int* __restrict__ ecol) {
  __shared__ __half t[kMaxBfSlices][32][34];
  const long r0 = (long)blockIdx.x * 32, c0 = (long)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int jj = ty; jj < 32; jj += 8) {
    const long r = r0 + tx, c = c0 + jj;
    if constexpr (std::is_same<T, float>::value) {
      // FP32 source: x 2^-e and every remainder are exact in FP32 (a value minus
      // its fp16 rounding fits the 24-bit significand), so the slices equal the
      // FP64 computation's
      float x = 0.f;
      if (r < m && c < n) x = src[c * lds + r];
      if (rmaj.p[0]) {
        float rem = (r < m) ? x * pow2f(-erow[r]) : 0.f;
        for (int k = 0; k < ns; ++k) {
          const __half h = __float2half_rn(rem);
          rem -= __half2float(h);
          t[k][tx][jj] = h;
        }
      }
      if (cmaj.p[0] && r < m && c < n) {
        float rem = x * pow2f(-ecol[c]);
        for (int k = 0; k < ns; ++k) {
          const __half h = __float2half_rn(rem);
          rem -= __half2float(h);
          static_cast<__half*>(cmaj.p[k])[c * ldc + r] = h;
        }
      }
    } else {
      double x = 0;
      if (r < m && c < n) x = (double)src[c * lds + r];
      if (rmaj.p[0]) {
        double rem = (r < m) ? x * pow2i(-erow[r]) : 0.0;
        for (int k = 0; k < ns; ++k) {
          const __half h = __double2half(rem);
          rem -= (double)__half2float(h);
          t[k][tx][jj] = h;
        }
      }
      if (cmaj.p[0] && r < m && c < n) {
        double rem = x * pow2i(-ecol[c]);
        for (int k = 0; k < ns; ++k) {
          const __half h = __double2half(rem);
          rem -= (double)__half2float(h);
          static_cast<__half*>(cmaj.p[k])[c * ldc + r] = h;
        }
      }
    }
  }
  if (!rmaj.p[0]) return;
  __syncthreads();
  for (int ii = ty; ii < 32; ii += 8) {
    const long r = r0 + ii, c = c0 + tx;
    if (r < m && c < n)
      for (int k = 0; k < ns; ++k) static_cast<__half*>(rmaj.p[k])[r * ldr + c] = t[k][ii][tx];
  }
}

// Row-major fp16 slices of an FP32 column-major m x kb block (kb <= kSplitMaxCols)
// from its row exponents; columns kb..kpad-1 of the slices get zeros (the tensor
// core reads K in steps of 64). Same exponents and slices as row_exponent_kernel +
// split_f16_kernel.
constexpr int kSplitMaxCols = 1024;

// A CTA takes a 32-row x 64-column tile, reads it column by column (coalesced
// over the rows) into shared memory and writes each row's 64 entries as 32
// half2 words per slice (coalesced over the columns); columns kb..kpad-1 are
// written as zeros.
__global__ void __launch_bounds__(256) split_rows_f16_t_kernel(const float* __restrict__ src,
                                                               long lds, long m, int kb, int ns,
                                                               BfSlices out, long ldx, int kpad,
                                                               const int* __restrict__ erow) {
  __shared__ float2 t[32][33];  // t[row][column pair]
  const long r0 = (long)blockIdx.x * 32;
  const int c0 = blockIdx.y * 64;
  const int tx = threadIdx.x, ty = threadIdx.y;
  float* tf = reinterpret_cast<float*>(&t[0][0]);
  for (int cc = ty; cc < 64; cc += 8) {
    const long r = r0 + tx;
    const int c = c0 + cc;
    tf[tx * 66 + cc] = (r < m && c < kb) ? src[(long)c * lds + r] : 0.f;
  }
  __syncthreads();
  const int c = c0 + 2 * tx;
  if (c >= kpad) return;
  for (int rr = ty; rr < 32; rr += 8) {
    const long row = r0 + rr;
    if (row >= m) continue;
    const float sc = pow2f(-erow[row]);
    const float2 v = t[rr][tx];
    float a = v.x * sc, b = v.y * sc;
    for (int k = 0; k < ns; ++k) {
      const __half ha = __float2half_rn(a), hb = __float2half_rn(b);
      a -= __half2float(ha);
      b -= __half2float(hb);
      *reinterpret_cast<__half2*>(static_cast<__half*>(out.p[k]) + row * ldx + c) =
          __halves2half2(ha, hb);
    }
  }
}

// Slices of the rows of a column-major m x n block into row-major int8 (ldo).
__global__ void split_rows_i8_kernel(const double* __restrict__ A, long lda, long m, long n,
                                     const int* __restrict__ e, int ns, int8_t* out, long ldo,
                                     long slice_stride) {
  __shared__ int8_t q[kMaxOzakiSlices][32][36];
  const long r0 = (long)blockIdx.x * 32, c0 = (long)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int jj = ty; jj < 32; jj += 8) {
    const long r = r0 + tx, c = c0 + jj;
    double v = 0;
    if (r < m && c < n) v = ldexp(A[c * lda + r], 6 - e[r]);
    for (int s = 0; s < ns; ++s) {
      const double qv = rint(v);
      q[s][tx][jj] = (int8_t)qv;
      v = (v - qv) * 128.0;
    }
  }
  __syncthreads();
  for (int ii = ty; ii < 32; ii += 8) {
    const long r = r0 + ii, c = c0 + tx;
    if (r < m && c < n)
      for (int s = 0; s < ns; ++s) out[s * slice_stride + r * ldo + c] = q[s][ii][tx];
  }
}

struct OffsetValues {
  double v[kMaxOffsetRanges];
};

OffsetValues values_of(const OffsetRanges& off) {
  OffsetValues o{};
  for (int w = 0; w < off.n; ++w) o.v[w] = off.value[w];
  return o;
}

// Stored element A(r, c) (r >= c) minus the offset of its block.
__device__ __forceinline__ double stored_minus(const double* A, long lda, long r, long c,
                                               const int* rid, const OffsetValues& ov) {
  double v = A[c * lda + r];
  if (rid) {
    const int w = rid[r];
    if (w >= 0 && w == rid[c]) v -= ov.v[w];
  }
  return v;
}

// Column maxima of sym(A) for a lower-stored n x n A: every stored (r >= c)
// element feeds column c and column r.
__global__ void sym_col_max_kernel(const double* __restrict__ A, long lda, long n,
                                   unsigned long long* __restrict__ cm, const int* rid,
                                   const OffsetValues ov) {
  const long r0 = (long)blockIdx.x * 32, c0 = (long)blockIdx.y * 32;
  if (r0 + 31 < c0) return;
  const int tx = threadIdx.x, ty = threadIdx.y;
  __shared__ double t[32][33];
  for (int jj = ty; jj < 32; jj += 8) {
    const long r = r0 + tx, c = c0 + jj;
    t[tx][jj] = (r < n && c < n && r >= c) ? fabs(stored_minus(A, lda, r, c, rid, ov)) : 0.0;
  }
  __syncthreads();
  if (ty == 0) {  // column c0 + tx: max over the 32 rows
    double mx = 0;
    for (int i = 0; i < 32; ++i) mx = fmax(mx, t[i][tx]);
    if (c0 + tx < n) atomicMax(&cm[c0 + tx], __double_as_longlong(mx));
  } else if (ty == 1) {  // row r0 + tx: max over the 32 columns (its mirrored column)
    double mx = 0;
    for (int j = 0; j < 32; ++j) mx = fmax(mx, t[tx][j]);
    if (r0 + tx < n) atomicMax(&cm[r0 + tx], __double_as_longlong(mx));
  }
}

__global__ void exponents_from_max_kernel(const unsigned long long* __restrict__ cm, long n,
                                          int* __restrict__ f) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) f[i] = exponent_of(__longlong_as_double((long long)cm[i]));
}

// Slices of sym(A) by columns, written as B[j * ldo + k] = slice(S(k, j)) (the
// K-major B operand of S), S(k, j) = A(max(k,j), min(k,j)).
__global__ void split_sym_i8_kernel(const double* __restrict__ A, long lda, long n,
                                    const int* __restrict__ f, int ns, int8_t* out, long ldo,
                                    long slice_stride, const int* rid, const OffsetValues ov) {
  __shared__ double t[32][33];  // t[jj][kk] = S(k0+kk, j0+jj)
  const long j0 = (long)blockIdx.x * 32, k0 = (long)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  if (k0 >= j0 + 32) {
    // k > j everywhere: S(k, j) = A(k, j), contiguous in k
    for (int jj = ty; jj < 32; jj += 8) {
      const long k = k0 + tx, j = j0 + jj;
      t[jj][tx] = (k < n && j < n) ? stored_minus(A, lda, k, j, rid, ov) : 0.0;
    }
  } else if (k0 + 32 <= j0) {
    // k < j everywhere: S(k, j) = A(j, k), contiguous in j
    for (int kk = ty; kk < 32; kk += 8) {
      const long j = j0 + tx, k = k0 + kk;
      t[tx][kk] = (k < n && j < n) ? stored_minus(A, lda, j, k, rid, ov) : 0.0;
    }
  } else {
    for (int jj = ty; jj < 32; jj += 8) {
      const long k = k0 + tx, j = j0 + jj;
      double v = 0;
      if (k < n && j < n)
        v = (k >= j) ? stored_minus(A, lda, k, j, rid, ov) : stored_minus(A, lda, j, k, rid, ov);
      t[jj][tx] = v;
    }
  }
  __syncthreads();
  // 4 consecutive k per thread, one 32-bit store per slice (the row stride ldo is
  // a multiple of 4; slice columns n..ldo-1 are never read, so a word that runs
  // past n may hold zeros there)
  const int tid = ty * 32 + tx;
  const int jj = tid >> 3, kq = (tid & 7) * 4;
  const long j = j0 + jj, k = k0 + kq;
  if (j >= n || k >= n) return;
  const double sc = pow2i(6 - f[j]);
  double v[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = (k + i < n) ? t[jj][kq + i] * sc : 0.0;
  for (int s = 0; s < ns; ++s) {
    uint32_t w = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const double qv = rint(v[i]);
      w |= (uint32_t)(uint8_t)(int8_t)qv << (8 * i);
      v[i] = (v[i] - qv) * 128.0;
    }
    *reinterpret_cast<uint32_t*>(out + s * slice_stride + j * ldo + k) = w;
  }
}

// ---- exact products by the Chinese remainder theorem

constexpr int crt_modinv(int a, int m) {  // a^-1 mod m (gcd(a, m) = 1), extended Euclid
  int t = 0, nt = 1, r = m, nr = a % m;
  while (nr != 0) {
    const int q = r / nr;
    const int t2 = t - q * nt;
    t = nt;
    nt = t2;
    const int r2 = r - q * nr;
    r = nr;
    nr = r2;
  }
  return t < 0 ? t + m : t;
}

// kCrtMod[i] as a constant expression usable in device code
constexpr int crt_mod(int i) {
  constexpr int tab[kCrtMaxModuli] = {256, 255, 253, 251, 247, 241, 239,
                                      233, 229, 227, 223, 217, 211};
  return tab[i];
}

constexpr bool crt_table_matches() {
  for (int i = 0; i < kCrtMaxModuli; ++i)
    if (crt_mod(i) != kCrtMod[i]) return false;
  return true;
}
static_assert(crt_table_matches(), "device and host moduli tables");
static_assert(crt_mod(0) == 256, "the first modulus is taken from the low byte");

// Rounding to the nearest integer by the FP64 magic constant 1.5 * 2^52: for
// |y| < 2^51, y + kMagic64 holds round(y) in its low mantissa bits, and
// subtracting kMagic64 again gives it as a double (exact); the low 32 bits of
// the sum are round(y) in two's complement.
constexpr double kMagic64 = 6755399441055744.0;
constexpr float kMagic32 = 12582912.0f;  // 1.5 * 2^23, for |y| < 2^22 in FP32

// Centred residue of the integer x (|x| <= 2^41, exact in FP64) modulo the
// I-th modulus and those after it, for I < nmod: r = x - M round(x / M). The
// quotient's error, |x / M| 2^-52 <= 2^-19, is far below the distance of x / M
// from a half-integer for odd M (at least 1 / 2M), so the rounding picks the
// nearest integer, r is exact and lies in [-(M - 1) / 2, (M - 1) / 2].
template <int I>
__device__ __forceinline__ void crt_residue_from(double x, int nmod, int8_t* r) {
  if constexpr (I < kCrtMaxModuli) {
    if (I < nmod) {
      constexpr int M = crt_mod(I);
      constexpr double INV = 1.0 / M;
      const double q = fma(x, INV, kMagic64) - kMagic64;
      const double t = fma(-(double)M, q, x);
      r[I] = (int8_t)__double2loint(t + kMagic64);
    }
    crt_residue_from<I + 1>(x, nmod, r);
  }
}

// Centred residues of the integer x (|x| <= 2^41) modulo the first nmod moduli:
// m_0 = 256 from the low byte of its two's complement.
__device__ __forceinline__ void crt_residues(double x, int nmod, int8_t* r) {
  r[0] = (int8_t)(__double2loint(x + kMagic64) & 0xFF);
  crt_residue_from<1>(x, nmod, r);
}

// The residues of four integers x[0..3] (|x| <= 2^41) modulo the I-th modulus
// and those after it, each packed into one word w[I] (byte q = residue of x[q]):
// the low 32 bits of r + kMagic64 hold r in two's complement, and two levels of
// byte permutes assemble the word.
template <int I>
__device__ __forceinline__ void crt_words_from(const double* x, int nmod, uint32_t* w) {
  if constexpr (I < kCrtMaxModuli) {
    if (I < nmod) {
      int l[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if constexpr (I == 0) {
          l[q] = __double2loint(x[q] + kMagic64);  // the low byte: x mod 256
        } else {
          constexpr int M = crt_mod(I);
          constexpr double INV = 1.0 / M;
          const double qt = fma(x[q], INV, kMagic64) - kMagic64;
          l[q] = __double2loint(fma(-(double)M, qt, x[q]) + kMagic64);
        }
      }
      w[I] = __byte_perm(__byte_perm(l[0], l[1], 0x0040), __byte_perm(l[2], l[3], 0x0040), 0x5410);
    }
    crt_words_from<I + 1>(x, nmod, w);
  }
}

// Garner's step for modulus I: t <- (((t - v_0) m_0^-1 - v_1) m_1^-1 - ...) mod m_I,
// centred, in FP32: every operand is an integer below 2^17 in magnitude (exact),
// and y / M (error <= 2^-14) is at least 1 / 2M from a half-integer.
template <int I, int J>
__device__ __forceinline__ float crt_garner_inner(float t, const float* v) {
  if constexpr (J < I) {
    constexpr int M = crt_mod(I);
    constexpr float INV = 1.0f / M;
    constexpr float MINV = (float)crt_modinv(crt_mod(J) % M, M);
    const float y = (t - v[J]) * MINV;
    t = fmaf(-(float)M, fmaf(y, INV, kMagic32) - kMagic32, y);
    return crt_garner_inner<I, J + 1>(t, v);
  } else {
    return t;
  }
}

// Centred mixed-radix digits v_I.. of the value whose residues are z_i
template <int I>
__device__ __forceinline__ void crt_digits_from(const uint8_t* __restrict__ Z, long idx,
                                                long zstride, int nmod, float* v) {
  if constexpr (I < kCrtMaxModuli) {
    if (I < nmod) {
      v[I] = crt_garner_inner<I, 0>((float)Z[I * zstride + idx], v);  // I >= 1 steps: centred
    }
    crt_digits_from<I + 1>(Z, idx, zstride, nmod, v);
  }
}

// Horner over the digits I..min(nmod, END)-1 in 64-bit integers:
// v_I + m_I (v_(I+1) + m_(I+1) (...)).
template <int I, int END>
__device__ __forceinline__ long long crt_horner64(const float* v, int nmod) {
  if constexpr (I < END) {
    if (I >= nmod) return 0;
    return (long long)(int)v[I] + (long long)crt_mod(I) * crt_horner64<I + 1, END>(v, nmod);
  } else {
    return 0;
  }
}

// The value of the digits as a double: P = L + W_7 H with L the first seven
// digits' part (|L| < 2^55) and H the rest's (|H| < 2^47), both exact in int64;
// W_7 = m_0 ... m_6 = 2^8 times a 48-bit odd number is exact in FP64, so P
// comes out within two roundings.
constexpr int kCrtSplit = 7;
constexpr double crt_w7() {
  double w = 1.0;
  for (int i = 0; i < kCrtSplit; ++i) w *= crt_mod(i);
  return w;
}
__device__ __forceinline__ double crt_digits_value(const float* v, int nmod) {
  const long long L = crt_horner64<0, kCrtSplit>(v, nmod);
  if (nmod <= kCrtSplit) return (double)L;
  const long long H = crt_horner64<kCrtSplit, kCrtMaxModuli>(v, nmod);
  return fma((double)H, crt_w7(), (double)L);
}

// Residues of the rows of a column-major m x n block into row-major int8 (ldo),
// X = rint(A(r, c) 2^(sh - e[r])), sh = 7 ns - 1.
__global__ void crt_rows_kernel(const double* __restrict__ A, long lda, long m, long n,
                                const int* __restrict__ e, int sh, int nmod, int8_t* out,
                                long ldo, long stride) {
  __shared__ int8_t q[kCrtMaxModuli][32][36];
  const long r0 = (long)blockIdx.x * 32, c0 = (long)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int jj = ty; jj < 32; jj += 8) {
    const long r = r0 + tx, c = c0 + jj;
    double v = 0;
    if (r < m && c < n) v = ldexp(A[c * lda + r], sh - e[r]);
    int8_t res[kCrtMaxModuli] = {};
    crt_residues((v + kMagic64) - kMagic64, nmod, res);
#pragma unroll
    for (int i = 0; i < kCrtMaxModuli; ++i)
      if (i < nmod) q[i][tx][jj] = res[i];
  }
  __syncthreads();
  for (int ii = ty; ii < 32; ii += 8) {
    const long r = r0 + ii, c = c0 + tx;
    if (r < m && c < n)
      for (int i = 0; i < nmod; ++i) out[i * stride + r * ldo + c] = q[i][ii][tx];
  }
}

// Residues of sym(A) by columns, written as B[j * ldo + k] = residue(S(k, j))
// (the K-major B operand), S(k, j) = A(max(k,j), min(k,j)) minus offsets,
// whose exponent is f[j]. B is not symmetric (the scale is per column), but
// B[j][k] and B[k][j] scale the same stored element: a block of 32 x 32 tiles
// at or below the diagonal (kb >= jb) loads its stored elements once and
// writes the residues of both orientations, each thread four consecutive
// entries of a row per residue (one 32-bit coalesced store).
__global__ void crt_sym_kernel(const double* __restrict__ A, long lda, long n,
                               const int* __restrict__ f, int sh, int nmod, int8_t* out,
                               long ldo, long stride, const int* rid, const OffsetValues ov) {
  __shared__ double t[32][33];  // t[jj][kk] = S(k0+kk, j0+jj)
  // tile (jb, kb) with kb >= jb from the linear index (kb rows of the lower triangle)
  const long tix = blockIdx.x;
  long kb = (long)((sqrt(8.0 * (double)tix + 1.0) - 1.0) * 0.5);
  while ((kb + 1) * (kb + 2) / 2 <= tix) ++kb;
  while (kb * (kb + 1) / 2 > tix) --kb;
  const long jb = tix - kb * (kb + 1) / 2;
  const long j0 = jb * 32, k0 = kb * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  if (k0 > j0) {
    // k > j everywhere: S(k, j) = A(k, j), contiguous in k
    for (int jj = ty; jj < 32; jj += 8) {
      const long k = k0 + tx, j = j0 + jj;
      t[jj][tx] = (k < n && j < n) ? stored_minus(A, lda, k, j, rid, ov) : 0.0;
    }
  } else {
    for (int jj = ty; jj < 32; jj += 8) {
      const long k = k0 + tx, j = j0 + jj;
      double v = 0;
      if (k < n && j < n)
        v = (k >= j) ? stored_minus(A, lda, k, j, rid, ov) : stored_minus(A, lda, j, k, rid, ov);
      t[jj][tx] = v;
    }
  }
  __syncthreads();
  const int tid = ty * 32 + tx;
  const int a = tid >> 3, q4 = (tid & 7) * 4;
  // direct orientation: row j0 + a, entries k0 + q4 .. + 3 at f[j]
  {
    const long j = j0 + a, k = k0 + q4;
    if (j < n && k < n) {
      const double sc = pow2i(sh - f[j]);
      double x[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double v = (k + q < n) ? t[a][q4 + q] * sc : 0.0;
        x[q] = (v + kMagic64) - kMagic64;
      }
      uint32_t w[kCrtMaxModuli];
      crt_words_from<0>(x, nmod, w);
#pragma unroll
      for (int i = 0; i < kCrtMaxModuli; ++i)
        if (i < nmod) *reinterpret_cast<uint32_t*>(out + i * stride + j * ldo + k) = w[i];
    }
  }
  if (k0 == j0) return;  // a diagonal tile's mirror is itself
  // mirrored orientation: row k0 + a (column k of S, exponent f[k]), entries
  // j0 + q4 .. + 3
  {
    const long k = k0 + a, j = j0 + q4;
    if (k < n && j < n) {
      const double sc = pow2i(sh - f[k]);
      double x[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double v = (j + q < n) ? t[q4 + q][a] * sc : 0.0;
        x[q] = (v + kMagic64) - kMagic64;
      }
      uint32_t w[kCrtMaxModuli];
      crt_words_from<0>(x, nmod, w);
#pragma unroll
      for (int i = 0; i < kCrtMaxModuli; ++i)
        if (i < nmod) *reinterpret_cast<uint32_t*>(out + i * stride + k * ldo + j) = w[i];
    }
  }
}

// E = C + alpha * P 2^(e[r] + f[c] - 2 sh) from P's residues: centred mixed-
// radix digits by Garner's method, then P from them (crt_digits_value). One
// element per thread: blockIdx.x is the column, blockIdx.y the block of rows.
__global__ void crt_combine_kernel(const uint8_t* __restrict__ Z, long m, long zstride, int nmod,
                                   int sh, const int* __restrict__ e, const int* __restrict__ f,
                                   const double* __restrict__ C, long ldc, double alpha,
                                   double* __restrict__ E, long lde) {
  const long r = (long)blockIdx.y * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const long c = blockIdx.x;
  const long idx = c * m + r;
  float v[kCrtMaxModuli];
  const int z0 = Z[idx];
  v[0] = (float)(z0 >= 128 ? z0 - 256 : z0);
  crt_digits_from<1>(Z, idx, zstride, nmod, v);
  const double val = crt_digits_value(v, nmod);
  E[c * lde + r] = C[c * ldc + r] + alpha * (val * pow2i(e[r] + f[c] - 2 * sh));
}

// ---- offsets by the Woodbury identity

__global__ void cvt_lower_minus_kernel(const double* __restrict__ s, long lds,
                                       float* __restrict__ d, long ldd, long n,
                                       const int* __restrict__ rid, const OffsetValues ov) {
  const long total = n * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, j = e / n;
    if (i < j) continue;
    d[j * ldd + i] = (float)stored_minus(s, lds, i, j, rid, ov);
  }
}

struct RangeList {
  int n;
  int begin[kMaxOffsetRanges], end[kMaxOffsetRanges];
};

RangeList ranges_of(const OffsetRanges& off) {
  RangeList r{};
  r.n = off.n;
  for (int w = 0; w < off.n; ++w) {
    r.begin[w] = off.begin[w];
    r.end[w] = off.end[w];
  }
  return r;
}

__global__ void fill_indicator_kernel(float* __restrict__ Y, long ldy, long n, const RangeList rl) {
  const long total = ldy * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long w = e % ldy, j = e / ldy;
    Y[e] = (w < rl.n && j >= rl.begin[w] && j < rl.end[w]) ? 1.f : 0.f;
  }
}

// One thread per (row i, range w): rows are contiguous in memory, so a warp
// reads 32 consecutive elements of each column of the range.
template <typename T>
__global__ void range_sums_kernel(const T* __restrict__ Z, long ldz, long m, const RangeList rl,
                                  double* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int w = blockIdx.y;
  if (i >= m) return;
  double s0 = 0, s1 = 0;
  long j = rl.begin[w];
  for (; j + 1 < rl.end[w]; j += 2) {
    s0 += (double)Z[j * ldz + i];
    s1 += (double)Z[(j + 1) * ldz + i];
  }
  if (j < rl.end[w]) s0 += (double)Z[j * ldz + i];
  out[(long)w * m + i] = s0 + s1;
}

__global__ void mul_small_left_kernel(const double* __restrict__ S, int k,
                                      const float* __restrict__ Y, long ldy, long n,
                                      double* __restrict__ Y2) {
  __shared__ double sS[kMaxOffsetRanges * kMaxOffsetRanges];
  for (int t = threadIdx.x; t < k * k; t += blockDim.x) sS[t] = S[t];
  __syncthreads();
  const long j = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (j >= n) return;
  double y[kMaxOffsetRanges];
  for (int w = 0; w < k; ++w) y[w] = (double)Y[j * ldy + w];
  for (int v = 0; v < k; ++v) {
    double a = 0;
    for (int w = 0; w < k; ++w) a = fma(sS[w * k + v], y[w], a);
    Y2[j * k + v] = a;
  }
}

// 256 rows per block, 64 columns per block; ZU(i, :) stays in registers.
// KMAX >= k bounds the unrolled range loops (registers for ZU's row).
template <int KMAX>
__global__ void woodbury_kernel(const float* __restrict__ Z, long ldz, long m, long n,
                                const double* __restrict__ ZU, int k,
                                const double* __restrict__ Y2, double* __restrict__ R, long ldr,
                                int accumulate) {
  // the block's 64 columns of Y2 (k values each) in shared memory, read as
  // broadcasts; four columns' Z values in flight per thread
  __shared__ double ys[64 * KMAX];
  const long j0 = (long)blockIdx.y * 64;
  const long j1 = min(n, j0 + 64);
  for (int t = threadIdx.x; t < (int)(j1 - j0) * k; t += blockDim.x) ys[t] = Y2[j0 * k + t];
  __syncthreads();
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= m) return;
  double zu[KMAX];
#pragma unroll
  for (int w = 0; w < KMAX; ++w) zu[w] = w < k ? ZU[(long)w * m + i] : 0.0;
  for (long j = j0; j < j1; j += 4) {
    float zv[4];
    double rv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      zv[q] = j + q < j1 ? Z[(j + q) * ldz + i] : 0.f;
      rv[q] = (accumulate && j + q < j1) ? R[(j + q) * ldr + i] : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (j + q >= j1) break;
      const double* y = ys + (j + q - j0) * k;
      double a = (double)zv[q];
#pragma unroll
      for (int w = 0; w < KMAX; ++w)
        if (w < k) a = fma(-zu[w], y[w], a);
      R[(j + q) * ldr + i] = rv[q] + a;
    }
  }
}

__global__ void fill_range_ids_kernel(int* __restrict__ rid, long n, const RangeList rl) {
  for (long j = blockIdx.x * (long)blockDim.x + threadIdx.x; j < n; j += (long)gridDim.x * blockDim.x) {
    int w = -1;
    for (int r = 0; r < rl.n; ++r)
      if (j >= rl.begin[r] && j < rl.end[r]) w = r;
    rid[j] = w;
  }
}

// S^-1 for S = diag(1 / value) + YU (k x k, k <= 32), by Gauss-Jordan elimination
// with partial pivoting in one block; Sinv column-major. *bad = 1 if singular.
__global__ void capacitance_inverse_kernel(const double* __restrict__ YU, int k,
                                           const OffsetValues ov, double* __restrict__ Sinv,
                                           int* bad) {
  __shared__ double a[kMaxOffsetRanges][2 * kMaxOffsetRanges + 1];
  __shared__ int piv;
  const int t = threadIdx.x;  // one thread per column of [S | I]
  for (int r = 0; r < k; ++r) {
    if (t < k) a[r][t] = YU[(long)t * k + r] + (r == t ? 1.0 / ov.v[r] : 0.0);
    else if (t < 2 * k) a[r][t] = (r == t - k) ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int c = 0; c < k; ++c) {
    if (t == 0) {
      int p = c;
      for (int r = c + 1; r < k; ++r)
        if (fabs(a[r][c]) > fabs(a[p][c])) p = r;
      piv = p;
      if (!(fabs(a[p][c]) > 0)) *bad = 1;
    }
    __syncthreads();
    if (t < 2 * k && piv != c) {
      const double x = a[piv][t];
      a[piv][t] = a[c][t];
      a[c][t] = x;
    }
    __syncthreads();
    const double d = a[c][c];
    __syncthreads();
    if (t < 2 * k) a[c][t] /= d;
    __syncthreads();
    for (int r = 0; r < k; ++r) {
      if (r == c) continue;
      const double f = a[r][c];
      __syncthreads();
      if (t < 2 * k) a[r][t] -= f * a[c][t];
      __syncthreads();
    }
  }
  if (t < k)
    for (int r = 0; r < k; ++r) Sinv[(long)t * k + r] = a[r][k + t];
}

__global__ void subtract_offset_kernel(double* __restrict__ E, long lde, long m, long n,
                                       const double* __restrict__ RU,
                                       const int* __restrict__ rid, const OffsetValues ov) {
  const long total = m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    const int w = rid[j];
    if (w >= 0) E[j * lde + i] -= RU[(long)w * m + i] * ov.v[w];
  }
}

}  // namespace

moao_status cvt_lower_minus_offsets(const double* s, long lds, float* d, long ldd, long n,
                                    const int* rid, const OffsetRanges& off, cudaStream_t st) {
  if (n <= 0) return MOAO_OK;
  cvt_lower_minus_kernel<<<blocks_for(n * n), 256, 0, st>>>(s, lds, d, ldd, n,
                                                            off.n ? rid : nullptr, values_of(off));
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status fill_range_indicators(float* Y, long ldy, long n, const OffsetRanges& off,
                                  cudaStream_t st) {
  if (n <= 0) return MOAO_OK;
  fill_indicator_kernel<<<blocks_for(ldy * n), 256, 0, st>>>(Y, ldy, n, ranges_of(off));
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

template <typename T>
static moao_status range_sums_impl(const T* Z, long ldz, long m, const OffsetRanges& off,
                                   double* out, cudaStream_t st) {
  if (m <= 0 || off.n <= 0) return MOAO_OK;
  dim3 grid((unsigned)((m + 255) / 256), (unsigned)off.n);
  range_sums_kernel<T><<<grid, 256, 0, st>>>(Z, ldz, m, ranges_of(off), out);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status range_sums(const float* Z, long ldz, long m, const OffsetRanges& off, double* out,
                       cudaStream_t st) {
  return range_sums_impl(Z, ldz, m, off, out, st);
}

moao_status range_sums(const double* Z, long ldz, long m, const OffsetRanges& off, double* out,
                       cudaStream_t st) {
  return range_sums_impl(Z, ldz, m, off, out, st);
}

moao_status mul_small_left(const double* S, int k, const float* Y, long ldy, long n, double* Y2,
                           cudaStream_t st) {
  if (n <= 0 || k <= 0) return MOAO_OK;
  if (k > kMaxOffsetRanges) return set_error(MOAO_ERR_BAD_ARG, "mul_small_left: k");
  mul_small_left_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(S, k, Y, ldy, n, Y2);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status woodbury_apply(const float* Z, long ldz, long m, long n, const double* ZU, int k,
                           const double* Y2, double* R, long ldr, bool accumulate,
                           cudaStream_t st) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  if (k < 1 || k > kMaxOffsetRanges) return set_error(MOAO_ERR_BAD_ARG, "woodbury_apply: k");
  dim3 grid((unsigned)((m + 255) / 256), (unsigned)((n + 63) / 64));
  const int acc = accumulate ? 1 : 0;
  static_assert(kMaxOffsetRanges <= 32, "woodbury_kernel instantiations");
  if (k <= 8) woodbury_kernel<8><<<grid, 256, 0, st>>>(Z, ldz, m, n, ZU, k, Y2, R, ldr, acc);
  else if (k <= 16) woodbury_kernel<16><<<grid, 256, 0, st>>>(Z, ldz, m, n, ZU, k, Y2, R, ldr, acc);
  else woodbury_kernel<32><<<grid, 256, 0, st>>>(Z, ldz, m, n, ZU, k, Y2, R, ldr, acc);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status fill_range_ids(int* rid, long n, const OffsetRanges& off, cudaStream_t st) {
  if (n <= 0) return MOAO_OK;
  fill_range_ids_kernel<<<blocks_for(n), 256, 0, st>>>(rid, n, ranges_of(off));
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status capacitance_inverse(const double* YU, const OffsetRanges& off, double* Sinv, int* bad,
                                cudaStream_t st) {
  if (off.n <= 0) return MOAO_OK;
  capacitance_inverse_kernel<<<1, 2 * kMaxOffsetRanges, 0, st>>>(YU, off.n, values_of(off), Sinv,
                                                                 bad);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status subtract_offset_products(double* E, long lde, long m, long n, const double* RU,
                                     const int* rid, const OffsetRanges& off, cudaStream_t st) {
  if (m <= 0 || n <= 0 || off.n <= 0) return MOAO_OK;
  subtract_offset_kernel<<<blocks_for(m * n), 256, 0, st>>>(E, lde, m, n, RU, rid,
                                                            values_of(off));
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status cvt_f32_to_f64(const float* s, long lds, double* d, long ldd, long m, long n,
                           bool lower, cudaStream_t st) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  cvt_f32_f64_kernel<<<blocks_for(m * n), 256, 0, st>>>(s, lds, d, ldd, m, n, lower);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status cvt_f64_to_f32(const double* s, long lds, float* d, long ldd, long m, long n,
                           bool lower, cudaStream_t st) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  cvt_f64_f32_kernel<<<blocks_for(m * n), 256, 0, st>>>(s, lds, d, ldd, m, n, lower);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status add_f32_to_f64(const float* s, long lds, double* d, long ldd, long m, long n,
                           cudaStream_t st) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  add_f32_to_f64_kernel<<<blocks_for(m * n), 256, 0, st>>>(s, lds, d, ldd, m, n);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status split_bf16(const double* src, long lds, long m, long n, int ns, BfSlices rmaj,
                       long ldr, BfSlices cmaj, long ldc, cudaStream_t st) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  if (ns < 1 || ns > kMaxBfSlices) return set_error(MOAO_ERR_BAD_ARG, "split_bf16: slices");
  dim3 grid((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
  split_bf16_kernel<<<grid, dim3(32, 8), 0, st>>>(src, lds, m, n, ns, rmaj, ldr, cmaj, ldc);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

template <typename T>
moao_status scale_exponents_t(const T* A, long lda, long m, long n, int bias, int* erow,
                              int* ecol, cudaStream_t st) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  if (erow) {
    row_exponent_kernel<T><<<(unsigned)((m + 31) / 32), dim3(32, 32), 0, st>>>(A, lda, m, n, erow,
                                                                              bias);
    ++tl_launches;
  }
  if (ecol) {
    col_exponent_kernel<T><<<(unsigned)n, 256, 0, st>>>(A, lda, m, n, ecol, bias);
    ++tl_launches;
  }
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

template <typename T>
moao_status split_f16_t(const T* src, long lds, long m, long n, int ns, BfSlices rmaj, long ldr,
                        const int* erow, BfSlices cmaj, long ldc, const int* ecol, cudaStream_t st) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  if (ns < 1 || ns > kMaxBfSlices) return set_error(MOAO_ERR_BAD_ARG, "split_f16: slices");
  if ((rmaj.p[0] && !erow) || (cmaj.p[0] && !ecol))
    return set_error(MOAO_ERR_BAD_ARG, "split_f16: exponents missing");
  dim3 grid((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
  split_f16_kernel<T><<<grid, dim3(32, 8), 0, st>>>(src, lds, m, n, ns, rmaj, ldr, erow, cmaj, ldc,
                                                    ecol);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status scale_exponents(const double* A, long lda, long m, long n, int bias, int* erow,
                            int* ecol, cudaStream_t st) {
  return scale_exponents_t(A, lda, m, n, bias, erow, ecol, st);
}
moao_status scale_exponents(const float* A, long lda, long m, long n, int bias, int* erow,
                            int* ecol, cudaStream_t st) {
  return scale_exponents_t(A, lda, m, n, bias, erow, ecol, st);
}

moao_status split_f16(const double* src, long lds, long m, long n, int ns, BfSlices rmaj,
                      long ldr, const int* erow, BfSlices cmaj, long ldc, const int* ecol,
                      cudaStream_t st) {
  return split_f16_t(src, lds, m, n, ns, rmaj, ldr, erow, cmaj, ldc, ecol, st);
}
moao_status split_f16(const float* src, long lds, long m, long n, int ns, BfSlices rmaj,
                      long ldr, const int* erow, BfSlices cmaj, long ldc, const int* ecol,
                      cudaStream_t st) {
  return split_f16_t(src, lds, m, n, ns, rmaj, ldr, erow, cmaj, ldc, ecol, st);
}

moao_status split_rows_f16(const float* src, long lds, long m, long kb, int ns, BfSlices out,
                           long ldx, long kpad, int* erow, int bias, cudaStream_t st) {
  if (m <= 0 || kb <= 0) return MOAO_OK;
  if (ns < 1 || ns > kMaxBfSlices) return set_error(MOAO_ERR_BAD_ARG, "split_rows_f16: slices");
  if (kb > kSplitMaxCols || kpad < kb || kpad > ldx || (kpad & 1) || (ldx & 1))
    return set_error(MOAO_ERR_BAD_ARG, "split_rows_f16: block shape");
  // row exponents, then the split through 32 x 64 tiles (the block stays in L2
  // between the two passes)
  row_exponent_kernel<float><<<(unsigned)((m + 31) / 32), dim3(32, 8), 0, st>>>(src, lds, m, kb,
                                                                              erow, bias);
  ++tl_launches;
  const dim3 grid((unsigned)((m + 31) / 32), (unsigned)((kpad + 63) / 64));
  split_rows_f16_t_kernel<<<grid, dim3(32, 8), 0, st>>>(src, lds, m, (int)kb, ns, out, ldx,
                                                        (int)kpad, erow);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status ozaki_split_rows(const double* A, long lda, long m, long n, int ns, int* e,
                             int8_t* out, long ldo, cudaStream_t st) {
  if (ns < 1 || ns > kMaxOzakiSlices) return set_error(MOAO_ERR_BAD_ARG, "ozaki: slices");
  row_exponent_kernel<double><<<(unsigned)((m + 31) / 32), dim3(32, 8), 0, st>>>(A, lda, m, n, e, 0);
  ++tl_launches;
  dim3 grid((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
  split_rows_i8_kernel<<<grid, dim3(32, 8), 0, st>>>(A, lda, m, n, e, ns, out, ldo, m * ldo);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status ozaki_split_sym(const double* A, long lda, long n, int ns, int* f,
                            unsigned long long* colmax, int8_t* out, long ldo, const int* rid,
                            const OffsetRanges& off, cudaStream_t st) {
  if (ns < 1 || ns > kMaxOzakiSlices) return set_error(MOAO_ERR_BAD_ARG, "ozaki: slices");
  if ((ldo & 3) || (reinterpret_cast<uintptr_t>(out) & 3))
    return set_error(MOAO_ERR_BAD_ARG, "ozaki: slice rows must be 4-byte aligned");
  MOAO_CUDA_TRY(cudaMemsetAsync(colmax, 0, n * sizeof(unsigned long long), st));
  const int* r = off.n ? rid : nullptr;
  const OffsetValues ov = values_of(off);
  dim3 grid((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
  sym_col_max_kernel<<<grid, dim3(32, 8), 0, st>>>(A, lda, n, colmax, r, ov);
  ++tl_launches;
  exponents_from_max_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(colmax, n, f);
  ++tl_launches;
  split_sym_i8_kernel<<<grid, dim3(32, 8), 0, st>>>(A, lda, n, f, ns, out, ldo, n * ldo, r, ov);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}


int crt_moduli_for(int ns, long K) {
  if (ns < 1 || ns > kMaxOzakiSlices || K < 1 || K >= (1L << 17)) return 0;
  // |product| <= K 2^(2 (7 ns - 1)); exact while it stays below M / 2
  const double need = std::log2((double)K) + 2.0 * (7 * ns - 1) + 1.0;
  double have = 0;
  for (int i = 0; i < kCrtMaxModuli; ++i) {
    have += std::log2((double)kCrtMod[i]);
    if (have > need + 1e-9) return i + 1;
  }
  return 0;
}

moao_status crt_split_rows(const double* A, long lda, long m, long n, int ns, int nmod,
                           const int* e, int8_t* out, long ldo, cudaStream_t st) {
  if (ns < 1 || ns > kMaxOzakiSlices || nmod < 2 || nmod > kCrtMaxModuli)
    return set_error(MOAO_ERR_BAD_ARG, "crt: slices or moduli");
  dim3 grid((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
  crt_rows_kernel<<<grid, dim3(32, 8), 0, st>>>(A, lda, m, n, e, 7 * ns - 1, nmod, out, ldo,
                                                 m * ldo);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status crt_split_sym(const double* A, long lda, long n, int ns, int nmod, int* f,
                          unsigned long long* colmax, int8_t* out, long ldo, const int* rid,
                          const OffsetRanges& off, cudaStream_t st) {
  if (ns < 1 || ns > kMaxOzakiSlices || nmod < 2 || nmod > kCrtMaxModuli)
    return set_error(MOAO_ERR_BAD_ARG, "crt: slices or moduli");
  if ((ldo & 3) || (reinterpret_cast<uintptr_t>(out) & 3))
    return set_error(MOAO_ERR_BAD_ARG, "crt: residue rows must be 4-byte aligned");
  MOAO_CUDA_TRY(cudaMemsetAsync(colmax, 0, n * sizeof(unsigned long long), st));
  const int* r = off.n ? rid : nullptr;
  const OffsetValues ov = values_of(off);
  dim3 grid((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32));
  sym_col_max_kernel<<<grid, dim3(32, 8), 0, st>>>(A, lda, n, colmax, r, ov);
  ++tl_launches;
  exponents_from_max_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(colmax, n, f);
  ++tl_launches;
  const long nt = (n + 31) / 32;
  crt_sym_kernel<<<(unsigned)(nt * (nt + 1) / 2), dim3(32, 8), 0, st>>>(
      A, lda, n, f, 7 * ns - 1, nmod, out, ldo, n * ldo, r, ov);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status crt_combine(const uint8_t* Z, long m, long n, int nmod, int ns, const int* e,
                        const int* f, const double* C, long ldc, double alpha, double* E,
                        long lde, cudaStream_t st) {
  if (nmod < 2 || nmod > kCrtMaxModuli) return set_error(MOAO_ERR_BAD_ARG, "crt: moduli");
  if (m <= 0 || n <= 0) return MOAO_OK;
  if ((m + 255) / 256 > 65535) return set_error(MOAO_ERR_BAD_ARG, "crt: too many rows");
  const dim3 grid((unsigned)n, (unsigned)((m + 255) / 256));
  crt_combine_kernel<<<grid, 256, 0, st>>>(Z, m, m * n, nmod, 7 * ns - 1, e, f, C, ldc, alpha, E,
                                           lde);
  ++tl_launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

}  // namespace moao
