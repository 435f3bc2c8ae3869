// FP64 dense kernels for the plain-FP64 reconstructor path.
//
// Blackwell has no FP64 kind for tcgen05.mma, so FP64 contractions run on the
// FP64 DMMA path (mma.sync m16n8k16 .f64), fed by a 4-stage cp.async pipeline of
// 128x64x16 (or 64x64x16) tiles in shared memory (bank-conflict-free padded
// layouts). One kernel template serves every contraction of the path:
//   trailing SYRK of the tiled Cholesky   (transB, lowerC)
//   panel TRSM as a product with the inverse diagonal block
//   the two triangular solves of R        (NN / NT)
//   SYR2K / SYMM / GEMM of the Cee/Cvv chain (triB masks a lower-stored
//   symmetric operand; no symmetric copy is ever materialised)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>

#include "dense.h"
#include "leaf_f64.cuh"

namespace moao {
namespace {

constexpr int PAD_MN = 4;  // doubles of padding on m/n-contiguous rows
constexpr int PAD_K = 4;   // doubles of padding on k-contiguous rows

// CTA tile BM x BN; each warp computes WM x 32 (warps: BM/WM along m, BN/32
// along n). 128x64 (8 warps of 32x32, ~120 registers, two CTAs per SM so one
// CTA's prologue and C epilogue overlap the other's DMMA loop) for large
// products: 26.2 TF/s on the ELT FP64 build against 21.4 for 128x128 tiles with
// one CTA per SM and 24.4 for 128x64 with 4 warps of 64x32. 64x64 (4 warps of
// 32x32) when even that would leave most SMs idle (the small products of the
// diagonal-block recursion). BK (K per pipeline stage, a multiple of 16) and
// STAGES (the cp.async ring) are the other dimensions a configuration sets
// (GemmArgs::cfg, chosen per context: moao_ctx_set_gemm_tile / the autotuner).
template <int BM_, int BN_, int WM_, int BK_ = 16, int STAGES_ = 4>
struct Tile {
  static constexpr int BM = BM_, BN = BN_, WM = WM_, BK = BK_, STAGES = STAGES_;
  static constexpr int WARPS_M = BM / WM, WARPS_N = BN / 32;
  static constexpr int NTHREADS = 32 * WARPS_M * WARPS_N;
  static constexpr int MF = WM / 8;             // 8-row fragments per warp
  static constexpr int LDA_S = BM + PAD_MN;     // As[k][m]
  static constexpr int LDB_S = BN + PAD_MN;     // Bs[k][n]   (transB)
  static constexpr int LDBT_S = BK + PAD_K;     // Bs[n][k]   (!transB)
  static constexpr int A_STAGE = BK * LDA_S;
  static constexpr int B_STAGE = (BK * LDB_S > BN * LDBT_S) ? BK * LDB_S : BN * LDBT_S;
  static constexpr size_t SMEM_BYTES = (size_t)STAGES * (A_STAGE + B_STAGE) * sizeof(double);
};
using TileL = Tile<128, 64, 32>;
using TileS = Tile<64, 64, 32>;
// alternative large-product configurations (GemmArgs::cfg 1..3)
using TileL32x2 = Tile<128, 64, 32, 32, 2>;   // 102 KB: two CTAs per SM, two k16 steps per barrier
using TileL32x3 = Tile<128, 64, 32, 32, 3>;   // 154 KB: one CTA per SM
using TileL16x6 = Tile<128, 64, 32, 16, 6>;   // 154 KB: one CTA per SM, deeper ring

__device__ __forceinline__ void cp_async(double* smem, const double* gmem, int vec, int valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int bytes = valid * 8;
  if (vec == 2) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(bytes));
  } else {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(bytes));
  }
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

// m16n8k16 FP64 MMA: A 16x16 (8 per thread: rows gid, gid+8; cols tig + 4r),
// B 16x8 (4 per thread: rows tig + 4r, col gid), C 16x8 (rows gid, gid+8;
// cols 2 tig, 2 tig + 1).
__device__ __forceinline__ void dmma16(double& c0, double& c1, double& c2, double& c3,
                                       const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

struct KParams {
  long M, N, K;
  double alpha, beta;
  const double* A;
  long lda;
  const double* B;
  long ldb;
  double* C;
  long ldc;
  int triB;
  // tile order (set by the launcher): bands of group_m row tiles; inside a band
  // the column tiles in turn, the band's row tiles fastest
  int tiles_m, tiles_n, group_m;
};

// Tile v of the launch in band order. Consecutive CTAs share one column strip
// of B and the band's row strips of A stay in L2 while the band sweeps the
// columns: the CTAs resident together touch group_m strips of A and a few of B
// instead of every row strip of A (which, for a 1,024-wide panel of an
// nmeas ~ 15k-48k factorisation, no longer fits in L2). For a lower C the sweep
// of a band stops at the diagonal. Returns false past the last tile.
template <int BM, int BN, bool LOWERC>
__device__ __forceinline__ bool band_tile(const KParams& p, long v, long* m0, long* n0) {
  for (int b0 = 0; b0 < p.tiles_m; b0 += p.group_m) {
    const int rows = min(p.group_m, p.tiles_m - b0);
    long cols = p.tiles_n;
    if (LOWERC) cols = min((long)p.tiles_n, ((long)(b0 + rows) * BM - 1) / BN + 1);
    const long cnt = rows * cols;
    if (v < cnt) {
      *m0 = (long)(b0 + (int)(v % rows)) * BM;
      *n0 = (v / rows) * BN;
      return true;
    }
    v -= cnt;
  }
  return false;
}

// Load one BK-slice of an MN-contiguous operand (A, or B when transB): the tile
// rows r0..r0+R-1 of columns k0..k0+15 of a column-major rows x K matrix, stored
// with row stride LDS (R = BM, LDS = LDA_S for A; R = BN, LDS = LDB_S for B).
template <class TL, int VEC, int R, int LDS>
__device__ __forceinline__ void load_mn_tile(double* s, const double* g, long ld, long rows,
                                             long K, long r0, long k0) {
  constexpr int CH = R / VEC;                // chunks per k column
  constexpr int TOTAL = CH * TL::BK;
  for (int c = threadIdx.x; c < TOTAL; c += TL::NTHREADS) {
    const int kk = c / CH, rr = (c % CH) * VEC;
    const long gr = r0 + rr, gk = k0 + kk;
    int valid = 0;
    if (gk < K && gr < rows) valid = (int)min((long)VEC, rows - gr);
    const double* src = valid ? g + gk * ld + gr : g;
    cp_async(s + kk * LDS + rr, src, VEC, valid);
  }
}

// Load one BK-slice of a K-contiguous operand (B when !transB): rows k0..k0+15
// of columns n0..n0+BN-1 of a column-major K x N matrix, stored Bs[n][k].
template <class TL, int VEC>
__device__ __forceinline__ void load_k_tile(double* s, const double* g, long ld, long N,
                                            long K, long n0, long k0) {
  constexpr int CH = TL::BK / VEC;
  constexpr int TOTAL = CH * TL::BN;
  for (int c = threadIdx.x; c < TOTAL; c += TL::NTHREADS) {
    const int nn = c / CH, kk = (c % CH) * VEC;
    const long gn = n0 + nn, gk = k0 + kk;
    int valid = 0;
    if (gn < N && gk < K) valid = (int)min((long)VEC, K - gk);
    const double* src = valid ? g + gn * ld + gk : g;
    cp_async(s + nn * TL::LDBT_S + kk, src, VEC, valid);
  }
}

template <class TL, bool TRANSB, bool LOWERC, int VEC, bool MMA16>
__global__ void __launch_bounds__(TL::NTHREADS) gemm_f64_kernel(const KParams p) {
  constexpr int BM = TL::BM, BN = TL::BN, NTHREADS = TL::NTHREADS, MF = TL::MF;
  constexpr int BK = TL::BK, STAGES = TL::STAGES;
  constexpr int LDA_S = TL::LDA_S, LDB_S = TL::LDB_S, LDBT_S = TL::LDBT_S;
  constexpr int A_STAGE = TL::A_STAGE, B_STAGE = TL::B_STAGE;
  extern __shared__ __align__(16) double smem[];
  double* As = smem;
  double* Bs = smem + STAGES * A_STAGE;

  long m0 = 0, n0 = 0;
  if (!band_tile<BM, BN, LOWERC>(p, blockIdx.x, &m0, &n0)) return;
  if (LOWERC && m0 + BM <= n0) return;  // tile strictly above the diagonal

  // K range (tile aligned); a triangular B limits it.
  long kb = 0, ke = p.K;
  if (p.triB != 0) {
    if (!TRANSB) kb = n0;                      // B(k, n) with k >= n
    else ke = min(p.K, n0 + BN);               // B(n, k) with n >= k
  }
  kb = (kb / BK) * BK;
  const int ntiles = (ke > kb) ? (int)((ke - kb + BK - 1) / BK) : 0;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp % TL::WARPS_M) * TL::WM, wn = (warp / TL::WARPS_M) * 32;
  const int gid = lane >> 2, tig = lane & 3;

  // acc[i][j][h]: k4 layout = MF m-frags of 8 rows x 4 n-frags x 2;
  // k16 layout = MF/2 m-frags of 16 rows x 4 n-frags x 4.
  double acc[MF][4][2];
#pragma unroll
  for (int i = 0; i < MF; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  auto issue = [&](int stage, int t) {
    const long k0 = kb + (long)t * BK;
    load_mn_tile<TL, VEC, BM, LDA_S>(As + stage * A_STAGE, p.A, p.lda, p.M, p.K, m0, k0);
    if (TRANSB)
      load_mn_tile<TL, VEC, BN, LDB_S>(Bs + stage * B_STAGE, p.B, p.ldb, p.N, p.K, n0, k0);
    else load_k_tile<TL, VEC>(Bs + stage * B_STAGE, p.B, p.ldb, p.N, p.K, n0, k0);
  };

#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ntiles) issue(s, s);
    cp_commit();
  }

  for (int t = 0; t < ntiles; ++t) {
    cp_wait<STAGES - 2>();
    __syncthreads();
    const int stage = t % STAGES;
    double* as = As + stage * A_STAGE;
    double* bs = Bs + stage * B_STAGE;
    if (p.triB != 0) {
      // Zero the entries of the stored B outside its lower (or strictly lower)
      // triangle when this slice crosses the diagonal.
      const long k0 = kb + (long)t * BK;
      const bool crosses = TRANSB ? (k0 + BK - 1 >= n0) : (k0 <= n0 + BN - 1);
      if (crosses) {
        for (int e = threadIdx.x; e < BK * BN; e += NTHREADS) {
          const int kk = e / BN, nn = e % BN;
          const long gk = k0 + kk, gn = n0 + nn;
          // stored row / column of this element
          const long row = TRANSB ? gn : gk, col = TRANSB ? gk : gn;
          const bool keep = (p.triB == 1) ? (row >= col) : (row > col);
          if (!keep) {
            if (TRANSB) bs[kk * LDB_S + nn] = 0.0;
            else bs[nn * LDBT_S + kk] = 0.0;
          }
        }
        __syncthreads();
      }
    }
    {
      const int nt = t + STAGES - 1;
      if (nt < ntiles) issue(nt % STAGES, nt);
      cp_commit();
    }
    if (MMA16) {
#pragma unroll
      for (int k16 = 0; k16 < BK; k16 += 16) {
        double bf[4][4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int r = 0; r < 4; ++r) {
            const int k = k16 + r * 4 + tig, n = wn + j * 8 + gid;
            bf[j][r] = TRANSB ? bs[k * LDB_S + n] : bs[n * LDBT_S + k];
          }
#pragma unroll
        for (int i = 0; i < MF / 2; ++i) {
          double af[8];
#pragma unroll
          for (int r = 0; r < 8; ++r)
            af[r] = as[(k16 + (r >> 1) * 4 + tig) * LDA_S + wm + i * 16 + gid + 8 * (r & 1)];
#pragma unroll
          for (int j = 0; j < 4; ++j)
            dmma16(acc[2 * i][j][0], acc[2 * i][j][1], acc[2 * i + 1][j][0], acc[2 * i + 1][j][1],
                   af, bf[j]);
        }
      }
    } else {
#pragma unroll
      for (int k4 = 0; k4 < BK; k4 += 4) {
        double a[MF], b[4];
#pragma unroll
        for (int i = 0; i < MF; ++i) a[i] = as[(k4 + tig) * LDA_S + wm + i * 8 + gid];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          if (TRANSB) b[j] = bs[(k4 + tig) * LDB_S + wn + j * 8 + gid];
          else b[j] = bs[(wn + j * 8 + gid) * LDBT_S + k4 + tig];
        }
#pragma unroll
        for (int i = 0; i < MF; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
    }
  }
  cp_wait<0>();

  // Epilogue through shared memory (the operand ring is free now): the C tile
  // is read with coalesced loads, all in flight (only when beta != 0), each
  // thread combines its accumulators with it in place, and the tile goes back
  // with coalesced stores, lower part only for a lower C. Leading dimension
  // BM + 2 keeps the fragment accesses free of bank conflicts.
  // k4: fragment i covers rows wm + 8 i; k16: acc[2q][j] and acc[2q+1][j] hold
  // the 4 values of m16 fragment q (rows wm + 16 q + gid and + 8).
  constexpr int LDC_S = BM + 2;
  static_assert((size_t)BN * LDC_S * sizeof(double) <= TL::SMEM_BYTES, "C tile exceeds the ring");
  __syncthreads();
  double* Cs = smem;
  const bool read_c = p.beta != 0.0;
  for (int e = threadIdx.x; e < BM * BN; e += NTHREADS) {
    const int rr = e % BM, cc = e / BM;
    const long r = m0 + rr, c = n0 + cc;
    Cs[cc * LDC_S + rr] = (read_c && r < p.M && c < p.N) ? p.C[c * p.ldc + r] : 0.0;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < MF; ++i) {
    const int rr = MMA16 ? wm + (i >> 1) * 16 + (i & 1) * 8 + gid : wm + i * 8 + gid;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int cc = wn + j * 8 + 2 * tig + h;
        double* d = Cs + cc * LDC_S + rr;
        *d = read_c ? p.alpha * acc[i][j][h] + p.beta * *d : p.alpha * acc[i][j][h];
      }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < BM * BN; e += NTHREADS) {
    const int rr = e % BM, cc = e / BM;
    const long r = m0 + rr, c = n0 + cc;
    if (r < p.M && c < p.N && !(LOWERC && r < c)) p.C[c * p.ldc + r] = Cs[cc * LDC_S + rr];
  }
}

// FP64 MMA shape: m16n8k16 unless MOAO_GEMM_MMA=k4 selects m8n8k4.
bool use_mma16() {
  static const bool v = [] {
    const char* e = getenv("MOAO_GEMM_MMA");
    return !(e && e[0] == 'k' && e[1] == '4');
  }();
  return v;
}

template <class TL, bool TRANSB, bool LOWERC, int VEC, bool MMA16>
moao_status launch_gemm_t(const KParams& p, cudaStream_t s) {
  static std::atomic<unsigned long long> configured{0};
  auto kern = gemm_f64_kernel<TL, TRANSB, LOWERC, VEC, MMA16>;
  MOAO_CUDA_TRY(set_smem_limit(kern, (int)TL::SMEM_BYTES, configured));
  KParams q = p;
  q.tiles_m = (int)((p.M + TL::BM - 1) / TL::BM);
  q.tiles_n = (int)((p.N + TL::BN - 1) / TL::BN);
  q.group_m = std::max(1, 4096 / TL::BM);  // bands of 4,096 rows
  long total = 0;
  for (int b0 = 0; b0 < q.tiles_m; b0 += q.group_m) {
    const int rows = std::min(q.group_m, q.tiles_m - b0);
    long cols = q.tiles_n;
    if (LOWERC) cols = std::min((long)q.tiles_n, ((long)(b0 + rows) * TL::BM - 1) / TL::BN + 1);
    total += rows * cols;
  }
  if (total <= 0) return MOAO_OK;
  if (total > 0x7fffffffL) return set_error(MOAO_ERR_BAD_ARG, "gemm: too many tiles");
  kern<<<(unsigned)total, TL::NTHREADS, TL::SMEM_BYTES, s>>>(q);
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

// Products whose 128x128-tile count would fill fewer than two waves of the 148
// SMs take the 64x64 tiles (twice the CTAs of the 128x64 ones).
bool small_tiles(const KParams& p) {
  const long tiles = ((p.M + 127) / 128) * ((p.N + 127) / 128);
  return tiles < 2 * 148;
}

template <bool TRANSB, bool LOWERC, int VEC>
moao_status launch_gemm(const KParams& p, int cfg, cudaStream_t s) {
  if (small_tiles(p))
    return use_mma16() ? launch_gemm_t<TileS, TRANSB, LOWERC, VEC, true>(p, s)
                       : launch_gemm_t<TileS, TRANSB, LOWERC, VEC, false>(p, s);
  switch (cfg) {
    case 1: return launch_gemm_t<TileL32x2, TRANSB, LOWERC, VEC, true>(p, s);
    case 2: return launch_gemm_t<TileL32x3, TRANSB, LOWERC, VEC, true>(p, s);
    case 3: return launch_gemm_t<TileL16x6, TRANSB, LOWERC, VEC, true>(p, s);
    default: break;
  }
  return use_mma16() ? launch_gemm_t<TileL, TRANSB, LOWERC, VEC, true>(p, s)
                     : launch_gemm_t<TileL, TRANSB, LOWERC, VEC, false>(p, s);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Leaf kernel of the blocked factorisation (leaf_factor_inverse, one CTA).
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1) potrf_inv_leaf_kernel(double* A, long lda,
                                                                    double* Linv, long ldi, int n,
                                                                    long col0, int* info) {
  extern __shared__ __align__(16) double leaf_smem[];
  leaf_factor_inverse<THREADS>(A, lda, Linv, ldi, n, col0, info, leaf_smem);
}

// The leaf CTA has 1,024 threads (two or three triangle elements each): 54 us
// per 64 x 64 block against 66 us with 512 and 91 us with 256 threads (B200,
// CUDA events over the leaves of an nmeas 15,936 FP64 build).
constexpr int kLeafThreads = 1024;

__global__ void copy_kernel(const double* __restrict__ src, long lds, double* __restrict__ dst,
                            long ldd, long m, long n) {
  const long total = m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    dst[j * ldd + i] = src[j * lds + i];
  }
}

__global__ void fill_kernel(double* A, long lda, long m, long n, double v) {
  const long total = m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    A[j * lda + i] = v;
  }
}

// Cee(i, j) = Cpp(max(i,j), min(i,j)); the diagonal goes through 2d * 0.5
// exactly like the reference's geadd + scal sequence.
__global__ void sym_from_lower_kernel(const double* __restrict__ P, long ldp,
                                      double* __restrict__ E, long lde, long n) {
  const long total = n * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total;
       e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, j = e / n;
    double v;
    if (i > j) v = P[j * ldp + i];
    else if (i < j) v = P[i * ldp + j];
    else v = (P[j * ldp + i] + P[j * ldp + i]) * 0.5;
    E[j * lde + i] = v;
  }
}

unsigned grid_for(long total) {
  long b = (total + 255) / 256;
  return (unsigned)std::max(1L, std::min(b, 148L * 16));
}

}  // namespace

moao_status gemm_f64(const GemmArgs& g, cudaStream_t s, long long* launches) {
  if (g.M < 0 || g.N < 0 || g.K < 0) return set_error(MOAO_ERR_BAD_ARG, "gemm: negative size");
  if (g.M == 0 || g.N == 0) return MOAO_OK;
  if (g.lowerC && g.triB != TRI_FULL)
    return set_error(MOAO_ERR_UNSUPPORTED, "gemm: lowerC with a triangular B");
  if (g.lda < std::max(1L, g.M) || g.ldc < std::max(1L, g.M) ||
      g.ldb < std::max(1L, g.transB ? g.N : g.K))
    return set_error(MOAO_ERR_BAD_ARG, "gemm: leading dimension too small");
  KParams p{g.M, g.N, g.K, g.alpha, g.beta, g.A, g.lda, g.B, g.ldb, g.C, g.ldc, (int)g.triB};
  if (g.K == 0) {  // C = beta C
    p.alpha = 0.0;
  }
  const bool v2 = aligned16(g.A) && aligned16(g.B) && (g.lda % 2 == 0) && (g.ldb % 2 == 0);
  moao_status st;
  const int c = g.cfg;
  if (v2) {
    if (g.transB) st = g.lowerC ? launch_gemm<true, true, 2>(p, c, s) : launch_gemm<true, false, 2>(p, c, s);
    else st = g.lowerC ? launch_gemm<false, true, 2>(p, c, s) : launch_gemm<false, false, 2>(p, c, s);
  } else {
    if (g.transB) st = g.lowerC ? launch_gemm<true, true, 1>(p, c, s) : launch_gemm<true, false, 1>(p, c, s);
    else st = g.lowerC ? launch_gemm<false, true, 1>(p, c, s) : launch_gemm<false, false, 1>(p, c, s);
  }
  if (st == MOAO_OK && launches) ++*launches;
  return st;
}

moao_status potrf_inv_leaf(double* A, long lda, double* Linv, long ldi, int n, long col0,
                           int* d_info, cudaStream_t s, long long* launches) {
  if (n <= 0) return MOAO_OK;
  if (n > LEAF) return set_error(MOAO_ERR_BAD_ARG, "potrf leaf: n > 64");
  static std::atomic<unsigned long long> configured{0};
  const int smem = LEAF_SMEM_BYTES;
  MOAO_CUDA_TRY(set_smem_limit(potrf_inv_leaf_kernel<kLeafThreads>, smem, configured));
  potrf_inv_leaf_kernel<kLeafThreads><<<1, kLeafThreads, smem, s>>>(A, lda, Linv, ldi, n, col0,
                                                                    d_info);
  if (launches) ++*launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status copy_matrix(const double* src, long lds, double* dst, long ldd, long m, long n,
                        cudaStream_t s) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  MOAO_CUDA_TRY(cudaMemcpy2DAsync(dst, ldd * sizeof(double), src, lds * sizeof(double),
                                  m * sizeof(double), n, cudaMemcpyDeviceToDevice, s));
  return MOAO_OK;
}

moao_status fill_matrix(double* A, long lda, long m, long n, double v, cudaStream_t s,
                        long long* launches) {
  if (m <= 0 || n <= 0) return MOAO_OK;
  fill_kernel<<<grid_for(m * n), 256, 0, s>>>(A, lda, m, n, v);
  if (launches) ++*launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

moao_status sym_from_lower(const double* Cpp, long ldp, double* Cee, long lde, long n,
                           cudaStream_t s, long long* launches) {
  if (n <= 0) return MOAO_OK;
  sym_from_lower_kernel<<<grid_for(n * n), 256, 0, s>>>(Cpp, ldp, Cee, lde, n);
  if (launches) ++*launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

}  // namespace moao
