// tcgen05 tensor-core GEMM for the mixed-precision path (sm_100a).
//
//   C[M x N] (+)= sum over segments s of  A_s[M x K_s] * B_s[N x K_s]^T
//
// Both operands are K-major (rows of K contiguous elements) and are fetched by
// TMA (cp.async.bulk.tensor, 128-byte swizzle, each CTA loading only its own
// tiles) into a shared-memory ring; one thread issues tcgen05.mma into a
// double-buffered TMEM accumulator;
// eight epilogue warps drain TMEM with tcgen05.ld and update C. A tile is 128 x
// 256 on one CTA, or 256 x 256 on a cluster of two CTAs (M = 256 MMAs,
// cta_group::2). The K dimension is a list of segments, each naming its own A
// and B tensor (slices) and K offset, so that a split-precision product
// (hi*hi + hi*lo + lo*hi, or the int8 slice pairs of one Ozaki diagonal)
// accumulates in one accumulator and C is read and written once.
//
// Kinds:
//   BF16 -> FP32 accumulate (kind::f16);   epilogue C32 = alpha*acc + beta*C32
//   FP16 -> FP32 accumulate (kind::f16);   epilogue C32 = alpha*acc*2^(erow[r]+ecol[c]+shift)
//           + beta*C32 (power-of-two scales of operands stored scaled into fp16 range)
//   INT8 -> INT32 accumulate (kind::i8), exact for K*64*64*pairs < 2^31;
//           epilogue C64 += acc * 2^(erow[r] + ecol[c] + shift)
// Waits on mbarriers are bounded; on expiry the kernel records an error code in
// *err and stops issuing work instead of spinning forever.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "tc_gemm.h"
#include "context.h"
#include "moao_b200_debug.h"

namespace moao {
namespace {

constexpr int TBM = 128, TBN = 256;      // accumulator of one CTA: TMEM lanes x columns
constexpr int BOX_ROWS = 128;            // rows of one TMA box (A and B operands alike)
constexpr int KBYTES = 128;              // bytes of K per stage row (one 128B swizzle atom)
constexpr int A_TILE = TBM * KBYTES;     // 16 KB
constexpr int BOX_BYTES = BOX_ROWS * KBYTES;
constexpr int EPI_WARPS = 8;             // two warps per TMEM lane quadrant
constexpr int THREADS = (4 + EPI_WARPS) * 32;
constexpr int ACC_COLS = TBN;            // fp32 / int32 columns of one accumulator
constexpr int TMEM_COLS = 2 * ACC_COLS;  // double-buffered accumulator
constexpr int STAGE_C = 32 * 32 * 4;     // per epilogue warp: one 32x32 FP32 chunk for TMA
constexpr unsigned long long kSpinLimit = 1ull << 28;  // default polls of a bounded wait
constexpr int kBandRows = 2048;          // rows of C per band of the tile order
constexpr int kMaxBands = 64;

// PAIR = 0: one CTA computes a 128 x 256 tile of C.
// PAIR = 1: a cluster of two CTAs computes a 256 x 256 tile with M = 256 MMAs
// (tcgen05.mma.cta_group::2): each CTA holds 128 rows of A and 128 rows of B in
// its shared memory and 128 rows of the accumulator in its TMEM; the first CTA
// of the pair issues the MMAs for both. Per SM a stage then carries 32 KB of
// operands instead of 48 KB for the same tensor work.
template <int PAIR>
struct TcCfg {
  static constexpr int B_ROWS = PAIR ? TBN / 2 : TBN;  // B rows held by one CTA
  static constexpr int B_TILE = B_ROWS * KBYTES;
  static constexpr int STAGE_BYTES = A_TILE + B_TILE;
  static constexpr int STAGES = PAIR ? 6 : 4;
  static constexpr int TILE_M = PAIR ? 2 * TBM : TBM;  // rows of C per tile
  static constexpr size_t SMEM = (size_t)STAGES * STAGE_BYTES + 1024 /*align*/ + 256 /*barriers*/ +
                                 EPI_WARPS * 32 * sizeof(float) /*per-warp column scales*/ +
                                 (size_t)EPI_WARPS * STAGE_C /*per-warp C staging*/;
  static_assert(SMEM <= 232448, "shared memory per CTA");
  static_assert(2 * STAGES + 5 <= 31, "barrier area");
};

struct __align__(64) TcParams {
  CUtensorMap mapA[kTcMaxMaps];
  CUtensorMap mapB[kTcMaxMaps];
  CUtensorMap mapC;        // FP32 C (rows inner) for the TMA reduce-add epilogue
  int c_tma;               // 1: C += alpha*acc*scales through cp.reduce.async.bulk.tensor
  TcSegment seg[kTcMaxSegs];
  int nseg;
  int M, N;
  int a_row0, b_row0;      // row coordinate of C(0,0) in the A / B tensors
  int lower;               // 1: only C(r, c) with r + diag_off >= c
  int diag_off;
  int kind;                // TcKind
  int epi;                 // TcEpilogue
  float alpha, beta;
  void* C;
  long long ldc;
  const int* erow;         // INT8: per-row exponent of A (length M, indexed by r)
  const int* ecol;         // INT8: per-column exponent of B (length N)
  int shift;
  int modulus;             // kTcEpiMod8
  int tile_m;              // rows of C per tile (128, or 256 for CTA pairs)
  int tiles_m, tiles_n;
  int total_tiles;         // tiles that intersect the written part of C
  int band;                // row tiles per band of the tile order
  int band_start[kMaxBands + 1];  // tiles before each band
  int* err;
  unsigned long long spin_limit;  // polls of a role's bounded wait before it gives up
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Arrive on a barrier named by its shared::cluster address (this CTA's or the
// pair's other CTA's), releasing this thread's prior accesses to the cluster.
__device__ __forceinline__ void mbar_arrive_cluster(uint32_t caddr) {
  asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];\n" ::"r"(caddr)
               : "memory");
}

// shared::cluster address of the variable at shared address saddr in CTA rank.
__device__ __forceinline__ uint32_t cluster_addr(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}

// Every thread of both CTAs of the cluster (release / acquire on shared memory).
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release;\nbarrier.cluster.wait.acquire;\n" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait; returns false (and records code) if the phase does not
// complete within limit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int code,
                                          unsigned long long limit) {
  for (unsigned long long i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((i & 1023) == 1023 && *(volatile int*)err) return false;  // another role gave up
  }
  atomicCAS(err, 0, code);
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Load into this CTA's shared memory, the bytes counted on the barrier at
// shared::cluster address bar (in either CTA of the pair).
__device__ __forceinline__ void tma_load_2d_pair(void* dst, const CUtensorMap* map, int x, int y,
                                                 uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.cta_group::2.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3}], [%4];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// C += (staged chunk) through the TMA unit: a 32-row x 32-column FP32 box at
// (row x, column y) of the C tensor map, reduced (added) into global memory.
__device__ __forceinline__ void tma_reduce_add_2d(const CUtensorMap* map, int x, int y,
                                                  const void* src) {
  asm volatile(
      "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.tile.bulk_group [%0, {%1, %2}], [%3];\n"
      ::"l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(src))
      : "memory");
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}

// Shared-memory matrix descriptor for a K-major tile written by TMA with the
// 128-byte swizzle: 8-row core groups 1024 bytes apart (SBO), LBO = 16 bytes
// (unused for swizzled K-major), descriptor version 1 (tcgen05), SWIZZLE_128B.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
  d |= (uint64_t)(16 >> 4) << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= (uint64_t)1 << 46;
  d |= (uint64_t)2 << 61;
  return d;
}

__device__ __forceinline__ void mma_f16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_i8(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(acc));
}

// M = 256 across the pair: A and B descriptors name this CTA's stage; the
// other CTA's tiles sit at the same shared-memory offsets. No output lane is
// disabled (all-zero mask).
__device__ __forceinline__ void mma_f16_pair(uint32_t tmem, uint64_t a, uint64_t b,
                                             uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::2.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n}\n"
      ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u));
}

__device__ __forceinline__ void mma_i8_pair(uint32_t tmem, uint64_t a, uint64_t b,
                                            uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::2.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5, %5, %5, %5, %5}, p;\n}\n"
      ::"r"(tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
          smem_u32(bar))
      : "memory");
}

// Arrives (once each) on the barrier at this shared offset in both CTAs of the
// pair when every MMA the thread issued before has completed.
__device__ __forceinline__ void mma_commit_pair(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::2.mbarrier::arrive::one.shared::cluster.multicast::cluster.b64 "
      "[%0], %1;\n" ::"r"(smem_u32(bar)),
      "h"((unsigned short)3)
      : "memory");
}

// Instruction descriptors (N = 256, both operands K-major; M = 128 for one
// CTA, 256 for a pair).
//   bits 4-5 D format (1 F32, 2 S32), 7-9 A format, 10-12 B format
//   (kind::f16: 1 BF16; kind::i8: 1 S8), 15/16 A/B major (0 = K),
//   17-22 N >> 3, 24-28 M >> 4.
constexpr uint32_t idesc_of(int dfmt, int abfmt, int m) {
  return (uint32_t)(dfmt << 4) | (uint32_t)(abfmt << 7) | (uint32_t)(abfmt << 10) |
         (uint32_t)((TBN >> 3) << 17) | (uint32_t)((m >> 4) << 24);
}

// First row tile of column tile nt that reaches the written (lower) part.
__device__ __forceinline__ int first_mt(const TcParams& p, int nt) {
  if (!p.lower) return 0;
  const int num = nt * TBN - p.diag_off - (p.tile_m - 1);
  return num <= 0 ? 0 : (num + p.tile_m - 1) / p.tile_m;
}

// v-th tile of the walk over the tiles that are written. The row tiles are
// taken in bands of p.band (about 2,048 rows); a band is walked column by
// column and each column down the band's rows. A wave of the persistent grid
// then covers a block of roughly 2,048 rows by 2,300 columns of C, whose A rows
// and B rows stay in L2 while its tiles run (a column-major walk over all rows
// streams every A row through L2 in every wave).
__device__ __forceinline__ void decode_tile(const TcParams& p, int v, int* mt, int* nt) {
  int b = 0;
  while (b + 1 < kMaxBands && p.band_start[b + 1] <= v && b + 1 < (p.tiles_m + p.band - 1) / p.band)
    ++b;
  v -= p.band_start[b];
  const int r0 = b * p.band, r1 = min(r0 + p.band, p.tiles_m), h = r1 - r0;
  // columns whose first written row tile is at or above r0 hold all h tiles of the band
  int full = p.tiles_n;
  if (p.lower) {
    const int num = r0 * p.tile_m + p.diag_off + p.tile_m - 1;
    full = num < 0 ? 0 : min(p.tiles_n, num / TBN + 1);
  }
  if (v < full * h) {
    *nt = v / h;
    *mt = r0 + v % h;
    return;
  }
  v -= full * h;
  for (int c = full; c < p.tiles_n; ++c) {
    const int f = max(r0, first_mt(p, c));
    const int cnt = max(0, r1 - f);
    if (v < cnt || c == p.tiles_n - 1) {
      *nt = c;
      *mt = f + v;
      return;
    }
    v -= cnt;
  }
  *nt = p.tiles_n - 1;
  *mt = r0;
}

// Persistent warp-specialised kernel: warp 0 TMA producer, warp 1 MMA issuer,
// warp 2 TMEM allocator, warps 4.. epilogue. The accumulator is double-buffered
// in TMEM so the epilogue of one tile overlaps the main loop of the next. With
// PAIR, a cluster of two CTAs walks the tiles together: both load their halves
// of the operands (the bytes counted on the first CTA's barrier), the first
// CTA's issuer runs the MMAs and its commits reach both CTAs, and both
// epilogues drain their own TMEM and report to the first CTA.
template <int PAIR>
__global__ void __launch_bounds__(THREADS, 1) tc_gemm_kernel(const __grid_constant__ TcParams p) {
  using Cfg = TcCfg<PAIR>;
  constexpr int STAGES = Cfg::STAGES, STAGE_BYTES = Cfg::STAGE_BYTES;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint64_t* full_bar = reinterpret_cast<uint64_t*>(smem + STAGES * STAGE_BYTES);
  uint64_t* empty_bar = full_bar + STAGES;
  uint64_t* tfull_bar = empty_bar + STAGES;  // [2]
  uint64_t* tempty_bar = tfull_bar + 2;      // [2]
  uint64_t* drain_bar = tempty_bar + 2;      // the issuer's last commit (every MMA done)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(drain_bar + 1);
  // per epilogue warp: 2^ecol of the 32 columns of its current chunk, and a
  // 32x32 FP32 staging chunk for the TMA reduce-add of C
  float* col_scale = reinterpret_cast<float*>(smem + STAGES * STAGE_BYTES + 256);
  float* c_stage = col_scale + EPI_WARPS * 32;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t crank = PAIR ? cluster_rank() : 0;        // 0: the CTA that issues MMAs
  const int group = PAIR ? (int)(blockIdx.x >> 1) : (int)blockIdx.x;
  const int ngroups = PAIR ? (int)(gridDim.x >> 1) : (int)gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&empty_bar[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&tfull_bar[b], 1);
      mbar_init(&tempty_bar[b], PAIR ? 2 * EPI_WARPS : EPI_WARPS);
    }
    mbar_init(drain_bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 2) {
    if (PAIR) {
      asm volatile("tcgen05.alloc.cta_group::2.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                       smem_u32(tmem_slot)),
                   "r"(TMEM_COLS));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::2.sync.aligned;\n");
    } else {
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                       smem_u32(tmem_slot)),
                   "r"(TMEM_COLS));
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
    }
  }
  __syncthreads();
  if (PAIR) cluster_sync_all();  // both CTAs' barriers initialised, both allocations done
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = *tmem_slot;

  int kblocks = 0;  // K blocks per tile over all segments
  for (int s = 0; s < p.nseg; ++s) kblocks += p.seg[s].nk;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer
    const uint32_t full0 = PAIR ? cluster_addr(smem_u32(full_bar), 0) : 0;
    int it = 0;
    bool ok = true;
    for (int v = group; v < p.total_tiles && ok; v += ngroups) {
      int mt, nt;
      decode_tile(p, v, &mt, &nt);
      const int m0 = mt * Cfg::TILE_M + (int)crank * TBM;
      const int n0 = nt * TBN + (int)crank * Cfg::B_ROWS;
      for (int s = 0; s < p.nseg && ok; ++s) {
        const TcSegment sg = p.seg[s];
        for (int kb = 0; kb < sg.nk; ++kb, ++it) {
          const int st = it % STAGES;
          const uint32_t use = it / STAGES;
          if (use > 0 && !mbar_wait(&empty_bar[st], (use - 1) & 1, p.err, 1, p.spin_limit)) {
            ok = false;
            break;
          }
          uint8_t* sa = smem + st * STAGE_BYTES;
          uint8_t* sb = sa + A_TILE;
          const int xa = sg.ka + kb * sg.kstep, xb = sg.kb + kb * sg.kstep;
          if (PAIR) {
            if (crank == 0) mbar_expect_tx(&full_bar[st], 2 * STAGE_BYTES);
            const uint32_t fb = full0 + (uint32_t)(st * 8);
            tma_load_2d_pair(sa, &p.mapA[sg.a], xa, p.a_row0 + m0, fb);
            tma_load_2d_pair(sb, &p.mapB[sg.b], xb, p.b_row0 + n0, fb);
          } else {
            mbar_expect_tx(&full_bar[st], STAGE_BYTES);
            tma_load_2d(sa, &p.mapA[sg.a], xa, p.a_row0 + m0, &full_bar[st]);
            tma_load_2d(sb, &p.mapB[sg.b], xb, p.b_row0 + n0, &full_bar[st]);
            tma_load_2d(sb + BOX_BYTES, &p.mapB[sg.b], xb, p.b_row0 + n0 + BOX_ROWS, &full_bar[st]);
          }
        }
      }
    }
    // Never leave the CTA with a bulk copy still writing shared memory: wait for
    // the last stages to land (their full barriers) or, in the second CTA of a
    // pair, whose loads are counted on the first CTA's barriers, to be consumed.
    for (int j = (it > STAGES ? it - STAGES : 0); j < it; ++j) {
      const int st = j % STAGES;
      uint64_t* bar = (PAIR && crank != 0) ? &empty_bar[st] : &full_bar[st];
      for (unsigned long long i = 0; i < kSpinLimit && !mbar_try_wait(bar, (j / STAGES) & 1); ++i) {
      }
    }
  } else if (warp == 1 && lane == 0) {
    if (!PAIR || crank == 0) {
      // ---------------- MMA issuer
      const uint32_t idesc =
          (p.kind == kTcBf16) ? idesc_of(1, 1, Cfg::TILE_M)
                              : (p.kind == kTcF16 ? idesc_of(1, 0, Cfg::TILE_M)
                                                  : idesc_of(2, 1, Cfg::TILE_M));
      int it = 0, tc = 0;
      bool ok = true;
      for (int v = group; v < p.total_tiles && ok; v += ngroups, ++tc) {
        const int buf = tc & 1;
        const uint32_t use = tc >> 1;
        if (use > 0 && !mbar_wait(&tempty_bar[buf], (use - 1) & 1, p.err, 4, p.spin_limit)) break;
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t acc = tmem + (uint32_t)(buf * ACC_COLS);
        for (int k = 0; k < kblocks; ++k, ++it) {
          const int st = it % STAGES;
          if (!mbar_wait(&full_bar[st], (it / STAGES) & 1, p.err, 2, p.spin_limit)) {
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t sa = smem_u32(smem + st * STAGE_BYTES);
          const uint64_t da = sw128_desc(sa), db = sw128_desc(sa + A_TILE);
#pragma unroll
          for (int kk = 0; kk < 4; ++kk) {
            const uint64_t off = (uint64_t)((kk * 32) >> 4);
            const uint32_t accum = (k | kk) ? 1u : 0u;
            if (PAIR) {
              if (p.kind != kTcI8) mma_f16_pair(acc, da + off, db + off, idesc, accum);
              else mma_i8_pair(acc, da + off, db + off, idesc, accum);
            } else {
              if (p.kind != kTcI8) mma_f16(acc, da + off, db + off, idesc, accum);
              else mma_i8(acc, da + off, db + off, idesc, accum);
            }
          }
          if (PAIR) mma_commit_pair(&empty_bar[st]);
          else mma_commit(&empty_bar[st]);
        }
        if (!ok) break;  // this tile's accumulator is incomplete: never hand it on
        if (PAIR) mma_commit_pair(&tfull_bar[buf]);
        else mma_commit(&tfull_bar[buf]);
      }
      // Every MMA this thread issued has finished writing TMEM (both CTAs' in a
      // pair) before the CTAs free it, also when a wait gave up mid-tile.
      if (PAIR) mma_commit_pair(drain_bar);
      else mma_commit(drain_bar);
    }
    for (unsigned long long i = 0; i < kSpinLimit && !mbar_try_wait(drain_bar, 0); ++i) {
    }
  } else if (warp >= 4) {
    // ---------------- epilogue: warp w owns TMEM lanes 32 (w % 4).. and one
    // half of the tile's columns
    const int q = warp & 3;
    const int half = (warp - 4) >> 2;
    const uint32_t tempty0 = PAIR ? cluster_addr(smem_u32(tempty_bar), 0) : 0;
    int tc = 0;
    for (int v = group; v < p.total_tiles; v += ngroups, ++tc) {
      int mt, nt;
      decode_tile(p, v, &mt, &nt);
      const int m0 = mt * Cfg::TILE_M + (int)crank * TBM, n0 = nt * TBN;
      const int buf = tc & 1;
      // every lane waits; the warp leaves together if any lane gave up
      const bool got = mbar_wait(&tfull_bar[buf], (tc >> 1) & 1, p.err, 3, p.spin_limit);
      if (!__all_sync(0xffffffffu, got)) break;
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int r = m0 + q * 32 + lane;
      // warp-uniform (lane 0's reading): the loop below holds warp-collective
      // tcgen05.ld and __syncwarp
      const bool live =
          __shfl_sync(0xffffffffu, (int)(kblocks > 0 && !*(volatile int*)p.err), 0) != 0;
      float* wscale = col_scale + (warp - 4) * 32;
      for (int c0 = half * (TBN / 2); c0 < (half + 1) * (TBN / 2) && live; c0 += 32) {
        if (p.epi == kTcEpiF32 && p.erow) {
          // one coalesced load of the chunk's column exponents, shared by the warp
          const int c = n0 + c0 + lane;
          const int e = c < p.N ? p.ecol[c] : 0;
          __syncwarp();
          wscale[lane] = __int_as_float((min(max(e, -126), 127) + 127) << 23);
          __syncwarp();
        }
        uint32_t v32[32];
        const uint32_t taddr =
            tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * ACC_COLS + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
            "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
            : "=r"(v32[0]), "=r"(v32[1]), "=r"(v32[2]), "=r"(v32[3]), "=r"(v32[4]), "=r"(v32[5]),
              "=r"(v32[6]), "=r"(v32[7]), "=r"(v32[8]), "=r"(v32[9]), "=r"(v32[10]),
              "=r"(v32[11]), "=r"(v32[12]), "=r"(v32[13]), "=r"(v32[14]), "=r"(v32[15]),
              "=r"(v32[16]), "=r"(v32[17]), "=r"(v32[18]), "=r"(v32[19]), "=r"(v32[20]),
              "=r"(v32[21]), "=r"(v32[22]), "=r"(v32[23]), "=r"(v32[24]), "=r"(v32[25]),
              "=r"(v32[26]), "=r"(v32[27]), "=r"(v32[28]), "=r"(v32[29]), "=r"(v32[30]),
              "=r"(v32[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        if (p.c_tma) {
          // the previous chunk's reduction must have read the staging buffer
          if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
          __syncwarp();
        }
        if (r < p.M) {
          // Mask of the chunk's columns that this row writes.
          uint32_t mask = 0;
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int c = n0 + c0 + j;
            if (c < p.N && !(p.lower && r + p.diag_off < c)) mask |= 1u << j;
          }
          // All loads of C first (independent, in flight together), then the
          // stores: interleaving them would serialise each load behind the
          // previous store, since the compiler cannot rule out aliasing.
          if (p.epi == kTcEpiF32 && p.c_tma) {
            // staged in shared memory column by column (lane = row: conflict-free), then
            // added into C by one bulk tensor reduction per chunk; masked entries add 0
            float* stg = c_stage + (warp - 4) * (STAGE_C / 4);
            float ra = p.alpha;
            if (p.erow)
              ra *= __int_as_float((min(max(p.erow[r] + p.shift, -126), 127) + 127) << 23);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const float sj = p.erow ? ra * wscale[j] : ra;
              stg[j * 32 + lane] = (mask >> j & 1u) ? sj * __uint_as_float(v32[j]) : 0.f;
            }
          } else if (p.epi == kTcEpiF32) {
            float* dst = static_cast<float*>(p.C) + (size_t)(n0 + c0) * p.ldc + r;
            float old[32];
            // alpha * 2^(erow[r] + shift) from the exponent bits (normal range)
            float ra = p.alpha;
            if (p.erow)
              ra *= __int_as_float((min(max(p.erow[r] + p.shift, -126), 127) + 127) << 23);
#pragma unroll
            for (int j = 0; j < 32; ++j)
              old[j] = (p.beta != 0.f && (mask >> j & 1u)) ? dst[(size_t)j * p.ldc] : 0.f;
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (mask >> j & 1u) {
                const float sj = p.erow ? ra * wscale[j] : ra;
                dst[(size_t)j * p.ldc] = sj * __uint_as_float(v32[j]) + p.beta * old[j];
              }
          } else if (p.epi == kTcEpiMod8) {
            // the exact int32 sum reduced modulo p.modulus, one byte per element
            uint8_t* dst = static_cast<uint8_t*>(p.C) + (size_t)(n0 + c0) * p.ldc + r;
            const int md = p.modulus;
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (mask >> j & 1u) {
                const int t = (int)v32[j] % md;
                dst[(size_t)j * p.ldc] = (uint8_t)(t < 0 ? t + md : t);
              }
          } else {
            double* dst = static_cast<double*>(p.C) + (size_t)(n0 + c0) * p.ldc + r;
            const int er = p.erow[r] + p.shift;
            double old[32];
            int ec[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) {
              const bool w = mask >> j & 1u;
              old[j] = w ? dst[(size_t)j * p.ldc] : 0.0;
              ec[j] = w ? p.ecol[n0 + c0 + j] : 0;
            }
#pragma unroll
            for (int j = 0; j < 32; ++j)
              if (mask >> j & 1u)
                dst[(size_t)j * p.ldc] =
                    old[j] + (double)p.alpha * ldexp((double)(int)v32[j], er + ec[j]);
          }
        }
        if (p.c_tma) {
          // make the staged chunk visible to the TMA unit, then one lane adds it to C
          asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
          __syncwarp();
          if (lane == 0)
            tma_reduce_add_2d(&p.mapC, m0 + q * 32, n0 + c0, c_stage + (warp - 4) * (STAGE_C / 4));
        }
      }
      // release this accumulator buffer to the MMA issuer
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        if (PAIR) mbar_arrive_cluster(tempty0 + (uint32_t)(buf * 8));
        else mbar_arrive(&tempty_bar[buf]);
      }
    }
    // every reduction into C complete before the CTA's shared memory goes away
    if (p.c_tma && lane == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
  }
  __syncthreads();
  if (PAIR) cluster_sync_all();  // neither CTA leaves while the other may still signal it
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (warp == 2) {
    if (PAIR)
      asm volatile("tcgen05.dealloc.cta_group::2.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                   "r"(TMEM_COLS));
    else
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                   "r"(TMEM_COLS));
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

}  // namespace

moao_status make_tc_map(TcTensor* t, const void* base, int kind, long long rows, long long kcols,
                        long long row_stride_elems, int box_rows) {
  if (box_rows != TBM && box_rows != TBN)
    return set_error(MOAO_ERR_BAD_ARG, "tc map: box rows must be 128 (A) or 256 (B)");
  auto fn = encode_fn();
  if (!fn) return set_error(MOAO_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
  const int esz = (kind == kTcI8) ? 1 : 2;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((row_stride_elems * esz) & 15))
    return set_error(MOAO_ERR_BAD_ARG, "tc map: base or row stride not 16-byte aligned");
  if (rows <= 0 || kcols <= 0 || box_rows <= 0 || box_rows > 256)
    return set_error(MOAO_ERR_BAD_ARG, "tc map: bad extents");
  cuuint64_t dims[2] = {(cuuint64_t)kcols, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)(row_stride_elems * esz)};
  // Every box is 128 rows; a B operand's 256-row tile is two boxes (one per CTA
  // of a pair).
  cuuint32_t box[2] = {(cuuint32_t)(KBYTES / esz), (cuuint32_t)BOX_ROWS};
  cuuint32_t estr[2] = {1, 1};
  const CUtensorMapDataType dt = kind == kTcBf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                 : kind == kTcF16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                  : CU_TENSOR_MAP_DATA_TYPE_UINT8;
  CUresult r = fn(&t->map, dt,
                  2, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    return set_error(MOAO_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  t->kind = kind;
  t->kstep = KBYTES / esz;
  t->box_rows = box_rows;
  return MOAO_OK;
}

moao_status tc_gemm(const TcGemm& g, cudaStream_t s, long long* launches) {
  if (g.M <= 0 || g.N <= 0) return MOAO_OK;
  if (g.nA < 1 || g.nA > kTcMaxMaps || g.nB < 1 || g.nB > kTcMaxMaps || g.nseg < 1 ||
      g.nseg > kTcMaxSegs || !g.err)
    return set_error(MOAO_ERR_BAD_ARG, "tc_gemm: bad operand lists");
  if (g.epi == kTcEpiF64Scaled && (g.kind != kTcI8 || !g.erow || !g.ecol))
    return set_error(MOAO_ERR_BAD_ARG, "tc_gemm: scaled epilogue needs int8 and exponents");
  if (g.epi == kTcEpiF32 && g.kind == kTcI8)
    return set_error(MOAO_ERR_BAD_ARG, "tc_gemm: fp32 epilogue needs bf16 or fp16 operands");
  if (g.epi == kTcEpiMod8 && (g.kind != kTcI8 || g.modulus < 2 || g.modulus > 256))
    return set_error(MOAO_ERR_BAD_ARG, "tc_gemm: modular epilogue needs int8 and a modulus <= 256");
  if (g.epi == kTcEpiF32 && (!g.erow) != (!g.ecol))
    return set_error(MOAO_ERR_BAD_ARG, "tc_gemm: row and column exponents go together");
  TcParams p;
  std::memset(&p, 0, sizeof(p));
  for (int i = 0; i < g.nA; ++i) {
    if (g.A[i]->kind != g.kind || g.A[i]->box_rows != TBM)
      return set_error(MOAO_ERR_BAD_ARG, "tc_gemm: A operand kind or box mismatch");
    p.mapA[i] = g.A[i]->map;
  }
  for (int i = 0; i < g.nB; ++i) {
    if (g.B[i]->kind != g.kind || g.B[i]->box_rows != TBN)
      return set_error(MOAO_ERR_BAD_ARG, "tc_gemm: B operand kind or box mismatch");
    p.mapB[i] = g.B[i]->map;
  }
  const int kstep = g.A[0]->kstep;
  for (int i = 0; i < g.nseg; ++i) {
    TcSegment sg = g.seg[i];
    if (sg.a < 0 || sg.a >= g.nA || sg.b < 0 || sg.b >= g.nB || sg.nk < 0 || sg.ka < 0 ||
        sg.kb < 0 || sg.ka % kstep || sg.kb % kstep)
      return set_error(MOAO_ERR_BAD_ARG, "tc_gemm: bad segment");
    sg.kstep = kstep;
    p.seg[i] = sg;
  }
  p.nseg = g.nseg;
  p.M = (int)g.M;
  p.N = (int)g.N;
  p.a_row0 = g.a_row0;
  p.b_row0 = g.b_row0;
  p.lower = g.lower;
  p.diag_off = g.diag_off;
  p.kind = g.kind;
  p.epi = g.epi;
  p.alpha = g.alpha;
  p.beta = g.beta;
  p.C = g.C;
  p.ldc = g.ldc;
  p.erow = g.erow;
  p.ecol = g.ecol;
  p.shift = g.shift;
  p.modulus = g.modulus;
  p.err = g.err;
  p.spin_limit = g.spin_limit > 0 ? g.spin_limit : kSpinLimit;
  // Pairs of CTAs (256-row tiles) when asked for and C has more than one
  // 128-row tile; a grid capped below four CTAs keeps single CTAs.
  const bool pair = g.pair && g.M > TBM && (g.max_ctas <= 0 || g.max_ctas >= 4);
  p.tile_m = pair ? TcCfg<1>::TILE_M : TcCfg<0>::TILE_M;
  p.tiles_m = (int)((g.M + p.tile_m - 1) / p.tile_m);
  p.tiles_n = (int)((g.N + TBN - 1) / TBN);
  p.band = std::max(kBandRows / p.tile_m, (p.tiles_m + kMaxBands - 1) / kMaxBands);
  const int nbands = (p.tiles_m + p.band - 1) / p.band;
  long total = 0;
  for (int b = 0; b < nbands; ++b) {
    p.band_start[b] = (int)total;
    const long r0 = (long)b * p.band, r1 = std::min<long>(r0 + p.band, p.tiles_m);
    for (int nt = 0; nt < p.tiles_n; ++nt) {
      long first = 0;
      if (g.lower) {
        const long num = (long)nt * TBN - g.diag_off - (p.tile_m - 1);
        first = num <= 0 ? 0 : (num + p.tile_m - 1) / p.tile_m;
      }
      total += std::max(0L, r1 - std::max(r0, first));
    }
  }
  for (int b = nbands; b <= kMaxBands; ++b) p.band_start[b] = (int)total;
  if (total == 0) return MOAO_OK;
  p.total_tiles = (int)total;
  // C += alpha * acc (beta 1) through TMA reductions when C's layout allows a
  // tensor map: 16-byte aligned base and row stride.
  p.c_tma = 0;
  if (g.epi == kTcEpiF32 && g.beta == 1.f && !(reinterpret_cast<uintptr_t>(g.C) & 15) &&
      (g.ldc % 4) == 0) {
    auto fn = encode_fn();
    if (fn) {
      cuuint64_t dims[2] = {(cuuint64_t)g.M, (cuuint64_t)g.N};
      cuuint64_t strides[1] = {(cuuint64_t)g.ldc * sizeof(float)};
      cuuint32_t box[2] = {32, 32};
      cuuint32_t estr[2] = {1, 1};
      if (fn(&p.mapC, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, g.C, dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
        p.c_tma = 1;
    }
  }
  static int num_sms = 0;
  if (!num_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, dev);
    if (num_sms <= 0) num_sms = 148;
  }
  if (!pair) {
    static std::atomic<unsigned long long> configured{0};
    MOAO_CUDA_TRY(set_smem_limit(tc_gemm_kernel<0>, (int)TcCfg<0>::SMEM, configured));
    const long ctas =
        std::min<long>(total, g.max_ctas > 0 ? std::min(g.max_ctas, num_sms) : num_sms);
    tc_gemm_kernel<0><<<(unsigned)ctas, THREADS, TcCfg<0>::SMEM, s>>>(p);
  } else {
    static std::atomic<unsigned long long> configured{0};
    MOAO_CUDA_TRY(set_smem_limit(tc_gemm_kernel<1>, (int)TcCfg<1>::SMEM, configured));
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 2;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = TcCfg<1>::SMEM;
    cfg.stream = s;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    // Pairs that can be resident at once (an SM without a partner in its
    // cluster group stays idle), looked up once per device.
    static std::atomic<int> resident[64] = {};
    int dev = 0;
    MOAO_CUDA_TRY(cudaGetDevice(&dev));
    int groups = dev < 64 ? resident[dev].load() : 0;
    if (groups <= 0) {
      cfg.gridDim = dim3((unsigned)(num_sms & ~1));
      MOAO_CUDA_TRY(cudaOccupancyMaxActiveClusters(&groups, tc_gemm_kernel<1>, &cfg));
      if (groups <= 0) groups = num_sms / 2;
      if (dev < 64) resident[dev].store(groups);
    }
    if (g.max_ctas > 0) groups = std::min(groups, g.max_ctas / 2);
    groups = (int)std::min<long>(groups, total);
    cfg.gridDim = dim3((unsigned)(2 * groups));
    MOAO_CUDA_TRY(cudaLaunchKernelEx(&cfg, tc_gemm_kernel<1>, p));
  }
  if (launches) ++*launches;
  MOAO_CUDA_TRY(cudaGetLastError());
  return MOAO_OK;
}

}  // namespace moao

extern "C" moao_status moao_debug_tc_gemm(moao_ctx* ctx, int kind, long M, long N, long K,
                                          const void* A, long lda, int na, const void* B, long ldb,
                                          int nb, int npairs, const int* pa, const int* pb, void* C,
                                          long ldc, float alpha, float beta, const int* erow,
                                          const int* ecol, int shift, int lower) {
  using namespace moao;
  if (!ctx || !A || !B || !C || !pa || !pb || kind < 0 || kind > 2 || na < 1 ||
      na > kTcMaxMaps || nb < 1 || nb > kTcMaxMaps || npairs < 1 || npairs > kTcMaxSegs ||
      ldc < M || lda < K || ldb < K)
    return set_error(MOAO_ERR_BAD_ARG, "debug_tc_gemm: bad arguments");
  std::lock_guard<std::mutex> lk(ctx->mu);
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  const int esz = kind == kTcI8 ? 1 : 2;
  TcTensor ta[kTcMaxMaps], tb[kTcMaxMaps];
  TcGemm g;
  g.kind = kind;
  g.epi = kind == kTcI8 ? kTcEpiF64Scaled : kTcEpiF32;
  g.M = M;
  g.N = N;
  for (int i = 0; i < na; ++i) {
    MOAO_TRY(make_tc_map(&ta[i], (const char*)A + (size_t)i * M * lda * esz, kind, M, K, lda));
    g.A[i] = &ta[i];
  }
  for (int i = 0; i < nb; ++i) {
    MOAO_TRY(make_tc_map(&tb[i], (const char*)B + (size_t)i * N * ldb * esz, kind, N, K, ldb, 256));
    g.B[i] = &tb[i];
  }
  g.nA = na;
  g.nB = nb;
  const int kstep = ta[0].kstep;
  for (int p = 0; p < npairs; ++p) {
    g.seg[p].a = pa[p];
    g.seg[p].b = pb[p];
    g.seg[p].ka = 0;
    g.seg[p].kb = 0;
    g.seg[p].nk = (int)((K + kstep - 1) / kstep);
  }
  g.nseg = npairs;
  g.lower = lower;
  g.alpha = alpha;
  g.beta = beta;
  g.C = C;
  g.ldc = ldc;
  g.erow = erow;
  g.ecol = ecol;
  g.shift = shift;
  g.pair = ctx->tc_pair;
  MOAO_TRY(ctx->ws_info.ensure(2 * sizeof(int)));
  int* err = ctx->ws_info.as<int>() + 1;
  MOAO_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), ctx->stream));
  g.err = err;
  MOAO_TRY(tc_gemm(g, ctx->stream, &ctx->launches));
  int herr = 0;
  MOAO_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  if (herr) return set_error(MOAO_ERR_TIMEOUT, "tc_gemm: bounded wait expired (" + std::to_string(herr) + ")");
  return MOAO_OK;
}
