// Persistent tile-task kernel: the FP64 factorisation and both triangular
// solves of many small reconstructor instances in ONE launch.
//
// The reference schedules the tiled Cholesky and the solves of one instance as
// a DAG of tile tasks on its runtime (chameleon/compute/reconstructor.cpp:27-55
// submits dpotrf / dtrsm / dsyrk / dgemm tile tasks to StarPU; the codelets
// are chameleon/runtime/starpu/codelet/*). Here the DAG of every instance of a
// batch is flattened into one task list on the device, and the CTAs of one
// persistent grid claim tasks in list order from an atomic counter.
//
// Tiles are 64 x 64 (FP64). Per instance, with nt column tiles of Cmm (n) and
// mt row tiles of Ctm (m):
//   POTRF(k)       A_kk = L_kk, Linv_k = L_kk^-1      (leaf_factor_inverse)
//   TRSM(i,k)      A_ik = A_ik Linv_k^T                i > k
//   UPDATE(i,j,k)  A_ij -= A_ik A_jk^T                 i >= j > k (lower if i = j)
//   FUPD(r,c,j)    C_rc -= X_rj L_cj^T                 j < c      (X = Ctm L^-T)
//   FDIAG(r,c)     C_rc = C_rc Linv_c^T
//   BUPD(r,c,j)    C_rc -= R_rj L_jc                   j > c      (R = X L^-1)
//   BDIAG(r,c)     C_rc = C_rc Linv_c
// so that C ends as R = Ctm Cmm^-1 (the reference's dpotrf + two dtrsm,
// lapack/compute/reconstructor.cpp:48-70, in tile order).
//
// Dependencies are tile version counters, not edge lists: a(i,j) counts the
// steps applied to tile (i,j) of A (it is final at k+1 once TRSM(i,k) or
// POTRF(k) ran); w(r,c) counts the forward steps of tile (r,c) of C (X_rc final
// at c+1), then the backward ones (R_rc final at nt+1). A task waits until the
// counters of the tiles it reads and writes reach the values its step needs,
// runs, and publishes the new version of the tile it wrote (release store after
// a fence; waits are acquire loads; tile data is read through L2).
//
// Progress: the list is sorted by DAG level (longest dependency chain from the
// start), so every task a task waits for sits earlier in the list and has
// already been claimed by a CTA that is running. A CTA claims its next task
// only once the inputs of its current one are ready (the current one then
// runs to the end without waiting), so a claimed task is always either being
// waited for by a running CTA or queued behind a task that will finish. The
// earliest unfinished claimed task therefore always has its inputs and
// completes, whether or not the whole grid is resident. Every wait is bounded
// as well (poll count and a global-timer deadline): on expiry the CTA raises
// the error flag and every CTA stops at its next claim or poll; the host
// reports MOAO_ERR_TIMEOUT.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "context.h"
#include "leaf_f64.cuh"
#include "packed.h"

namespace moao {
namespace {

constexpr int T = 64;               // tile edge
constexpr int TLD = T + 4;          // shared-memory leading dimension (conflict-free fragments)
constexpr int NTHREADS = 256;       // 8 warps: 4 along m (16 rows) x 2 along n (32 columns)
constexpr int TILE_SMEM = T * TLD * 8;
// P, Q and (for an update) the old value of the tile written: 102 KB, two CTAs per SM
constexpr int SMEM_BYTES = 3 * TILE_SMEM > LEAF_SMEM_BYTES ? 3 * TILE_SMEM : LEAF_SMEM_BYTES;

enum TaskType { kPotrf = 0, kTrsm, kUpdate, kFUpd, kFDiag, kBUpd, kBDiag };

struct PkInst {
  double* A;         // n x n, lower, column-major (lda)
  double* C;         // m x n, column-major (ldc): Ctm in, R out
  double* Linv;      // nt tiles of 64 x 64 (ld 64)
  unsigned* cnt;     // nt*nt counters of A's tiles, then mt*nt of C's
  long lda, ldc;
  int n, m, nt, mt;
  int* info;         // first failing Cholesky column (1-based), or untouched
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;\n" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}

// m16n8k16 FP64 MMA. Fragments (fixed by the instruction): A 16x16, 8 per
// lane, a[r] = A(gid + 8 (r & 1), 4 (r >> 1) + tig); B 16x8, 4 per lane,
// b[r] = B(4 r + tig, gid); C 16x8, c0, c1 = C(gid, 2 tig + {0,1}),
// c2, c3 = C(gid + 8, 2 tig + {0,1}).
__device__ __forceinline__ void mma16(double (&c)[4], const double (&a)[8], const double (&b)[4]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
      "{%4,%5,%6,%7,%8,%9,%10,%11}, {%12,%13,%14,%15}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(a[4]), "d"(a[5]), "d"(a[6]), "d"(a[7]),
        "d"(b[0]), "d"(b[1]), "d"(b[2]), "d"(b[3]));
}

// s (column-major, ld TLD) <- the rv x cv corner of the tile at g (ld), zeros
// elsewhere; read through L2 with a thread's 16 loads in flight before its
// first store.
__device__ __forceinline__ void load_tile(double* s, const double* g, long ld, int rv, int cv) {
  constexpr int PER = T * T / NTHREADS;  // 16
  double v[PER];
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = threadIdx.x + q * NTHREADS;
    const int r = e & (T - 1), c = e >> 6;
    v[q] = (r < rv && c < cv) ? __ldcg(g + (long)c * ld + r) : 0.0;
  }
#pragma unroll
  for (int q = 0; q < PER; ++q) {
    const int e = threadIdx.x + q * NTHREADS;
    s[(e >> 6) * TLD + (e & (T - 1))] = v[q];
  }
}

// acc = P op(Q) over the 64-wide K of two staged tiles: op(Q) = Q^T (TRANSQ) or
// Q. Warp w computes rows 16 (w & 3) .. +16, columns 32 (w >> 2) .. +32.
template <bool TRANSQ>
__device__ __forceinline__ void tile_product(const double* Ps, const double* Qs,
                                             double (&acc)[4][4]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 32;
  const int gid = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int h = 0; h < 4; ++h) acc[j][h] = 0.0;
#pragma unroll
  for (int k0 = 0; k0 < T; k0 += 16) {
    double a[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) a[r] = Ps[(k0 + 4 * (r >> 1) + tig) * TLD + wm + gid + 8 * (r & 1)];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      double b[4];
      const int col = wn + 8 * j + gid;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int k = k0 + 4 * r + tig;
        b[r] = TRANSQ ? Qs[k * TLD + col] : Qs[col * TLD + k];
      }
      mma16(acc[j], a, b);
    }
  }
}

// D (rv x cv, ld) = acc (SET) or D = Ds - acc (SUB, Ds the staged old value);
// lower: only r >= c.
__device__ __forceinline__ void store_tile(double* D, long ld, int rv, int cv, bool sub, bool lower,
                                           const double* Ds, const double (&acc)[4][4]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 32;
  const int gid = lane >> 2, tig = lane & 3;
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int h = 0; h < 4; ++h) {
      const int r = wm + gid + 8 * (h >> 1), c = wn + 8 * j + 2 * tig + (h & 1);
      if (r >= rv || c >= cv || (lower && r < c)) continue;
      D[(long)c * ld + r] = sub ? Ds[c * TLD + r] - acc[j][h] : acc[j][h];
    }
}

// One GEMM-shaped task: D op= P op(Q), P at Pg (prv x pcv), Q at Qg (qrv x qcv).
// The output is prv x (TRANSQ ? qrv : qcv). D may be P's own tile (SET).
template <bool TRANSQ>
__device__ __forceinline__ void tile_task(double* smem, const double* Pg, long ldp, int prv, int pcv,
                                          const double* Qg, long ldq, int qrv, int qcv, double* D,
                                          long ldd, bool sub, bool lower) {
  double* Ps = smem;
  double* Qs = smem + T * TLD;
  double* Ds = smem + 2 * T * TLD;
  const int dcv = TRANSQ ? qrv : qcv;
  load_tile(Ps, Pg, ldp, prv, pcv);
  load_tile(Qs, Qg, ldq, qrv, qcv);
  if (sub) load_tile(Ds, D, ldd, prv, dcv);
  __syncthreads();
  double acc[4][4];
  tile_product<TRANSQ>(Ps, Qs, acc);
  store_tile(D, ldd, prv, dcv, sub, lower, Ds, acc);
}

struct Wait {
  const unsigned* p;
  unsigned v;
};

__global__ void __launch_bounds__(NTHREADS, 2)
    packed_tasks_kernel(const PkInst* __restrict__ insts, const int4* __restrict__ tasks,
                        long ntasks, unsigned long long* next, int* err,
                        unsigned long long poll_limit, unsigned long long wait_ns) {
  extern __shared__ __align__(16) double smem[];
  // The task this CTA runs and the next one it has claimed: thread 0 claims the
  // next task once the current one's inputs are ready (it then runs without
  // further waits), so the claim and the task fetch overlap the current work.
  __shared__ int4 s_task[2];
  __shared__ int s_valid[2];
  __shared__ int stop;
  const int tid = threadIdx.x;
  auto claim = [&](int slot) {  // thread 0
    const long t = (long)atomicAdd(next, 1ull);
    const bool ok = t < ntasks && *(volatile int*)err == 0;
    s_valid[slot] = ok;
    if (ok) s_task[slot] = tasks[t];
  };
  if (tid == 0) claim(0);
  __syncthreads();
  for (int it = 0;; ++it) {
    const int sl = it & 1;
    if (!s_valid[sl]) break;
    const int4 tk = s_task[sl];
    const PkInst I = insts[tk.x];
    const int type = tk.y, i = tk.z >> 16, j = tk.z & 0xffff, k = tk.w;
    const int nt = I.nt;
    unsigned* a = I.cnt;                      // a[i * nt + j]
    unsigned* w = I.cnt + (size_t)nt * nt;    // w[r * nt + c]
    auto tn = [&](int q) { return min(T, I.n - q * T); };  // valid size of tile q of n
    auto tm = [&](int q) { return min(T, I.m - q * T); };  // of m
    auto At = [&](int r, int c) { return I.A + (long)c * T * I.lda + (long)r * T; };
    auto Ct = [&](int r, int c) { return I.C + (long)c * T * I.ldc + (long)r * T; };
    const double* Lk = I.Linv + (size_t)k * T * T;
    // waits (up to three) and the published counter
    Wait wt[3];
    int nw = 0;
    unsigned* out = nullptr;
    unsigned outv = 0;
    switch (type) {
      case kPotrf:  // i = j = k
        wt[nw++] = {a + k * nt + k, (unsigned)k};
        out = a + k * nt + k; outv = k + 1;
        break;
      case kTrsm:   // tile (i, k)
        wt[nw++] = {a + k * nt + k, (unsigned)k + 1};
        wt[nw++] = {a + i * nt + k, (unsigned)k};
        out = a + i * nt + k; outv = k + 1;
        break;
      case kUpdate:  // tile (i, j), step k
        wt[nw++] = {a + i * nt + k, (unsigned)k + 1};
        wt[nw++] = {a + j * nt + k, (unsigned)k + 1};
        wt[nw++] = {a + i * nt + j, (unsigned)k};
        out = a + i * nt + j; outv = k + 1;
        break;
      case kFUpd:  // tile (r = i, c = j), step k (< c)
        wt[nw++] = {w + i * nt + k, (unsigned)k + 1};
        wt[nw++] = {a + j * nt + k, (unsigned)k + 1};
        wt[nw++] = {w + i * nt + j, (unsigned)k};
        out = w + i * nt + j; outv = k + 1;
        break;
      case kFDiag:  // tile (r = i, c = k)
        wt[nw++] = {w + i * nt + k, (unsigned)k};
        wt[nw++] = {a + k * nt + k, (unsigned)k + 1};
        out = w + i * nt + k; outv = k + 1;
        break;
      case kBUpd:  // tile (r = i, c = j), source column k (> c)
        wt[nw++] = {w + i * nt + k, (unsigned)nt + 1};
        wt[nw++] = {w + i * nt + j, (unsigned)(j + nt - k)};
        out = w + i * nt + j; outv = j + 1 + nt - k;
        break;
      default:  // kBDiag: tile (r = i, c = k)
        wt[nw++] = {w + i * nt + k, (unsigned)nt};
        out = w + i * nt + k; outv = nt + 1;
        break;
    }
    if (tid == 0) {
      // all counters polled together; bounded by poll count and deadline
      int ok = 1;
      const unsigned long long deadline = global_ns() + wait_ns;
      unsigned long long polls = 0;
      for (;;) {
        bool ready = true;
        unsigned v[3];
#pragma unroll
        for (int q = 0; q < 3; ++q) v[q] = q < nw ? ld_acquire(wt[q].p) : 0u;
#pragma unroll
        for (int q = 0; q < 3; ++q) ready &= q >= nw || v[q] >= wt[q].v;
        if (ready) break;
        if (*(volatile int*)err != 0) { ok = 0; break; }
        if (++polls >= poll_limit || global_ns() > deadline) {
          atomicCAS(err, 0, 1);
          ok = 0;
          break;
        }
        __nanosleep(128);
      }
      stop = !ok;
      if (ok) claim(sl ^ 1);
    }
    __syncthreads();
    if (stop) break;
    switch (type) {
      case kPotrf:
        leaf_factor_inverse<NTHREADS>(At(k, k), I.lda, I.Linv + (size_t)k * T * T, T, tn(k), (long)k * T,
                            I.info, smem);
        break;
      case kTrsm:
        tile_task<true>(smem, At(i, k), I.lda, tn(i), tn(k), Lk, T, tn(k), tn(k), At(i, k), I.lda,
                        false, false);
        break;
      case kUpdate:
        tile_task<true>(smem, At(i, k), I.lda, tn(i), tn(k), At(j, k), I.lda, tn(j), tn(k),
                        At(i, j), I.lda, true, i == j);
        break;
      case kFUpd:
        tile_task<true>(smem, Ct(i, k), I.ldc, tm(i), tn(k), At(j, k), I.lda, tn(j), tn(k),
                        Ct(i, j), I.ldc, true, false);
        break;
      case kFDiag:
        tile_task<true>(smem, Ct(i, k), I.ldc, tm(i), tn(k), Lk, T, tn(k), tn(k), Ct(i, k), I.ldc,
                        false, false);
        break;
      case kBUpd:
        tile_task<false>(smem, Ct(i, k), I.ldc, tm(i), tn(k), At(k, j), I.lda, tn(k), tn(j),
                         Ct(i, j), I.ldc, true, false);
        break;
      default:
        tile_task<false>(smem, Ct(i, k), I.ldc, tm(i), tn(k), Lk, T, tn(k), tn(k), Ct(i, k), I.ldc,
                         false, false);
        break;
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      st_release(out, outv);
    }
  }
}

int4 task(int inst, int type, int i, int j, int k) { return make_int4(inst, type, (i << 16) | j, k); }

// Task list: every instance's DAG in program order with its level (longest
// chain of dependencies), then all tasks bucketed by level (stable: instance,
// then program order, inside a level).
void task_list(const std::vector<long>& ns, const std::vector<long>& ms, std::vector<int4>* out,
               int* levels) {
  std::vector<int4> all;
  std::vector<int> lev;
  for (size_t q = 0; q < ns.size(); ++q) {
    const int nt = (int)((ns[q] + T - 1) / T), mt = (int)((ms[q] + T - 1) / T), id = (int)q;
    std::vector<int> lw((size_t)nt * nt, 0), lf((size_t)nt * nt, 0);     // A: last write, final
    std::vector<int> cw((size_t)mt * nt, 0), cf((size_t)mt * nt, 0), cb((size_t)mt * nt, 0);
    auto A_ = [&](std::vector<int>& x, int r, int c) -> int& { return x[(size_t)r * nt + c]; };
    auto C_ = [&](std::vector<int>& x, int r, int c) -> int& { return x[(size_t)r * nt + c]; };
    auto push = [&](int4 t, int l) {
      all.push_back(t);
      lev.push_back(l);
    };
    for (int k = 0; k < nt; ++k) {
      int l = A_(lw, k, k) + 1;
      A_(lw, k, k) = A_(lf, k, k) = l;
      push(task(id, kPotrf, k, k, k), l);
      for (int i = k + 1; i < nt; ++i) {
        l = std::max(A_(lf, k, k), A_(lw, i, k)) + 1;
        A_(lw, i, k) = A_(lf, i, k) = l;
        push(task(id, kTrsm, i, k, k), l);
      }
      for (int j = k + 1; j < nt; ++j)
        for (int i = j; i < nt; ++i) {
          l = std::max({A_(lf, i, k), A_(lf, j, k), A_(lw, i, j)}) + 1;
          A_(lw, i, j) = l;
          push(task(id, kUpdate, i, j, k), l);
        }
    }
    for (int c = 0; c < nt; ++c)
      for (int r = 0; r < mt; ++r) {
        for (int j = 0; j < c; ++j) {
          const int l = std::max({C_(cf, r, j), A_(lf, c, j), C_(cw, r, c)}) + 1;
          C_(cw, r, c) = l;
          push(task(id, kFUpd, r, c, j), l);
        }
        const int l = std::max(C_(cw, r, c), A_(lf, c, c)) + 1;
        C_(cw, r, c) = C_(cf, r, c) = l;
        push(task(id, kFDiag, r, c, c), l);
      }
    for (int c = nt - 1; c >= 0; --c)
      for (int r = 0; r < mt; ++r) {
        for (int j = nt - 1; j > c; --j) {
          const int l = std::max(C_(cb, r, j), C_(cw, r, c)) + 1;
          C_(cw, r, c) = l;
          push(task(id, kBUpd, r, c, j), l);
        }
        const int l = std::max(C_(cw, r, c), A_(lf, c, c)) + 1;
        C_(cw, r, c) = C_(cb, r, c) = l;
        push(task(id, kBDiag, r, c, c), l);
      }
  }
  int maxl = 0;
  for (int l : lev) maxl = std::max(maxl, l);
  std::vector<size_t> start((size_t)maxl + 2, 0);
  for (int l : lev) ++start[(size_t)l + 1];
  for (size_t l = 1; l < start.size(); ++l) start[l] += start[l - 1];
  out->assign(all.size(), int4{});
  for (size_t e = 0; e < all.size(); ++e) (*out)[start[(size_t)lev[e]]++] = all[e];
  *levels = maxl;
}

}  // namespace

void PackedPlan::release() {
  inst.release();
  tasks.release();
  cnt.release();
  linv.release();
  ctl.release();
  ntasks = 0;
}

size_t packed_workspace_bytes(long n, long m) {
  const long nt = (n + T - 1) / T, mt = (m + T - 1) / T;
  return sizeof(double) * (size_t)nt * T * T + sizeof(unsigned) * (size_t)nt * (nt + mt) +
         sizeof(int4) * (size_t)(nt * nt * nt / 6 + nt * nt + nt * nt * mt + 2 * nt * mt + 64);
}

moao_status packed_prepare(const std::vector<PackedInst>& v, PackedPlan* plan, cudaStream_t s) {
  plan->ntasks = 0;
  if (v.empty()) return MOAO_OK;
  std::vector<PkInst> hi(v.size());
  size_t cnt_words = 0, linv_elems = 0;
  for (size_t q = 0; q < v.size(); ++q) {
    const PackedInst& p = v[q];
    if (p.n <= 0 || p.m < 0 || p.n > 65535L * T || p.m > 65535L * T || p.lda < p.n ||
        (p.m > 0 && p.ldc < p.m))
      return set_error(MOAO_ERR_BAD_ARG, "packed: instance sizes");
    PkInst& h = hi[q];
    h.A = p.A;
    h.C = p.C;
    h.lda = p.lda;
    h.ldc = p.ldc;
    h.n = (int)p.n;
    h.m = (int)p.m;
    h.nt = (int)((p.n + T - 1) / T);
    h.mt = (int)((p.m + T - 1) / T);
    h.info = p.info;
    cnt_words += (size_t)h.nt * (h.nt + h.mt);
    linv_elems += (size_t)h.nt * T * T;
  }
  std::vector<long> ns(v.size()), ms(v.size());
  for (size_t q = 0; q < v.size(); ++q) {
    ns[q] = v[q].n;
    ms[q] = v[q].m;
  }
  std::vector<int4> sorted;
  int maxl = 0;
  task_list(ns, ms, &sorted, &maxl);
  // device copies
  MOAO_TRY(plan->linv.ensure(sizeof(double) * linv_elems));
  MOAO_TRY(plan->cnt.ensure(sizeof(unsigned) * cnt_words));
  size_t lo = 0, co = 0;
  for (PkInst& h : hi) {
    h.Linv = plan->linv.as<double>() + lo;
    h.cnt = plan->cnt.as<unsigned>() + co;
    lo += (size_t)h.nt * T * T;
    co += (size_t)h.nt * (h.nt + h.mt);
  }
  MOAO_TRY(plan->inst.ensure(sizeof(PkInst) * hi.size()));
  MOAO_TRY(plan->tasks.ensure(sizeof(int4) * sorted.size()));
  MOAO_TRY(plan->ctl.ensure(sizeof(unsigned long long) + sizeof(int)));
  MOAO_CUDA_TRY(cudaMemcpyAsync(plan->inst.p, hi.data(), sizeof(PkInst) * hi.size(),
                                cudaMemcpyHostToDevice, s));
  MOAO_CUDA_TRY(cudaMemcpyAsync(plan->tasks.p, sorted.data(), sizeof(int4) * sorted.size(),
                                cudaMemcpyHostToDevice, s));
  MOAO_CUDA_TRY(cudaStreamSynchronize(s));
  plan->ntasks = (long)sorted.size();
  plan->levels = maxl;
  plan->cnt_bytes = sizeof(unsigned) * cnt_words;
  return MOAO_OK;
}

moao_status packed_launch(const PackedPlan& plan, cudaStream_t s, unsigned long long polls,
                          double wait_s, long long* launches) {
  if (plan.ntasks <= 0) return MOAO_OK;
  static std::atomic<unsigned long long> configured{0};
  MOAO_CUDA_TRY(set_smem_limit(packed_tasks_kernel, SMEM_BYTES, configured));
  int dev = 0, sms = 0, per_sm = 0;
  MOAO_CUDA_TRY(cudaGetDevice(&dev));
  MOAO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  MOAO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, packed_tasks_kernel,
                                                              NTHREADS, SMEM_BYTES));
  const long grid = std::min<long>((long)std::max(1, per_sm) * sms, plan.ntasks);
  MOAO_CUDA_TRY(cudaMemsetAsync(plan.cnt.p, 0, plan.cnt_bytes, s));
  MOAO_CUDA_TRY(cudaMemsetAsync(plan.ctl.p, 0, sizeof(unsigned long long) + sizeof(int), s));
  unsigned long long* next = plan.ctl.as<unsigned long long>();
  int* err = reinterpret_cast<int*>(next + 1);
  const unsigned long long ns = (unsigned long long)(std::max(1e-3, wait_s) * 1e9);
  packed_tasks_kernel<<<(unsigned)grid, NTHREADS, SMEM_BYTES, s>>>(
      plan.inst.as<PkInst>(), plan.tasks.as<int4>(), plan.ntasks, next, err,
      polls > 0 ? polls : ~0ull, ns);
  MOAO_CUDA_TRY(cudaGetLastError());
  if (launches) *launches += 1;
  return MOAO_OK;
}

const int* packed_error_flag(const PackedPlan& plan) {
  return reinterpret_cast<const int*>(plan.ctl.as<unsigned long long>() + 1);
}

}  // namespace moao

extern "C" moao_status moao_packed_task_list(int count, const long* nmeas, const long* nmeasts,
                                             int* tasks, long cap, long* ntasks, int* levels) {
  using namespace moao;
  if (count < 0 || (count > 0 && (!nmeas || !nmeasts)) || !ntasks || (cap > 0 && !tasks))
    return set_error(MOAO_ERR_BAD_ARG, "packed_task_list: null argument");
  std::vector<long> ns(nmeas, nmeas + count), ms(nmeasts, nmeasts + count);
  for (int q = 0; q < count; ++q)
    if (ns[q] <= 0 || ms[q] < 0 || ns[q] > 65535L * T || ms[q] > 65535L * T)
      return set_error(MOAO_ERR_BAD_ARG, "packed_task_list: instance sizes");
  std::vector<int4> list;
  int maxl = 0;
  task_list(ns, ms, &list, &maxl);
  *ntasks = (long)list.size();
  if (levels) *levels = maxl;
  const long n = std::min<long>(cap, (long)list.size());
  for (long e = 0; e < n; ++e) {
    const int4 t = list[(size_t)e];
    int* d = tasks + 5 * e;
    d[0] = t.x;
    d[1] = t.y;
    d[2] = t.z >> 16;
    d[3] = t.z & 0xffff;
    d[4] = t.w;
  }
  return MOAO_OK;
}
