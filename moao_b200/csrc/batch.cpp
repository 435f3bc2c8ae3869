// Batched instances: many independent reconstructor builds (covariance
// generation, factorisation, solves) captured as one CUDA graph and launched
// once.
//
// Instances are assigned to S streams, longest first onto the least-loaded
// stream (estimated cost n^3/3 + n^2 m plus the covariance term); each stream
// has its own context (workspaces sized before capture for the largest
// instance it runs) and reuses one Cmm / Ctm pair for its instances in stream
// order, so device memory is S x (largest instance), not the sum. Geometry
// tables are uploaded before capture. Inside the capture nothing waits for the
// device: each instance's failure flags are copied to a status array read after
// the graph ran. The graph is one launch however many instances it holds; small
// instances, whose kernels are short, overlap with each other and with the
// large ones on the other streams.
//
// Instances up to a size bound (packed_max) are taken out of the streams and
// built together by the persistent tile-task kernel (packed.cu) in a branch of
// the same graph: their covariance launches, then one launch for all of their
// factorisations and solves.
//
// Autotuner: per nmeas size class and precision, the panel width (the tile
// size of the blocked factorisation) with the shortest measured build, the
// size bound of the packed instances, and the number of streams with the
// shortest measured batch; kept on the context and saved to / loaded from a
// text file.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "context.h"
#include "moao_b200.h"
#include "dense.h"
#include "packed.h"

namespace moao {
namespace {

constexpr int kClasses = 6;  // nmeas < 2k, 4k, 8k, 16k, 32k, larger

int size_class(long n) {
  int c = 0;
  for (long lim = 2048; c < kClasses - 1 && n >= lim; lim *= 2) ++c;
  return c;
}

struct TuneEntry {
  int nb = 0;     // 0: not tuned
  int gemm = 1;   // tile configuration of the large FP64 products (GemmArgs::cfg)
};

}  // namespace
}  // namespace moao

// Tuning table kept per context (allocated on first use).
struct moao_tuning {
  moao::TuneEntry entry[2][moao::kClasses];  // [prec][class]
  int streams[2] = {0, 0};
  long packed[2] = {0, 0};  // nmeas bound of the packed instances (0: none)
};

namespace moao {
namespace {

std::map<const moao_ctx*, moao_tuning>& tuning_tables() {
  static std::map<const moao_ctx*, moao_tuning> t;
  return t;
}
std::mutex& tuning_mutex() {
  static std::mutex m;
  return m;
}

int default_nb(long n) { return n < 4096 ? 128 : 256; }

int tuned_nb(const moao_ctx* ctx, moao_prec prec, long n) {
  std::lock_guard<std::mutex> lk(tuning_mutex());
  auto it = tuning_tables().find(ctx);
  if (it != tuning_tables().end()) {
    const int nb = it->second.entry[prec == MOAO_PREC_MIXED][size_class(n)].nb;
    if (nb > 0) return nb;
  }
  return default_nb(n);
}

int tuned_gemm(const moao_ctx* ctx, moao_prec prec, long n) {
  std::lock_guard<std::mutex> lk(tuning_mutex());
  auto it = tuning_tables().find(ctx);
  if (it != tuning_tables().end()) return it->second.entry[prec == MOAO_PREC_MIXED][size_class(n)].gemm;
  return 1;
}

int tuned_streams(const moao_ctx* ctx, moao_prec prec) {
  std::lock_guard<std::mutex> lk(tuning_mutex());
  auto it = tuning_tables().find(ctx);
  if (it != tuning_tables().end() && it->second.streams[prec == MOAO_PREC_MIXED] > 0)
    return it->second.streams[prec == MOAO_PREC_MIXED];
  return 4;
}

long tuned_packed(const moao_ctx* ctx, moao_prec prec) {
  std::lock_guard<std::mutex> lk(tuning_mutex());
  auto it = tuning_tables().find(ctx);
  return it != tuning_tables().end() ? it->second.packed[prec == MOAO_PREC_MIXED] : 0;
}

// Size bound of class c (nmeas below it).
long class_limit(int c) { return 2048L << c; }

struct Inst {
  int item;
  long n, m;
  int nb;
  int gemm;
  double cost;
  const DevGeometry* g;
  int stream;
  bool packed;
};

// Builds one instance on sub-context sc (stream sc->stream): covariances into
// Cmm / Ctm, factorisation and solves, R copied to the caller, flags to status.
moao_status enqueue_instance(moao_ctx* sc, const moao_tomo* tomo, const Inst& in, moao_prec prec,
                             double* Cmm, double* Ctm, double* d_R, int* status) {
  cudaStream_t s = sc->stream;
  const long n = in.n, m = in.m;
  sc->nb = in.nb;
  sc->gemm_cfg = in.gemm;
  MOAO_TRY(launch_matcov(*in.g, Cmm, (int)n, (int)n, 0, 0, (int)n, 1, s, &sc->launches));
  MOAO_TRY(launch_matcov(*in.g, Ctm, (int)m, (int)n, 0, 0, (int)m, 3, s, &sc->launches));
  int* d_info = sc->ws_info.as<int>();
  if (prec == MOAO_PREC_MIXED) {
    MOAO_TRY(moao_ctx_set_offsets_from_tomo(sc, tomo));
    moao_solve_report rep{};
    MOAO_TRY(reconstructor_mixed(sc, n, m, Cmm, n, Ctm, m, false, &rep));
  } else {
    MOAO_CUDA_TRY(cudaMemsetAsync(d_info, 0, 3 * sizeof(int), s));
    MOAO_TRY(potrf_f64(sc, Cmm, n, n, sc->ws_dinv.as<double>(), d_info));
    MOAO_TRY(solve_right_f64(sc, Cmm, n, n, sc->ws_dinv.as<double>(), Ctm, m, m));
  }
  MOAO_CUDA_TRY(cudaMemcpyAsync(status, d_info, 3 * sizeof(int), cudaMemcpyDeviceToDevice, s));
  if (d_R)
    MOAO_CUDA_TRY(cudaMemcpyAsync(d_R, Ctm, sizeof(double) * (size_t)m * n,
                                  cudaMemcpyDeviceToDevice, s));
  return MOAO_OK;
}

// Sub-contexts of a context for batched work (created on first use).
std::vector<moao_ctx*>& sub_contexts(moao_ctx* ctx) {
  static std::map<const moao_ctx*, std::vector<moao_ctx*>> subs;
  static std::mutex mu;
  std::lock_guard<std::mutex> lk(mu);
  return subs[ctx];
}

}  // namespace

void release_batch_state(moao_ctx* ctx) {
  {
    std::lock_guard<std::mutex> lk(tuning_mutex());
    tuning_tables().erase(ctx);
  }
  std::vector<moao_ctx*>& v = sub_contexts(ctx);
  for (moao_ctx* c : v) moao_ctx_destroy(c);
  v.clear();
}

namespace {

moao_status ensure_subs(moao_ctx* ctx, int S) {
  std::vector<moao_ctx*>& v = sub_contexts(ctx);
  while ((int)v.size() < S) {
    moao_ctx* c = nullptr;
    MOAO_TRY(moao_ctx_create(ctx->device, &c));
    c->lookahead_sms = 0;  // concurrent instances fill the SMs; no side stream in the capture
    v.push_back(c);
  }
  return MOAO_OK;
}

moao_status run_batch(moao_ctx* ctx, int count, moao_batch_item* items, moao_batch_opts* o) {
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  const moao_prec prec = o->prec;
  const long pmax = o->packed_max > 0 ? o->packed_max
                                      : (o->packed_max == 0 ? tuned_packed(ctx, prec) : 0);
  std::vector<Inst> inst;
  for (int i = 0; i < count; ++i) {
    const Tomo_struct<double>& t = items[i].tomo->t;
    Inst in;
    in.item = i;
    in.n = t.getNMeas();
    in.m = t.getNMeasTS();
    in.nb = items[i].nb > 0 ? items[i].nb : tuned_nb(ctx, prec, in.n);
    if (in.nb % 64 || in.nb < 64 || in.nb > 2048)
      return set_error(MOAO_ERR_BAD_ARG, "batch: panel width must be a multiple of 64 in [64, 2048]");
    in.gemm = o->gemm_tile > 0 ? o->gemm_tile - 1 : tuned_gemm(ctx, prec, in.n);
    const double n = (double)in.n, m = (double)in.m;
    in.cost = n * n * n / 3 + n * n * m + 40.0 * t.atm.nLayer * n * (n / 2 + m);
    MOAO_TRY(device_geometry(ctx, items[i].tomo, &in.g));
    in.stream = 0;
    in.packed = in.n <= pmax;
    inst.push_back(in);
  }
  // packed instances: their own Cmm (ld n) and Ctm (into d_R when given), the
  // plan's state; counted against the budget first
  std::vector<int> pk;
  size_t pk_bytes = 0, pk_data = 0;
  for (int i = 0; i < count; ++i)
    if (inst[i].packed) {
      pk.push_back(i);
      const size_t nn = (size_t)inst[i].n, mm = (size_t)inst[i].m;
      pk_data += nn * nn + (items[i].d_R ? 0 : mm * nn);
      pk_bytes += packed_workspace_bytes(inst[i].n, inst[i].m);
    }
  pk_bytes += sizeof(double) * pk_data;
  const int ngraph = count - (int)pk.size();
  int S = o->streams > 0 ? o->streams : tuned_streams(ctx, prec);
  S = std::max(0, std::min({S, ngraph, 16}));
  if (ngraph > 0) S = std::max(S, 1);
  // Device bytes of one instance: Cmm, Ctm and the workspace of its path.
  MOAO_TRY(ensure_subs(ctx, std::max(S, 1)));
  const moao_ctx* proto = sub_contexts(ctx)[0];
  auto bytes_of_inst = [&](const Inst& in) {
    size_t b = sizeof(double) * ((size_t)in.n * in.n + (size_t)in.m * in.n);
    if (prec == MOAO_PREC_MIXED) {
      const Tomo_struct<double>& t = items[in.item].tomo->t;
      const int nro = t.sys.lgsCst > 0 ? 2 * t.sys.nLgs : 0;
      b += mixed_sizes(in.n, in.m, in.nb, std::max(2, std::min(kMaxBfSlices, proto->bf16_slices)),
                       proto->ozaki_slices, nro, proto->residual_crt != 0).total();
    } else {
      b += sizeof(double) * (size_t)in.nb * ((size_t)in.n + std::max(in.n, in.m));
    }
    return b;
  };
  // Budget: what is free plus what the sub-contexts already hold (reused).
  size_t fr = 0, tot = 0, held = 0;
  MOAO_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
  for (moao_ctx* c : sub_contexts(ctx)) held += c->bytes_held();
  const size_t budget_all = o->hbm_budget_gb > 0 ? (size_t)(o->hbm_budget_gb * 1e9)
                                                 : (size_t)(0.85 * (double)(fr + held));
  if (pk_bytes > budget_all)
    return set_error(MOAO_ERR_OOM, "batch: the packed instances exceed the device budget");
  const size_t budget = budget_all - pk_bytes;
  // Longest first onto the least-loaded stream; a new stream is opened only
  // while its first (largest) instance fits the budget, since a stream holds
  // buffers for its largest instance and instances arrive largest first.
  std::vector<int> order;
  for (int i = 0; i < count; ++i)
    if (!inst[i].packed) order.push_back(i);
  std::sort(order.begin(), order.end(), [&](int a, int b) { return inst[a].cost > inst[b].cost; });
  std::vector<double> load;
  std::vector<size_t> foot;
  std::vector<std::vector<int>> per;
  size_t planned = 0;
  for (int i : order) {
    const size_t f = bytes_of_inst(inst[i]);
    int k = -1;
    if (!load.empty()) k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    const bool can_open = (int)load.size() < S && planned + f <= budget;
    auto open_stream = [&]() {
      load.push_back(0.0);
      foot.push_back(0);
      per.emplace_back();
      return (int)load.size() - 1;
    };
    if (can_open && (k < 0 || load[k] > 0)) {
      k = open_stream();
    } else if (k >= 0 && f > foot[k] && planned - foot[k] + f > budget) {
      // the least-loaded stream cannot grow to this instance: the least-loaded
      // one that holds it within the budget, else a new stream
      k = -1;
      double best = 0;
      for (size_t j = 0; j < load.size(); ++j) {
        const size_t grow = f > foot[j] ? f - foot[j] : 0;
        if (planned + grow <= budget && (k < 0 || load[j] < best)) {
          k = (int)j;
          best = load[j];
        }
      }
      if (k < 0 && can_open) k = open_stream();
    }
    if (k < 0) return set_error(MOAO_ERR_OOM, "batch: an instance exceeds the device budget");
    if (f > foot[k]) {
      planned += f - foot[k];
      foot[k] = f;
    }
    inst[i].stream = k;
    load[k] += inst[i].cost;
    per[k].push_back(i);
  }
  S = (int)per.size();
  // Workspaces kept from earlier batches: drop those much larger than this
  // plan needs and those of streams this batch does not use.
  {
    std::vector<moao_ctx*>& v = sub_contexts(ctx);
    for (size_t k = 0; k < v.size(); ++k) {
      const size_t want = (int)k < S ? foot[k] : 0;
      if (v[k]->bytes_held() > want + want / 2) {
        cudaStreamSynchronize(v[k]->stream);
        for (DevBuf* b : v[k]->workspaces()) b->release();
      }
    }
  }
  // memory: per stream its largest Cmm / Ctm pair and workspace
  std::vector<moao_ctx*>& subs = sub_contexts(ctx);
  std::vector<DevBuf> cmm(S), ctm(S);
  DevBuf status, pkbuf;
  PackedPlan plan;
  cudaStream_t ps = nullptr;  // the packed branch
  // the packed instances' covariance launches, spread over a few streams (small
  // instances' launches fill the GPU one at a time only partly)
  constexpr int kCovStreams = 4;
  std::vector<cudaStream_t> cs;
  // DevBuf frees nothing by itself: release the batch's own buffers on every exit
  struct Release {
    std::vector<DevBuf>& a;
    std::vector<DevBuf>& b;
    DevBuf& c;
    DevBuf& d;
    PackedPlan& e;
    cudaStream_t& f;
    std::vector<cudaStream_t>& g;
    ~Release() {
      for (DevBuf& x : a) x.release();
      for (DevBuf& x : b) x.release();
      c.release();
      d.release();
      e.release();
      if (f) cudaStreamDestroy(f);
      for (cudaStream_t x : g) cudaStreamDestroy(x);
    }
  } release_guard{cmm, ctm, status, pkbuf, plan, ps, cs};
  size_t total = 0;
  for (int k = 0; k < S; ++k) {
    moao_ctx* sc = subs[k];
    sc->graph_mode = (prec == MOAO_PREC_MIXED);
    sc->timing = false;
    long nmax = 0, mmax = 0;
    size_t ws = 0;
    for (int i : per[k]) {
      nmax = std::max(nmax, inst[i].n);
      mmax = std::max(mmax, inst[i].m);
      const Inst& in = inst[i];
      if (prec == MOAO_PREC_MIXED) {
        const Tomo_struct<double>& t = items[in.item].tomo->t;
        const int nro = t.sys.lgsCst > 0 ? 2 * t.sys.nLgs : 0;
        const MixedSizes z = mixed_sizes(in.n, in.m, in.nb, std::max(2, std::min(kMaxBfSlices, sc->bf16_slices)),
                                         sc->ozaki_slices, nro, sc->residual_crt != 0);
        // size every workspace buffer for the largest instance of this stream
        MOAO_TRY(sc->mx_a32.ensure(z.a32));
        MOAO_TRY(sc->mx_lr.ensure(z.lr));
        MOAO_TRY(sc->mx_lc.ensure(z.lr));
        MOAO_TRY(sc->mx_t32.ensure(z.t32));
        MOAO_TRY(sc->mx_w1.ensure(z.w));
        MOAO_TRY(sc->mx_w2.ensure(z.w));
        MOAO_TRY(sc->mx_x.ensure(z.x));
        MOAO_TRY(sc->mx_r64.ensure(z.r64));
        MOAO_TRY(sc->mx_e64.ensure(z.r64));
        MOAO_TRY(sc->mx_qa.ensure(z.qa));
        MOAO_TRY(sc->mx_qb.ensure(z.qb));
        MOAO_TRY(sc->mx_qr.ensure(z.qr));
        MOAO_TRY(sc->mx_qs.ensure(z.qs));
        MOAO_TRY(sc->mx_z.ensure(z.z));
        MOAO_TRY(sc->mx_ea.ensure(z.ea));
        MOAO_TRY(sc->mx_fb.ensure(z.fb));
        MOAO_TRY(sc->mx_colmax.ensure(z.colmax));
        MOAO_TRY(sc->mx_norm.ensure(z.norm));
        MOAO_TRY(sc->ws_dinv.ensure(z.dinv));
        MOAO_TRY(sc->ws_w.ensure(z.dinv));
        MOAO_TRY(sc->mx_exps.ensure(z.exps));
        MOAO_TRY(sc->mx_dsl.ensure(z.dsl));
        if (nro > 0) {
          MOAO_TRY(sc->mx_rid.ensure(sizeof(int) * (size_t)in.n));
          MOAO_TRY(sc->mx_y.ensure(sizeof(float) * (size_t)128 * in.n));
          MOAO_TRY(sc->mx_y2.ensure(sizeof(double) * (size_t)nro * in.n));
          MOAO_TRY(sc->mx_zu.ensure(sizeof(double) * (size_t)std::max(in.m, (long)nro) * nro));
          MOAO_TRY(sc->mx_sinv.ensure(sizeof(double) * (size_t)nro * nro));
        }
      } else {
        MOAO_TRY(sc->ws_dinv.ensure(sizeof(double) * (size_t)in.n * in.nb));
        MOAO_TRY(sc->ws_w.ensure(sizeof(double) * (size_t)std::max(in.n, in.m) * in.nb));
      }
      ws = sc->bytes_held();
    }
    MOAO_TRY(sc->ws_info.ensure(3 * sizeof(int)));
    MOAO_TRY(cmm[k].ensure(sizeof(double) * (size_t)nmax * nmax));
    MOAO_TRY(ctm[k].ensure(sizeof(double) * (size_t)mmax * nmax));
    total += ws + cmm[k].bytes + ctm[k].bytes;
  }
  MOAO_TRY(status.ensure(3 * sizeof(int) * (size_t)count));
  MOAO_CUDA_TRY(cudaMemsetAsync(status.p, 0, 3 * sizeof(int) * (size_t)count, ctx->stream));
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  // packed instances: buffers and the task list (host work, before the capture)
  std::vector<PackedInst> pv;
  if (!pk.empty()) {
    MOAO_TRY(pkbuf.ensure(sizeof(double) * std::max<size_t>(pk_data, 1)));
    size_t off = 0;
    for (int i : pk) {
      PackedInst q;
      q.n = inst[i].n;
      q.m = inst[i].m;
      q.A = pkbuf.as<double>() + off;
      q.lda = q.n;
      off += (size_t)q.n * q.n;
      if (items[i].d_R) {
        q.C = items[i].d_R;
      } else {
        q.C = pkbuf.as<double>() + off;
        off += (size_t)q.m * q.n;
      }
      q.ldc = std::max(q.m, 1L);
      q.info = status.as<int>() + 3 * (size_t)i;
      pv.push_back(q);
    }
    MOAO_TRY(packed_prepare(pv, &plan, ctx->stream));
    MOAO_CUDA_TRY(cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking));
    for (int k = 0; k < kCovStreams && k < (int)pk.size(); ++k) {
      cudaStream_t x;
      MOAO_CUDA_TRY(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
      cs.push_back(x);
    }
    total += pk_bytes;
  }

  // ---- capture: fork S streams (and the packed branch) from the context's
  // stream, join at the end. ev[S]: fork; ev[k]: stream k done; ev[S + 1]:
  // packed branch done; ev[S + 2]: the packed branch's covariance fork;
  // ev[S + 3 + c]: its covariance stream c done.
  std::vector<cudaEvent_t> ev(S + 3 + cs.size());
  for (auto& e : ev) MOAO_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  auto destroy_events = [&] {
    for (auto& e : ev) cudaEventDestroy(e);
  };
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const auto host0 = std::chrono::steady_clock::now();
  cudaStream_t s0 = ctx->stream;
  cudaGraph_t graph = nullptr;
  moao_status st = MOAO_OK;
  cudaError_t ce = cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal);
  if (ce == cudaSuccess) ce = cudaEventRecord(ev[S], s0);
  for (int k = 0; k < S && ce == cudaSuccess && st == MOAO_OK; ++k) {
    moao_ctx* sc = subs[k];
    ce = cudaStreamWaitEvent(sc->stream, ev[S], 0);
    for (int i : per[k]) {
      if (ce != cudaSuccess || st != MOAO_OK) break;
      const Inst& in = inst[i];
      st = enqueue_instance(sc, items[in.item].tomo, in, prec, cmm[k].as<double>(),
                            ctm[k].as<double>(), items[in.item].d_R,
                            status.as<int>() + 3 * (size_t)in.item);
    }
    if (ce == cudaSuccess && st == MOAO_OK) ce = cudaEventRecord(ev[k], sc->stream);
    if (ce == cudaSuccess && st == MOAO_OK) ce = cudaStreamWaitEvent(s0, ev[k], 0);
  }
  if (ps && ce == cudaSuccess && st == MOAO_OK) {
    ce = cudaStreamWaitEvent(ps, ev[S], 0);
    if (ce == cudaSuccess) ce = cudaEventRecord(ev[S + 2], ps);
    for (size_t c = 0; c < cs.size() && ce == cudaSuccess; ++c)
      ce = cudaStreamWaitEvent(cs[c], ev[S + 2], 0);
    for (size_t q = 0; q < pk.size() && ce == cudaSuccess && st == MOAO_OK; ++q) {
      const Inst& in = inst[pk[q]];
      cudaStream_t x = cs[q % cs.size()];
      st = launch_matcov(*in.g, pv[q].A, (int)in.n, (int)in.n, 0, 0, (int)pv[q].lda, 1, x,
                         &ctx->launches);
      if (st == MOAO_OK && in.m > 0)
        st = launch_matcov(*in.g, pv[q].C, (int)in.m, (int)in.n, 0, 0, (int)pv[q].ldc, 3, x,
                           &ctx->launches);
    }
    for (size_t c = 0; c < cs.size() && ce == cudaSuccess && st == MOAO_OK; ++c) {
      ce = cudaEventRecord(ev[S + 3 + c], cs[c]);
      if (ce == cudaSuccess) ce = cudaStreamWaitEvent(ps, ev[S + 3 + c], 0);
    }
    if (ce == cudaSuccess && st == MOAO_OK)
      st = packed_launch(plan, ps, ctx->wait_polls, 2.0,
                         &ctx->launches);
    if (ce == cudaSuccess && st == MOAO_OK) ce = cudaEventRecord(ev[S + 1], ps);
    if (ce == cudaSuccess && st == MOAO_OK) ce = cudaStreamWaitEvent(s0, ev[S + 1], 0);
  }
  cudaError_t ce_end = cudaStreamEndCapture(s0, &graph);
  for (int k = 0; k < S; ++k) subs[k]->graph_mode = false;
  if (st != MOAO_OK || ce != cudaSuccess || ce_end != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    destroy_events();
    cudaGetLastError();
    if (st != MOAO_OK) return st;
    return set_error(MOAO_ERR_CUDA, std::string("batch capture: ") +
                                        cudaGetErrorString(ce != cudaSuccess ? ce : ce_end));
  }
  cudaGraphExec_t exec = nullptr;
  ce = cudaGraphInstantiate(&exec, graph, 0);
  size_t nodes = 0;
  cudaGraphGetNodes(graph, nullptr, &nodes);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) {
    destroy_events();
    return set_error(MOAO_ERR_CUDA, std::string("batch graph instantiate: ") + cudaGetErrorString(ce));
  }
  const double build_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - host0).count();
  cudaEventRecord(t0, s0);
  ce = cudaGraphLaunch(exec, s0);
  cudaEventRecord(t1, s0);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(s0);
  float ms = 0;
  cudaEventElapsedTime(&ms, t0, t1);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaGraphExecDestroy(exec);
  destroy_events();
  if (ce != cudaSuccess) return set_error(MOAO_ERR_CUDA, std::string("batch graph launch: ") + cudaGetErrorString(ce));
  std::vector<int> hs(3 * (size_t)count);
  MOAO_CUDA_TRY(cudaMemcpy(hs.data(), status.p, hs.size() * sizeof(int), cudaMemcpyDeviceToHost));
  int pk_err = 0;
  if (!pk.empty())
    MOAO_CUDA_TRY(cudaMemcpy(&pk_err, packed_error_flag(plan), sizeof(int), cudaMemcpyDeviceToHost));
  int failed = 0;
  for (const Inst& in : inst) {
    moao_batch_item& it = items[in.item];
    const int* f = &hs[3 * (size_t)in.item];
    const bool timeout = f[1] || (in.packed && pk_err);
    it.info = f[0];
    it.nb_used = in.packed ? 64 : in.nb;
    it.stream = in.packed ? -1 : in.stream;
    it.packed = in.packed ? 1 : 0;
    it.status = timeout ? MOAO_ERR_TIMEOUT : (f[2] ? MOAO_ERR_BAD_ARG : (f[0] ? MOAO_ERR_NOT_SPD : MOAO_OK));
    failed += it.status != MOAO_OK;
  }
  o->ms_device = ms;
  o->ms_build = build_ms;
  o->graph_nodes = (long long)nodes;
  o->streams_used = S;
  o->device_gb = total / 1e9;
  o->failed = failed;
  o->packed_count = (int)pk.size();
  o->packed_tasks = plan.ntasks;
  return MOAO_OK;
}

}  // namespace
}  // namespace moao

using namespace moao;

extern "C" {

moao_status moao_batch_reconstructors(moao_ctx* ctx, int count, moao_batch_item* items,
                                      moao_batch_opts* opts) {
  if (!ctx || count < 0 || (count > 0 && !items) || !opts)
    return set_error(MOAO_ERR_BAD_ARG, "batch: null argument");
  if (opts->prec != MOAO_PREC_FP64 && opts->prec != MOAO_PREC_MIXED)
    return set_error(MOAO_ERR_BAD_ARG, "batch: precision");
  for (int i = 0; i < count; ++i)
    if (!items[i].tomo) return set_error(MOAO_ERR_BAD_ARG, "batch: item without tomo");
  if (count == 0) return MOAO_OK;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return run_batch(ctx, count, items, opts);
}

moao_status moao_autotune(moao_ctx* ctx, int count, const moao_tomo* const* samples,
                          moao_prec prec, const int* nb_candidates, int ncand) {
  if (!ctx || count <= 0 || !samples || (ncand > 0 && !nb_candidates))
    return set_error(MOAO_ERR_BAD_ARG, "autotune: bad arguments");
  static const int def[] = {128, 256, 384, 512, 768, 1024};
  const int* cand = ncand > 0 ? nb_candidates : def;
  const int nc = ncand > 0 ? ncand : (int)(sizeof(def) / sizeof(def[0]));
  const int p = prec == MOAO_PREC_MIXED;
  std::vector<double> best_ms(kClasses, 1e300);
  std::vector<int> best_nb(kClasses, 0);
  for (int i = 0; i < count; ++i) {
    const long n = samples[i]->t.getNMeas();
    const int c = size_class(n);
    for (int j = 0; j < nc; ++j) {
      if (cand[j] > n) continue;
      moao_batch_item it{};
      it.tomo = samples[i];
      it.nb = cand[j];
      moao_batch_opts o{};
      o.prec = prec;
      o.streams = 1;
      MOAO_TRY(moao_batch_reconstructors(ctx, 1, &it, &o));  // warm-up
      MOAO_TRY(moao_batch_reconstructors(ctx, 1, &it, &o));
      if (o.ms_device < best_ms[c]) {
        best_ms[c] = o.ms_device;
        best_nb[c] = cand[j];
      }
    }
  }
  {
    std::lock_guard<std::mutex> lk(tuning_mutex());
    moao_tuning& t = tuning_tables()[ctx];
    for (int c = 0; c < kClasses; ++c)
      if (best_nb[c] > 0) t.entry[p][c].nb = best_nb[c];
  }
  // FP64 tile configuration of the large products per class, at the class's panel width
  {
    std::vector<double> best_g(kClasses, 1e300);
    std::vector<int> cfg_of(kClasses, 0);
    for (int i = 0; i < count; ++i) {
      const int c = size_class(samples[i]->t.getNMeas());
      for (int g = 0; g < kGemmConfigs; ++g) {
        moao_batch_item it{};
        it.tomo = samples[i];
        moao_batch_opts o{};
        o.prec = prec;
        o.streams = 1;
        o.packed_max = -1;
        o.gemm_tile = g + 1;
        MOAO_TRY(moao_batch_reconstructors(ctx, 1, &it, &o));  // warm-up
        MOAO_TRY(moao_batch_reconstructors(ctx, 1, &it, &o));
        if (o.ms_device < best_g[c]) {
          best_g[c] = o.ms_device;
          cfg_of[c] = g;
        }
      }
    }
    std::lock_guard<std::mutex> lk(tuning_mutex());
    moao_tuning& t = tuning_tables()[ctx];
    for (int c = 0; c < kClasses; ++c)
      if (best_g[c] < 1e300) t.entry[p][c].gemm = cfg_of[c];
  }
  std::vector<moao_batch_item> items(count);
  // packed bound: from the smallest class up, while the class's samples build
  // faster together in the tile-task kernel than as graph instances (classes
  // below 8k only: the task list grows as (nmeas / 64)^3)
  long packed = 0;
  for (int c = 0; c < 3; ++c) {
    std::vector<const moao_tomo*> cls;
    for (int i = 0; i < count; ++i)
      if (size_class(samples[i]->t.getNMeas()) == c) cls.push_back(samples[i]);
    if (cls.empty()) continue;
    double ms[2] = {0, 0};
    for (int mode = 0; mode < 2; ++mode) {
      for (int rep = 0; rep < 2; ++rep) {  // warm-up, then timed
        for (size_t i = 0; i < cls.size(); ++i) {
          items[i] = moao_batch_item{};
          items[i].tomo = cls[i];
        }
        moao_batch_opts o{};
        o.prec = prec;
        o.streams = 2;
        o.packed_max = mode ? class_limit(c) : -1;
        MOAO_TRY(moao_batch_reconstructors(ctx, (int)cls.size(), items.data(), &o));
        ms[mode] = o.ms_device;
      }
    }
    if (ms[1] < ms[0]) packed = class_limit(c) - 1;
    else break;
  }
  {
    std::lock_guard<std::mutex> lk(tuning_mutex());
    tuning_tables()[ctx].packed[p] = packed;
  }
  // stream count: the whole sample set as one batch
  double best = 1e300;
  int bestS = 4;
  for (int S : {2, 4, 8}) {
    if (S > count * 2) break;
    for (int i = 0; i < count; ++i) {
      items[i] = moao_batch_item{};
      items[i].tomo = samples[i];
    }
    moao_batch_opts o{};
    o.prec = prec;
    o.streams = S;
    o.packed_max = packed > 0 ? packed : -1;
    MOAO_TRY(moao_batch_reconstructors(ctx, count, items.data(), &o));
    if (o.ms_device < best) {
      best = o.ms_device;
      bestS = S;
    }
  }
  std::lock_guard<std::mutex> lk(tuning_mutex());
  tuning_tables()[ctx].streams[p] = bestS;
  return MOAO_OK;
}

moao_status moao_tuning_get(moao_ctx* ctx, moao_prec prec, int* nb_per_class, int* streams) {
  if (!ctx || !nb_per_class || !streams) return set_error(MOAO_ERR_BAD_ARG, "tuning_get: null");
  const int p = prec == MOAO_PREC_MIXED;
  for (int c = 0; c < kClasses; ++c) {
    const long n = c == 0 ? 1024 : (1024L << c);
    nb_per_class[c] = tuned_nb(ctx, prec, n);
  }
  *streams = tuned_streams(ctx, prec);
  (void)p;
  return MOAO_OK;
}

moao_status moao_tuning_get_gemm(moao_ctx* ctx, moao_prec prec, int* cfg_per_class) {
  if (!ctx || !cfg_per_class) return set_error(MOAO_ERR_BAD_ARG, "tuning_get_gemm: null");
  for (int c = 0; c < kClasses; ++c) {
    const long n = c == 0 ? 1024 : (1024L << c);
    cfg_per_class[c] = tuned_gemm(ctx, prec, n);
  }
  return MOAO_OK;
}

moao_status moao_tuning_get_packed(moao_ctx* ctx, moao_prec prec, long* packed_max) {
  if (!ctx || !packed_max) return set_error(MOAO_ERR_BAD_ARG, "tuning_get_packed: null");
  *packed_max = tuned_packed(ctx, prec);
  return MOAO_OK;
}

moao_status moao_tuning_save(moao_ctx* ctx, const char* path) {
  if (!ctx || !path) return set_error(MOAO_ERR_BAD_ARG, "tuning_save: null");
  std::ofstream f(path);
  if (!f) return set_error(MOAO_ERR_IO, std::string("tuning_save: cannot create ") + path);
  f << "# moao_b200 tuning: nb prec class width / streams prec n / packed prec nmeas-bound /"
       " gemm prec class tile-configuration\n";
  for (int p = 0; p < 2; ++p) {
    int nbs[kClasses], S = 0;
    const moao_prec pr = p ? MOAO_PREC_MIXED : MOAO_PREC_FP64;
    moao_tuning_get(ctx, pr, nbs, &S);
    for (int c = 0; c < kClasses; ++c) f << "nb " << p << " " << c << " " << nbs[c] << "\n";
    f << "streams " << p << " " << S << "\n";
    f << "packed " << p << " " << tuned_packed(ctx, pr) << "\n";
    int g[kClasses];
    moao_tuning_get_gemm(ctx, pr, g);
    for (int c = 0; c < kClasses; ++c) f << "gemm " << p << " " << c << " " << g[c] << "\n";
  }
  return f ? MOAO_OK : set_error(MOAO_ERR_IO, "tuning_save: write failed");
}

moao_status moao_tuning_load(moao_ctx* ctx, const char* path) {
  if (!ctx || !path) return set_error(MOAO_ERR_BAD_ARG, "tuning_load: null");
  std::ifstream f(path);
  if (!f) return set_error(MOAO_ERR_IO, std::string("tuning_load: cannot open ") + path);
  moao_tuning t;
  std::string line;
  while (std::getline(f, line)) {
    if (line.empty() || line[0] == '#') continue;
    std::istringstream is(line);
    std::string key;
    int p = 0, c = 0, v = 0;
    is >> key;
    if (key == "nb" && (is >> p >> c >> v) && p >= 0 && p < 2 && c >= 0 && c < kClasses &&
        v % 64 == 0 && v >= 64 && v <= 2048)
      t.entry[p][c].nb = v;
    else if (key == "streams" && (is >> p >> v) && p >= 0 && p < 2 && v >= 1 && v <= 16)
      t.streams[p] = v;
    else if (key == "packed" && (is >> p >> v) && p >= 0 && p < 2 && v >= 0)
      t.packed[p] = v;
    else if (key == "gemm" && (is >> p >> c >> v) && p >= 0 && p < 2 && c >= 0 && c < kClasses &&
             v >= 0 && v < kGemmConfigs)
      t.entry[p][c].gemm = v;
    else
      return set_error(MOAO_ERR_IO, "tuning_load: bad line: " + line);
  }
  std::lock_guard<std::mutex> lk(tuning_mutex());
  tuning_tables()[ctx] = t;
  return MOAO_OK;
}

}  // extern "C"
