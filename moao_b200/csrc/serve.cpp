// Serving: a persistent request loop on one GPU.
//
// Requests name a registered system (geometry from its parameter file, plus
// optional Dx and PSF tables) and carry their own turbulence profile and
// target. A scheduler thread admits queued requests in arrival order onto
// worker slots: each slot owns a context (its own stream) whose workspaces
// and device buffers stay resident between requests. A request is admitted
// when a slot is idle and the device bytes it needs fit in the HBM budget
// next to what the other slots hold, so the device work of concurrent
// requests overlaps (continuous batching: a request arriving while others run
// starts as soon as a slot and memory free up, not when the batch drains).
// The head of the queue is never bypassed, so a large request cannot starve.
//
// Per request on its slot: set the profile and target; matcov Cmm (type 1)
// and Ctm (type 3); reconstructor (FP64 or mixed with the model's LGS
// offsets declared); if Cvv is wanted, Ctm and Ctt (type 4) again and Cee/Cvv
// with Cmm (the mixed path leaves Cmm intact; after an FP64 factorisation Cmm
// is regenerated, as the reference's driver does); if the PSF is wanted, the
// intersample step on Cvv; the results the caller asked for are copied to its
// host buffers.
//
// dry_run mode replaces the device work by a timed wait of the request's
// dry_run_ms with the same footprints and admission, for tests without a GPU.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "context.h"
#include "moao_b200.h"

namespace moao {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct System {
  Tomo_struct<double> tomo;  // as registered; slots keep their own copies
  long nmeas = 0, nmeasts = 0, nact = 0;
  std::vector<double> Dx;  // nact x nmeasts
  std::vector<long> idx;
  std::vector<double> abs2fi, otf;
  long np = 0, psf_n = 0;
  bool has_psf = false;
};

struct Request {
  long long id = 0;
  moao_request r{};
  std::vector<double> cn2, h, L0;
  size_t footprint = 0;
  Clock::time_point t_submit, t_start, t_done;
  moao_request_result res{};
  bool done = false, cancelled = false, running = false;
};

// Per-system device state of one slot.
struct SlotSystem {
  std::unique_ptr<moao_tomo> tomo;
  moao_isample* isample = nullptr;
};

struct Slot {
  int index = 0;
  moao_ctx* ctx = nullptr;
  DevBuf cmm, ctm, ctt, cee, cvv, tmp, dx, psf;
  std::map<int, SlotSystem> systems;
  std::shared_ptr<Request> job;
  size_t held = 0;  // device bytes this slot holds (buffers, workspaces, geometry)
  std::thread thread;
};

}  // namespace
}  // namespace moao

struct moao_server {
  moao_server_opts opt{};
  size_t budget = 0;
  std::mutex mu;
  std::condition_variable cv_sched, cv_slot, cv_done;
  std::vector<std::unique_ptr<moao::System>> systems;
  std::deque<std::shared_ptr<moao::Request>> queue;
  std::map<long long, std::shared_ptr<moao::Request>> requests;
  std::vector<std::unique_ptr<moao::Slot>> slots;
  long long next_id = 1;
  bool stopping = false;
  size_t in_flight_bytes = 0;
  moao_server_stats stats{};
  std::thread scheduler;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
};

namespace moao {
namespace {

size_t bytes_of(long a, long b) { return sizeof(double) * (size_t)std::max(a, 0L) * std::max(b, 0L); }

// Device bytes one request needs on a slot: its matrices plus the workspace
// of the chosen path, geometry and intersample state.
size_t footprint(const moao_server* s, const System& sys, const moao_request& r) {
  const long n = sys.nmeas, m = sys.nmeasts, a = sys.nact;
  const long nb = s->opt.nb > 0 ? s->opt.nb : 1024;
  size_t f = bytes_of(n, n) + bytes_of(m, n);
  if (r.prec == MOAO_PREC_MIXED) {
    const int nro = sys.tomo.sys.lgsCst > 0 ? 2 * sys.tomo.sys.nLgs : 0;
    f += mixed_sizes(n, m, nb, 3, 5, nro, true).total();
  } else {
    f += 2 * bytes_of(n, nb);
  }
  const bool cvv = (r.Cvv || r.psf) && a > 0;
  if (cvv) f += 2 * bytes_of(m, m) + bytes_of(a, a) + 3 * bytes_of(a, m) + bytes_of(m, n);
  if (r.psf && sys.has_psf)
    f += bytes_of(sys.psf_n, sys.psf_n) * 7 + sizeof(int) * 2 * (size_t)sys.idx.size();
  // geometry tables (u, v per layer, per-WFS tables)
  f += sizeof(double) * (size_t)sys.tomo.Nx * (2 * (size_t)r.nlayer + 8) + (1 << 20);
  return f;
}

void finish(moao_server* s, Slot& slot, const std::shared_ptr<Request>& q, moao_status st,
            const moao_solve_report& rep, const std::string& err) {
  std::lock_guard<std::mutex> lk(s->mu);
  q->t_done = Clock::now();
  q->res.status = st;
  q->res.info = rep.info;
  q->res.refine_steps = rep.refine_steps;
  q->res.refine_resid = rep.refine_resid;
  q->res.queue_ms = ms_between(q->t_submit, q->t_start);
  q->res.run_ms = ms_between(q->t_start, q->t_done);
  q->res.latency_ms = ms_between(q->t_submit, q->t_done);
  q->res.start_ms = ms_between(s->t0, q->t_start);
  q->res.end_ms = ms_between(s->t0, q->t_done);
  q->res.slot = slot.index;
  std::snprintf(q->res.message, sizeof(q->res.message), "%s", err.c_str());
  q->done = true;
  q->running = false;
  s->in_flight_bytes -= q->footprint;
  if (!s->opt.dry_run && slot.ctx) slot.held = slot.ctx->bytes_held() + slot.cmm.bytes +
                                               slot.ctm.bytes + slot.ctt.bytes + slot.cee.bytes +
                                               slot.cvv.bytes + slot.tmp.bytes + slot.dx.bytes +
                                               slot.psf.bytes;
  if (st == MOAO_OK) ++s->stats.completed;
  else ++s->stats.failed;
  slot.job.reset();
  s->cv_done.notify_all();
  s->cv_sched.notify_all();
}

moao_status run_request(moao_server* s, Slot& slot, Request& q, moao_solve_report* rep) {
  const System& sys = *s->systems[q.r.system];
  moao_ctx* ctx = slot.ctx;
  SlotSystem& ss = slot.systems[q.r.system];
  if (!ss.tomo) {
    ss.tomo.reset(new moao_tomo);
    ss.tomo->t = sys.tomo;
  }
  Tomo_struct<double>& t = ss.tomo->t;
  t.setProfile(q.r.nlayer, q.cn2.data(), q.h.data(), q.L0.data());
  t.setTarget(q.r.target);
  const long n = sys.nmeas, m = sys.nmeasts, a = sys.nact;
  MOAO_TRY(slot.cmm.ensure(bytes_of(n, n)));
  MOAO_TRY(slot.ctm.ensure(bytes_of(m, n)));
  double* Cmm = slot.cmm.as<double>();
  double* Ctm = slot.ctm.as<double>();
  MOAO_TRY(moao_matcov_tile(ctx, ss.tomo.get(), Cmm, (int)n, (int)n, 0, 0, (int)n, 1));
  MOAO_TRY(moao_matcov_tile(ctx, ss.tomo.get(), Ctm, (int)m, (int)n, 0, 0, (int)m, 3));
  const bool mixed = q.r.prec == MOAO_PREC_MIXED;
  if (mixed) MOAO_TRY(moao_ctx_set_offsets_from_tomo(ctx, ss.tomo.get()));
  ctx->keep_cmm = mixed;
  moao_status st = moao_reconstructor(ctx, n, m, Cmm, n, Ctm, m, 1, q.r.prec, rep);
  ctx->keep_cmm = false;
  if (st != MOAO_OK) return st;
  cudaStream_t cs = ctx->stream;
  if (q.r.R)
    MOAO_CUDA_TRY(cudaMemcpyAsync(q.r.R, Ctm, bytes_of(m, n), cudaMemcpyDeviceToHost, cs));
  const bool want_cvv = (q.r.Cvv || q.r.psf) && a > 0;
  if (want_cvv) {
    // R stays in Ctm's buffer; Cee_Cvv destroys its Ctm and Ctt inputs
    MOAO_TRY(slot.ctt.ensure(bytes_of(m, m)));
    MOAO_TRY(slot.cee.ensure(bytes_of(m, m)));
    MOAO_TRY(slot.cvv.ensure(bytes_of(a, a)));
    MOAO_TRY(slot.tmp.ensure(2 * bytes_of(a, m) + bytes_of(m, n)));
    MOAO_TRY(slot.dx.ensure(bytes_of(a, m)));
    double* Ctm2 = slot.tmp.as<double>() + (size_t)a * m;
    double* Tmp = slot.tmp.as<double>();
    MOAO_CUDA_TRY(cudaMemcpyAsync(slot.dx.as<double>(), sys.Dx.data(), bytes_of(a, m),
                                  cudaMemcpyHostToDevice, cs));
    // the FP64 path (or a mixed request that fell back to it) left the factor in Cmm
    if (!mixed || rep->fallback)
      MOAO_TRY(moao_matcov_tile(ctx, ss.tomo.get(), Cmm, (int)n, (int)n, 0, 0, (int)n, 1));
    MOAO_TRY(moao_matcov_tile(ctx, ss.tomo.get(), Ctm2, (int)m, (int)n, 0, 0, (int)m, 3));
    MOAO_TRY(moao_matcov_tile(ctx, ss.tomo.get(), slot.ctt.as<double>(), (int)m, (int)m, 0, 0,
                              (int)m, 4));
    if (mixed && !rep->fallback) {
      // Cee at the refinement's (R_k, E_k): no second R Cmm product (Cee is
      // stationary in R; second-order difference from Cee at the returned R)
      MOAO_TRY(cee_cvv_mixed(ctx, n, m, a, Cmm, n, slot.ctt.as<double>(), m, Ctm2, m, Ctm, m,
                             slot.dx.as<double>(), a, slot.cee.as<double>(), m,
                             slot.cvv.as<double>(), a, Tmp, a, true));
    } else {
      MOAO_TRY(moao_cee_cvv_prec(ctx, n, m, a, Cmm, n, slot.ctt.as<double>(), m, Ctm2, m, Ctm, m,
                                 slot.dx.as<double>(), a, slot.cee.as<double>(), m,
                                 slot.cvv.as<double>(), a, Tmp, a, q.r.prec));
    }
    if (q.r.Cvv)
      MOAO_CUDA_TRY(cudaMemcpyAsync(q.r.Cvv, slot.cvv.as<double>(), bytes_of(a, a),
                                    cudaMemcpyDeviceToHost, cs));
    if (q.r.psf && sys.has_psf) {
      if (!ss.isample)
        MOAO_TRY(moao_intersample_create(ctx, a * a, sys.np, sys.tomo.sys.diam, sys.idx.data(),
                                         sys.abs2fi.data(), sys.otf.data(), &ss.isample));
      MOAO_TRY(slot.psf.ensure(bytes_of(sys.psf_n, sys.psf_n)));
      MOAO_TRY(moao_intersample_process(ss.isample, slot.cvv.as<double>(), slot.psf.as<double>()));
      MOAO_CUDA_TRY(cudaMemcpyAsync(q.r.psf, slot.psf.as<double>(), bytes_of(sys.psf_n, sys.psf_n),
                                    cudaMemcpyDeviceToHost, cs));
    }
  }
  MOAO_CUDA_TRY(cudaStreamSynchronize(cs));
  return MOAO_OK;
}

void slot_main(moao_server* s, Slot* slot) {
  if (!s->opt.dry_run) cudaSetDevice(s->opt.device);
  for (;;) {
    std::shared_ptr<Request> q;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_slot.wait(lk, [&] { return s->stopping || slot->job; });
      if (!slot->job) return;  // stopping
      q = slot->job;
    }
    moao_solve_report rep;
    std::memset(&rep, 0, sizeof(rep));
    moao_status st = MOAO_OK;
    std::string err;
    if (s->opt.dry_run) {
      std::this_thread::sleep_for(std::chrono::duration<double, std::milli>(q->r.dry_run_ms));
    } else {
      st = run_request(s, *slot, *q, &rep);
      if (st != MOAO_OK) err = moao_last_error();
    }
    finish(s, *slot, q, st, rep, err);
  }
}

// Admits queue heads while a slot is idle and the head fits. Called with mu held.
void admit(moao_server* s) {
  while (!s->queue.empty()) {
    std::shared_ptr<Request> q = s->queue.front();
    if (q->cancelled) {
      s->queue.pop_front();
      continue;
    }
    // held bytes of the busy slots are covered by in_flight_bytes of their jobs
    // or by what they hold, whichever is larger; idle slots hold workspaces.
    Slot* best = nullptr;
    size_t best_need = 0;
    size_t total_held = 0;
    for (auto& sl : s->slots) total_held += sl->job ? std::max(sl->held, sl->job->footprint) : sl->held;
    for (auto& sl : s->slots) {
      if (sl->job) continue;
      const size_t need = total_held - sl->held + std::max(sl->held, q->footprint);
      if (need <= s->budget && (!best || need < best_need)) {
        best = sl.get();
        best_need = need;
      }
    }
    if (!best) {
      // free an idle slot's resident buffers if that makes the head fit
      for (auto& sl : s->slots) {
        if (sl->job || sl->held == 0) continue;
        if (total_held - sl->held + q->footprint <= s->budget) {
          if (!s->opt.dry_run) {
            cudaSetDevice(s->opt.device);
            cudaStreamSynchronize(sl->ctx->stream);
            for (DevBuf* b : sl->ctx->workspaces()) b->release();
            for (DevBuf* b : {&sl->cmm, &sl->ctm, &sl->ctt, &sl->cee, &sl->cvv, &sl->tmp, &sl->dx,
                              &sl->psf})
              b->release();
          }
          sl->held = 0;
          best = sl.get();
          best_need = total_held - 0 + q->footprint;
          break;
        }
      }
    }
    if (!best) return;  // wait for a slot or memory
    s->queue.pop_front();
    q->running = true;
    q->t_start = Clock::now();
    q->res.footprint_gb = q->footprint / 1e9;
    s->in_flight_bytes += q->footprint;
    best->job = q;
    if (s->opt.dry_run) best->held = std::max(best->held, q->footprint);
    int busy = 0;
    for (auto& sl : s->slots) busy += sl->job ? 1 : 0;
    s->stats.max_in_flight = std::max(s->stats.max_in_flight, busy);
    size_t admitted = 0;
    for (auto& sl : s->slots) admitted += sl->job ? std::max(sl->held, sl->job->footprint) : sl->held;
    s->stats.peak_admitted_gb = std::max(s->stats.peak_admitted_gb, admitted / 1e9);
    s->cv_slot.notify_all();
  }
}

void scheduler_main(moao_server* s) {
  std::unique_lock<std::mutex> lk(s->mu);
  while (!s->stopping) {
    admit(s);
    s->cv_sched.wait(lk);
  }
}

}  // namespace
}  // namespace moao

using namespace moao;

extern "C" {

moao_status moao_server_create(const moao_server_opts* o, moao_server** out) {
  if (!o || !out) return set_error(MOAO_ERR_BAD_ARG, "server_create: null");
  if (o->slots < 1 || o->slots > 16) return set_error(MOAO_ERR_BAD_ARG, "server_create: 1..16 slots");
  std::unique_ptr<moao_server> s(new moao_server);
  s->opt = *o;
  if (s->opt.queue_capacity <= 0) s->opt.queue_capacity = 4096;
  if (o->hbm_budget_gb > 0) {
    s->budget = (size_t)(o->hbm_budget_gb * 1e9);
  } else if (o->dry_run) {
    return set_error(MOAO_ERR_BAD_ARG, "server_create: dry_run needs an explicit budget");
  } else {
    size_t fr = 0, tot = 0;
    MOAO_CUDA_TRY(cudaSetDevice(o->device));
    MOAO_CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    s->budget = (size_t)(0.9 * (double)fr);
  }
  s->stats.budget_gb = s->budget / 1e9;
  for (int i = 0; i < o->slots; ++i) {
    std::unique_ptr<Slot> sl(new Slot);
    sl->index = i;
    s->slots.push_back(std::move(sl));
    if (!o->dry_run) {
      moao_status st = moao_ctx_create(o->device, &s->slots.back()->ctx);
      if (st == MOAO_OK && o->nb > 0) st = moao_ctx_set_block(s->slots.back()->ctx, o->nb);
      if (st != MOAO_OK) {
        for (auto& x : s->slots)
          if (x->ctx) moao_ctx_destroy(x->ctx);
        return st;
      }
    }
  }
  moao_server* raw = s.get();
  for (auto& sl : s->slots) sl->thread = std::thread(slot_main, raw, sl.get());
  s->scheduler = std::thread(scheduler_main, raw);
  *out = s.release();
  return MOAO_OK;
}

moao_status moao_server_add_system(moao_server* s, const char* sys_file, const char* atm_file,
                                   long nact, const double* Dx, const long* idx,
                                   const double* abs2fi, const double* otf_tel, int* system_id) {
  if (!s || !sys_file || !atm_file || !system_id)
    return set_error(MOAO_ERR_BAD_ARG, "server_add_system: null");
  std::unique_ptr<System> sys(new System);
  try {
    sys->tomo = Tomo_struct<double>(sys_file, atm_file);
  } catch (const std::exception& ex) {
    return set_error(MOAO_ERR_IO, ex.what());
  }
  sys->nmeas = sys->tomo.getNMeas();
  sys->nmeasts = sys->tomo.getNMeasTS();
  if (nact > 0) {
    if (!Dx) return set_error(MOAO_ERR_BAD_ARG, "server_add_system: nact > 0 needs Dx");
    sys->nact = nact;
    sys->Dx.assign(Dx, Dx + (size_t)nact * sys->nmeasts);
    if (idx && abs2fi && otf_tel) {
      sys->has_psf = true;
      sys->np = sys->tomo.Nssp[sys->tomo.sys.nW - 1] + 1;
      sys->psf_n = std::max(512L, (long)(8 * std::pow(2, (long)(std::log((double)sys->np) + 0.5))));
      sys->idx.assign(idx, idx + (size_t)nact * nact);
      sys->abs2fi.assign(abs2fi, abs2fi + (size_t)sys->psf_n * sys->psf_n);
      sys->otf.assign(otf_tel, otf_tel + (size_t)sys->psf_n * sys->psf_n);
    }
  }
  std::lock_guard<std::mutex> lk(s->mu);
  *system_id = (int)s->systems.size();
  s->systems.push_back(std::move(sys));
  return MOAO_OK;
}

moao_status moao_server_add_system_synth(moao_server* s, const char* sys_file,
                                         const char* atm_file, long nact, const double* Dx,
                                         double coupling, int* system_id) {
  if (!s || !sys_file || !atm_file || !system_id || !Dx || nact <= 0)
    return set_error(MOAO_ERR_BAD_ARG, "server_add_system_synth: null or nact <= 0");
  Tomo_struct<double> t;
  try {
    t = Tomo_struct<double>(sys_file, atm_file);
  } catch (const std::exception& ex) {
    return set_error(MOAO_ERR_IO, ex.what());
  }
  const long nssp = t.Nssp[t.sys.nW - 1];
  long na = 0, N = 0;
  MOAO_TRY(moao_intersample_inputs(nullptr, nssp, t.sys.diam, t.sys.obs, coupling, &na, &N,
                                   nullptr, nullptr, nullptr));
  if (na != nact)
    return set_error(MOAO_ERR_BAD_ARG, "server_add_system_synth: the truth sensor's DM has " +
                                           std::to_string(na) + " actuators, Dx has " +
                                           std::to_string(nact) + " rows");
  std::vector<long> idx((size_t)na * na);
  std::vector<double> a((size_t)N * N), o((size_t)N * N);
  if (s->opt.dry_run) {
    MOAO_TRY(moao_intersample_inputs(nullptr, nssp, t.sys.diam, t.sys.obs, coupling, &na, &N,
                                     idx.data(), nullptr, nullptr));
  } else {
    moao_ctx* ctx = nullptr;
    MOAO_TRY(moao_ctx_create(s->opt.device, &ctx));
    const moao_status st = moao_intersample_inputs(ctx, nssp, t.sys.diam, t.sys.obs, coupling, &na,
                                                   &N, idx.data(), a.data(), o.data());
    moao_ctx_destroy(ctx);
    MOAO_TRY(st);
  }
  return moao_server_add_system(s, sys_file, atm_file, nact, Dx, idx.data(), a.data(), o.data(),
                                system_id);
}

moao_status moao_server_system_info(moao_server* s, int system, long* nmeas, long* nmeasts,
                                    long* nact, long* psf_n) {
  if (!s) return set_error(MOAO_ERR_BAD_ARG, "server_system_info: null");
  std::lock_guard<std::mutex> lk(s->mu);
  if (system < 0 || system >= (int)s->systems.size())
    return set_error(MOAO_ERR_BAD_ARG, "server_system_info: unknown system");
  const System& y = *s->systems[system];
  if (nmeas) *nmeas = y.nmeas;
  if (nmeasts) *nmeasts = y.nmeasts;
  if (nact) *nact = y.nact;
  if (psf_n) *psf_n = y.has_psf ? y.psf_n : 0;
  return MOAO_OK;
}

moao_status moao_serve_submit(moao_server* s, const moao_request* r, long long* id) {
  if (!s || !r || !id) return set_error(MOAO_ERR_BAD_ARG, "serve_submit: null");
  if (r->nlayer < 1 || r->nlayer > kMaxLayers || !r->cn2 || !r->h || !r->L0)
    return set_error(MOAO_ERR_BAD_ARG, "serve_submit: profile needs 1..128 layers");
  if (r->prec != MOAO_PREC_FP64 && r->prec != MOAO_PREC_MIXED)
    return set_error(MOAO_ERR_BAD_ARG, "serve_submit: precision");
  std::shared_ptr<Request> q(new Request);
  q->r = *r;
  q->cn2.assign(r->cn2, r->cn2 + r->nlayer);
  q->h.assign(r->h, r->h + r->nlayer);
  q->L0.assign(r->L0, r->L0 + r->nlayer);
  std::lock_guard<std::mutex> lk(s->mu);
  if (r->system < 0 || r->system >= (int)s->systems.size())
    return set_error(MOAO_ERR_BAD_ARG, "serve_submit: unknown system");
  const System& sys = *s->systems[r->system];
  if (r->target < 0 || r->target >= std::max(1, sys.tomo.sys.nTarget))
    return set_error(MOAO_ERR_BAD_ARG, "serve_submit: target out of range");
  if ((r->Cvv || r->psf) && sys.nact == 0)
    return set_error(MOAO_ERR_BAD_ARG, "serve_submit: Cvv/PSF need a system registered with Dx");
  if (r->psf && !sys.has_psf)
    return set_error(MOAO_ERR_BAD_ARG, "serve_submit: PSF needs a system registered with its tables");
  q->footprint = footprint(s, sys, *r);
  if (q->footprint > s->budget) {
    ++s->stats.rejected;
    return set_error(MOAO_ERR_OOM, "serve_submit: request needs " + std::to_string(q->footprint) +
                                       " bytes, above the HBM budget");
  }
  if ((int)s->queue.size() >= s->opt.queue_capacity) {
    ++s->stats.rejected;
    return set_error(MOAO_ERR_BUSY, "serve_submit: queue full");
  }
  q->id = s->next_id++;
  q->t_submit = Clock::now();
  q->res.status = MOAO_ERR_BUSY;
  s->requests[q->id] = q;
  s->queue.push_back(q);
  ++s->stats.submitted;
  *id = q->id;
  s->cv_sched.notify_all();
  return MOAO_OK;
}

moao_status moao_serve_poll(moao_server* s, long long id, moao_request_result* out) {
  if (!s || !out) return set_error(MOAO_ERR_BAD_ARG, "serve_poll: null");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(id);
  if (it == s->requests.end()) return set_error(MOAO_ERR_BAD_ARG, "serve_poll: unknown request");
  const Request& q = *it->second;
  *out = q.res;
  if (q.cancelled) {
    out->status = MOAO_ERR_CANCELLED;
    return MOAO_OK;
  }
  if (!q.done) out->status = MOAO_ERR_BUSY;
  return MOAO_OK;
}

moao_status moao_serve_wait(moao_server* s, long long id, double timeout_s, moao_request_result* out) {
  if (!s || !out) return set_error(MOAO_ERR_BAD_ARG, "serve_wait: null");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->requests.find(id);
  if (it == s->requests.end()) return set_error(MOAO_ERR_BAD_ARG, "serve_wait: unknown request");
  std::shared_ptr<Request> q = it->second;
  const auto pred = [&] { return q->done || q->cancelled; };
  if (timeout_s < 0) s->cv_done.wait(lk, pred);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
    return set_error(MOAO_ERR_TIMEOUT, "serve_wait: request not finished");
  *out = q->res;
  if (q->cancelled) out->status = MOAO_ERR_CANCELLED;
  return MOAO_OK;
}

moao_status moao_serve_cancel(moao_server* s, long long id) {
  if (!s) return set_error(MOAO_ERR_BAD_ARG, "serve_cancel: null");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->requests.find(id);
  if (it == s->requests.end()) return set_error(MOAO_ERR_BAD_ARG, "serve_cancel: unknown request");
  Request& q = *it->second;
  if (q.running || q.done) return set_error(MOAO_ERR_BUSY, "serve_cancel: request already started");
  if (!q.cancelled) {
    q.cancelled = true;
    ++s->stats.cancelled;
    s->cv_done.notify_all();
    s->cv_sched.notify_all();
  }
  return MOAO_OK;
}

moao_status moao_server_get_stats(moao_server* s, moao_server_stats* out) {
  if (!s || !out) return set_error(MOAO_ERR_BAD_ARG, "server_get_stats: null");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->stats;
  return MOAO_OK;
}

void moao_server_destroy(moao_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
    for (auto& q : s->queue) q->cancelled = true;
    s->queue.clear();
  }
  s->cv_sched.notify_all();
  s->cv_slot.notify_all();
  if (s->scheduler.joinable()) s->scheduler.join();
  for (auto& sl : s->slots) {
    // a slot finishes the request it is running before it sees the stop flag
    if (sl->thread.joinable()) sl->thread.join();
    for (auto& kv : sl->systems)
      if (kv.second.isample) moao_intersample_destroy(kv.second.isample);
    for (DevBuf* b : {&sl->cmm, &sl->ctm, &sl->ctt, &sl->cee, &sl->cvv, &sl->tmp, &sl->dx, &sl->psf})
      b->release();
    if (sl->ctx) moao_ctx_destroy(sl->ctx);
  }
  delete s;
}

}  // extern "C"
