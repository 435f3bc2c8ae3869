// C ABI: status strings, system model, device context, covariance entry points
// and the host-buffer variants that keep the reference's in-place contracts.
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

#include "context.h"
#include "dense.h"
#include "mixed.h"

namespace moao {

namespace {
thread_local std::string g_last_error;
}

moao_status set_error(moao_status s, const std::string& msg) {
  g_last_error = msg;
  return s;
}

moao_status DevBuf::ensure(size_t n) {
  if (n <= bytes) return MOAO_OK;
  release();
  cudaError_t e = cudaMalloc(&p, n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    p = nullptr;
    bytes = 0;
    return set_error(MOAO_ERR_OOM, "cudaMalloc of " + std::to_string(n) + " bytes failed: " +
                                       cudaGetErrorString(e));
  }
  bytes = n;
  ++generation;
  return MOAO_OK;
}

void DevBuf::release() {
  if (p) cudaFree(p);
  p = nullptr;
  bytes = 0;
  ++generation;
}

moao_status device_geometry(moao_ctx* ctx, const moao_tomo* tp, const DevGeometry** out) {
  const Tomo_struct<double>& t = tp->t;
  GeomEntry& e = ctx->geom[tp];
  if (e.version == t.version && e.g.nLayer == t.atm.nLayer) {
    *out = &e.g;
    return MOAO_OK;
  }
  const int nW = t.sys.nW, nL = t.atm.nLayer, Nx = t.Nx;
  if (nW > kMaxWfs) return set_error(MOAO_ERR_UNSUPPORTED, "more than 16 WFS");
  if (nL > kMaxLayers) return set_error(MOAO_ERR_UNSUPPORTED, "more than 128 layers");
  DevGeometry g;
  g.nW = nW; g.nLgs = t.sys.nLgs; g.nLayer = nL; g.Nx = Nx;
  g.diam = t.sys.diam; g.lgsCst = t.sys.lgsCst;
  int off = 0;
  for (int w = 0; w < nW; ++w) {
    g.Nsubap[w] = (int)t.Nsubap[w];
    g.off[w] = off;
    g.Nssp[w] = (int)t.Nssp[w];
    off += (int)t.Nsubap[w];
  }
  // One host staging block, one copy.
  const size_t nu = (size_t)nL * Nx;
  const size_t nngs = (size_t)(nW - t.sys.nLgs);
  const size_t nlay = 3 * (size_t)nL + (size_t)nW * nL + nL;
  // per-WFS projection parameters and the subaperture grid of WFS 0
  const double rad = 3.14159265358979323846 / 180.;
  for (int w = 0; w < nW; ++w) {
    g.gsAlt[w] = t.sys.gsAlt[w];
    g.G[w] = t.diamPup[w] / (double)t.Nssp[w];
    g.cth[w] = std::cos(t.sys.thetaML[w] * rad);
    g.sth[w] = std::sin(t.sys.thetaML[w] * rad);
    g.XPup[w] = t.sys.XPup[w];
    g.YPup[w] = t.sys.YPup[w];
    g.alphaX[w] = t.alphaX[w];
    g.alphaY[w] = t.alphaY[w];
  }
  g.nssp_grid = (int)t.Nssp[0];
  g.pitch = t.sys.diam / (1. * t.Nssp[0]);
  const int ngrid = (int)t.Nsubap[0];
  std::vector<int> cr(2 * (size_t)ngrid);
  const double bornemin = -t.sys.diam / 2.;
  for (int i = 0; i < ngrid; ++i) {
    cr[2 * i] = (int)std::lround((t.X[i] - bornemin) / g.pitch - 0.5);
    cr[2 * i + 1] = (int)std::lround((t.Y[i] - bornemin) / g.pitch - 0.5);
  }
  // cell -> valid index of the common grid, and the tiles that hold valid cells
  const int N = g.nssp_grid;
  std::vector<int> cell((size_t)N * N, -1);
  for (int i = 0; i < ngrid; ++i)
    if (cr[2 * i] >= 0 && cr[2 * i] < N && cr[2 * i + 1] >= 0 && cr[2 * i + 1] < N)
      cell[(size_t)cr[2 * i + 1] * N + cr[2 * i]] = i;
  std::vector<int> ta, tb;
  auto tiles = [&](int T, std::vector<int>& out) {
    for (int r0 = 0; r0 < N; r0 += T)
      for (int c0 = 0; c0 < N; c0 += T) {
        bool any = false;
        for (int r = r0; r < std::min(N, r0 + T) && !any; ++r)
          for (int c = c0; c < std::min(N, c0 + T) && !any; ++c) any = cell[(size_t)r * N + c] >= 0;
        if (any) {
          out.push_back(c0);
          out.push_back(r0);
        }
      }
  };
  tiles(4, ta);
  tiles(8, tb);
  g.ntiles_a = (int)ta.size() / 2;
  g.ntiles_b = (int)tb.size() / 2;
  g.bornemin = bornemin;
  for (int w = 0; w < nW; ++w) {
    bool ok = g.G[w] == 1.0 && g.cth[w] == 1.0 && g.sth[w] == 0.0 && t.Nssp[w] == N &&
              t.Nsubap[w] == ngrid && N > 1;
    for (int l = 0; l < nL && ok; ++l) {
      const double sz = t.sspSizeL[(size_t)w * nL + l];
      const double spacing = g.pitch * (1. - t.atm.h[l] * g.gsAlt[w]);
      ok = std::fabs(sz - spacing) <= 1e-12 * std::fabs(sz);
    }
    g.aligned[w] = ok ? 1 : 0;
  }
  int npairs = 0;
  const long ntab = toeplitz_table_doubles(g, &npairs);
  const size_t tab_doubles = npairs ? (size_t)ntab + (size_t)npairs /* pair list */ + 4 : 0;
  const size_t grid_doubles =
      ((size_t)ngrid * 2 * sizeof(int) + cell.size() * sizeof(int) + (ta.size() + tb.size()) * sizeof(int) + 7) / 8;
  const size_t total = 2 * nu + 2 * Nx + 3 * (size_t)Nx + nngs + nlay;
  // table base rounded up to 32 doubles (256 bytes): the gather reads double4
  const size_t tab_off = (total + grid_doubles + 31) / 32 * 32;
  const size_t total_all = tab_off + tab_doubles;
  std::vector<double> h(total);
  size_t p = 0;
  auto put = [&](const double* src, size_t n) {
    std::memcpy(h.data() + p, src, n * sizeof(double));
    size_t at = p;
    p += n;
    return at;
  };
  const size_t ou = put(t.u.data(), nu), ov = put(t.v.data(), nu);
  const size_t oX = put(t.X.data(), Nx), oY = put(t.Y.data(), Nx);
  const size_t oxx = put(t.noiseLGSxx.data(), Nx), oyy = put(t.noiseLGSyy.data(), Nx);
  const size_t oxy = put(t.noiseLGSxy.data(), Nx);
  const size_t ongs = put(t.noiseNGS.data(), nngs);
  const size_t olay = p;
  const double pi = 3.1415926535897932384626433;
  const double k1 = 0.1716613621245709486;
  for (int l = 0; l < nL; ++l) {
    const double L0 = t.L0diff[l];
    h[olay + l] = 2 * pi / L0;                         // rodconan :107
    h[olay + nL + l] = k1 * std::pow(L0, 5. / 3.0);    // rodconan :114
    h[olay + 2 * nL + l] = t.atm.cn2[l];
  }
  for (int k = 0; k < nW * nL; ++k) h[olay + 3 * nL + k] = t.sspSizeL[k];
  for (int l = 0; l < nL; ++l) h[olay + 3 * nL + nW * nL + l] = t.atm.h[l];
  MOAO_TRY(e.buf.ensure(total_all * sizeof(double)));
  double* d = e.buf.as<double>();
  MOAO_CUDA_TRY(cudaMemcpyAsync(d, h.data(), total * sizeof(double), cudaMemcpyHostToDevice,
                                ctx->stream));
  g.grid_cr = reinterpret_cast<int*>(d + total);
  g.cell_idx = g.grid_cr + cr.size();
  g.tiles_a = g.cell_idx + cell.size();
  g.tiles_b = g.tiles_a + ta.size();
  {
    std::vector<int> ints(cr);
    ints.insert(ints.end(), cell.begin(), cell.end());
    ints.insert(ints.end(), ta.begin(), ta.end());
    ints.insert(ints.end(), tb.begin(), tb.end());
    MOAO_CUDA_TRY(cudaMemcpyAsync(g.grid_cr, ints.data(), ints.size() * sizeof(int),
                                  cudaMemcpyHostToDevice, ctx->stream));
    MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // pageable source goes out of scope
  }
  g.ttab = npairs ? d + tab_off : nullptr;
  // h is pageable, so the copy has completed on return from the call above
  // only for small sizes; synchronise before h goes out of scope.
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  g.u = d + ou; g.v = d + ov; g.X = d + oX; g.Y = d + oY;
  g.noiseLGSxx = d + oxx; g.noiseLGSyy = d + oyy; g.noiseLGSxy = d + oxy;
  g.noiseNGS = d + ongs; g.layer = d + olay;
  {
    KernelTimer kt(ctx, "matcov_table", (double)ntab / 4);
    MOAO_TRY(build_toeplitz_tables(g, ctx->stream, &ctx->launches));
  }
  e.g = g;
  e.version = t.version;
  *out = &e.g;
  return MOAO_OK;
}

namespace {
cudaEvent_t take_event(moao_ctx* ctx) {
  if (!ctx->event_pool.empty()) {
    cudaEvent_t e = ctx->event_pool.back();
    ctx->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

KernelTimer::KernelTimer(moao_ctx* ctx, const char* family, double work)
    : ctx_(ctx), family_(family), work_(work) {
  if (!ctx_->timing) return;
  a_ = take_event(ctx_);
  cudaEventRecord(a_, ctx_->stream);
}

KernelTimer::~KernelTimer() {
  if (!a_) return;
  cudaEvent_t b = take_event(ctx_);
  cudaEventRecord(b, ctx_->stream);
  ctx_->pending.push_back({family_, a_, b, work_});
}

moao_status collect_kernel_stats(moao_ctx* ctx) {
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (auto& p : ctx->pending) {
    float ms = 0;
    cudaEventElapsedTime(&ms, p.a, p.b);
    FamilyStats& f = ctx->stats[p.family];
    f.launches += 1;
    f.ms += ms;
    f.work += p.work;
    ctx->event_pool.push_back(p.a);
    ctx->event_pool.push_back(p.b);
  }
  ctx->pending.clear();
  return MOAO_OK;
}

// dst(r, c) = src(r, c) for the elements above the diagonal (r < c) of a
// w x w block (the host path's cached Cmm, moao_reconstructor_host).
__global__ void upper_of_block_kernel(double* __restrict__ dst, long ldd,
                                      const double* __restrict__ src, long w) {
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < w * w;
       e += (long)gridDim.x * blockDim.x) {
    const long r = e % w, c = e / w;
    if (r < c) dst[c * ldd + r] = src[c * w + r];
  }
}

}  // namespace moao

using namespace moao;

extern "C" {

const char* moao_status_string(moao_status s) {
  switch (s) {
    case MOAO_OK: return "MOAO_OK";
    case MOAO_ERR_BAD_ARG: return "MOAO_ERR_BAD_ARG";
    case MOAO_ERR_NOT_SPD: return "MOAO_ERR_NOT_SPD";
    case MOAO_ERR_OOM: return "MOAO_ERR_OOM";
    case MOAO_ERR_CUDA: return "MOAO_ERR_CUDA";
    case MOAO_ERR_IO: return "MOAO_ERR_IO";
    case MOAO_ERR_TIMEOUT: return "MOAO_ERR_TIMEOUT";
    case MOAO_ERR_UNSUPPORTED: return "MOAO_ERR_UNSUPPORTED";
    case MOAO_ERR_BUSY: return "MOAO_ERR_BUSY";
    case MOAO_ERR_CANCELLED: return "MOAO_ERR_CANCELLED";
  }
  return "MOAO_ERR_UNKNOWN";
}

const char* moao_last_error(void) { return g_last_error.c_str(); }

// ---------------------------------------------------------------- system model
moao_status moao_tomo_create(const char* sys_file, const char* atm_file, moao_tomo** out) {
  if (!sys_file || !atm_file || !out) return set_error(MOAO_ERR_BAD_ARG, "tomo_create: null");
  try {
    std::unique_ptr<moao_tomo> t(new moao_tomo);
    t->t = Tomo_struct<double>(sys_file, atm_file);
    if (t->t.Nx <= 0) return set_error(MOAO_ERR_IO, "tomo_create: no valid subaperture");
    *out = t.release();
  } catch (const std::exception& ex) {
    return set_error(MOAO_ERR_IO, ex.what());
  }
  return MOAO_OK;
}

moao_status moao_tomo_update_atm(moao_tomo* t, const char* atm_file) {
  if (!t || !atm_file) return set_error(MOAO_ERR_BAD_ARG, "tomo_update_atm: null");
  try {
    t->t.updateAtm(atm_file);
  } catch (const std::exception& ex) {
    return set_error(MOAO_ERR_IO, ex.what());
  }
  return MOAO_OK;
}

moao_status moao_tomo_set_profile(moao_tomo* t, int nLayer, const double* cn2, const double* h,
                                  const double* L0) {
  if (!t || !cn2 || !h || !L0 || nLayer < 1)
    return set_error(MOAO_ERR_BAD_ARG, "tomo_set_profile: bad arguments");
  for (int l = 0; l < nLayer; ++l)
    if (!(L0[l] > 0) || !std::isfinite(cn2[l]) || !std::isfinite(h[l]))
      return set_error(MOAO_ERR_BAD_ARG, "tomo_set_profile: non-finite layer or L0 <= 0");
  try {
    t->t.setProfile(nLayer, cn2, h, L0);
  } catch (const std::exception& ex) {
    return set_error(MOAO_ERR_BAD_ARG, ex.what());
  }
  return MOAO_OK;
}

moao_status moao_tomo_set_target(moao_tomo* t, int target) {
  if (!t) return set_error(MOAO_ERR_BAD_ARG, "tomo_set_target: null");
  try {
    t->t.setTarget(target);
  } catch (const std::exception& ex) {
    return set_error(MOAO_ERR_BAD_ARG, ex.what());
  }
  return MOAO_OK;
}

moao_status moao_tomo_get_info(const moao_tomo* tp, moao_tomo_info* o) {
  if (!tp || !o) return set_error(MOAO_ERR_BAD_ARG, "tomo_get_info: null");
  const Tomo_struct<double>& t = tp->t;
  o->nW = t.sys.nW;
  o->nLgs = t.sys.nLgs;
  o->nNgs = t.sys.nNgs;
  o->nTarget = t.sys.nTarget;
  o->nLayer = t.atm.nLayer;
  o->Nx = t.Nx;
  o->nmeas = t.getNMeas();
  o->nmeasts = t.getNMeasTS();
  o->diam = t.sys.diam;
  o->obs = t.sys.obs;
  o->lgsCst = t.sys.lgsCst;
  o->nssp_ts = (int)t.Nssp[t.sys.nW - 1];
  return MOAO_OK;
}

long moao_tomo_table(const moao_tomo* tp, const char* name, double* out, long cap) {
  if (!tp || !name) return -1;
  const Tomo_struct<double>& t = tp->t;
  const std::string n(name);
  auto cp = [&](const auto& v) -> long {
    const long len = (long)v.size();
    if (out)
      for (long i = 0; i < len && i < cap; ++i) out[i] = (double)v[i];
    return len;
  };
  if (n == "u") return cp(t.u);
  if (n == "v") return cp(t.v);
  if (n == "X") return cp(t.X);
  if (n == "Y") return cp(t.Y);
  if (n == "sspSizeL") return cp(t.sspSizeL);
  if (n == "L0diff")  // only the first nLayer entries are meaningful
    return cp(std::vector<double>(t.L0diff.begin(), t.L0diff.begin() + t.atm.nLayer));
  if (n == "cn2") return cp(t.atm.cn2);
  if (n == "h") return cp(t.atm.h);
  if (n == "Nsubap") return cp(t.Nsubap);
  if (n == "Nssp") return cp(t.Nssp);
  if (n == "noiseNGS") return cp(t.noiseNGS);
  if (n == "noiseLGSxx") return cp(t.noiseLGSxx);
  if (n == "noiseLGSyy") return cp(t.noiseLGSyy);
  if (n == "noiseLGSxy") return cp(t.noiseLGSxy);
  if (n == "alphaX") return cp(t.alphaX);
  if (n == "alphaY") return cp(t.alphaY);
  if (n == "lgsExt") return cp(t.lgsExt);
  if (n == "lgsTheta") return cp(t.lgsTheta);
  if (n == "mr") return cp(t.mr);
  return -1;
}

void moao_tomo_destroy(moao_tomo* t) { delete t; }

// ---------------------------------------------------------------- context
moao_status moao_ctx_create(int device, moao_ctx** out) {
  if (!out) return set_error(MOAO_ERR_BAD_ARG, "ctx_create: null");
  int n = 0;
  MOAO_CUDA_TRY(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return set_error(MOAO_ERR_BAD_ARG, "ctx_create: no such device");
  MOAO_CUDA_TRY(cudaSetDevice(device));
  std::unique_ptr<moao_ctx> c(new moao_ctx);
  c->device = device;
  MOAO_CUDA_TRY(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
  c->stream = c->own_stream;
  for (auto& e : c->ev) MOAO_CUDA_TRY(cudaEventCreate(&e));
  *out = c.release();
  return MOAO_OK;
}

void moao_ctx_destroy(moao_ctx* c) {
  if (!c) return;
  release_batch_state(c);
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  for (auto& kv : c->geom) kv.second.buf.release();
  for (moao::DevBuf* b : c->workspaces()) b->release();
  for (auto& e : c->ev)
    if (e) cudaEventDestroy(e);
  for (auto& p : c->pending) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto e : c->event_pool) cudaEventDestroy(e);
  for (auto& e : c->la_ev)
    if (e) cudaEventDestroy(e);
  if (c->aux) {
    cudaStreamSynchronize(c->aux);
    cudaStreamDestroy(c->aux);
  }
  if (c->copy) {
    cudaStreamSynchronize(c->copy);
    cudaStreamDestroy(c->copy);
  }
  for (auto e : c->copy_ev) cudaEventDestroy(e);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
}

moao_status moao_ctx_set_stream(moao_ctx* c, void* stream) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_stream: null");
  c->stream = static_cast<cudaStream_t>(stream);
  return MOAO_OK;
}

moao_status moao_ctx_use_own_stream(moao_ctx* c) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_use_own_stream: null");
  c->stream = c->own_stream;
  return MOAO_OK;
}

void* moao_ctx_stream(moao_ctx* c) { return c ? (void*)c->stream : nullptr; }

moao_status moao_ctx_synchronize(moao_ctx* c) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_synchronize: null");
  MOAO_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return MOAO_OK;
}

long long moao_ctx_launch_count(const moao_ctx* c) { return c ? c->launches : 0; }

moao_status moao_ctx_set_kernel_timing(moao_ctx* c, int enable) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_kernel_timing: null");
  std::lock_guard<std::mutex> lk(c->mu);
  c->timing = enable != 0;
  return MOAO_OK;
}

moao_status moao_ctx_kernel_stats(moao_ctx* c, const char* family, long long* launches,
                                  double* ms, double* work) {
  if (!c || !family) return set_error(MOAO_ERR_BAD_ARG, "ctx_kernel_stats: null");
  std::lock_guard<std::mutex> lk(c->mu);
  MOAO_CUDA_TRY(cudaSetDevice(c->device));
  MOAO_TRY(collect_kernel_stats(c));
  FamilyStats f;
  auto it = c->stats.find(family);
  if (it != c->stats.end()) f = it->second;
  if (launches) *launches = f.launches;
  if (ms) *ms = f.ms;
  if (work) *work = f.work;
  return MOAO_OK;
}

moao_status moao_ctx_reset_kernel_stats(moao_ctx* c) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_reset_kernel_stats: null");
  std::lock_guard<std::mutex> lk(c->mu);
  MOAO_CUDA_TRY(cudaSetDevice(c->device));
  MOAO_TRY(collect_kernel_stats(c));
  c->stats.clear();
  return MOAO_OK;
}

moao_status moao_ctx_set_mixed(moao_ctx* c, int bf16_slices, int corr_slices, int ozaki_slices,
                               int max_refine, double tol, int final_residual) {
  if (!c || bf16_slices < 2 || bf16_slices > 3 || corr_slices < 0 || corr_slices > bf16_slices ||
      ozaki_slices < 2 || ozaki_slices > 6 || max_refine < 0 || max_refine > 8 || tol < 0)
    return set_error(MOAO_ERR_BAD_ARG,
                     "ctx_set_mixed: bf16 slices in [2, 3], correction slices in [0, bf16 slices], "
                     "int8 slices in [2, 6], max_refine in [0, 8]");
  std::lock_guard<std::mutex> lk(c->mu);
  c->bf16_slices = bf16_slices;
  c->corr_slices = corr_slices;
  c->ozaki_slices = ozaki_slices;
  c->max_refine = max_refine;
  c->refine_tol = tol;
  c->final_residual = final_residual != 0;
  c->mx_factored_n = -1;
  return MOAO_OK;
}

moao_status moao_ctx_set_offsets(moao_ctx* c, int nranges, const int* begin, const int* end,
                                 const double* value) {
  if (!c || nranges < 0 || nranges > kMaxOffsetRanges || (nranges > 0 && (!begin || !end || !value)))
    return set_error(MOAO_ERR_BAD_ARG, "ctx_set_offsets: 0..32 ranges with begin, end and value");
  OffsetRanges o;
  for (int w = 0; w < nranges; ++w) {
    if (begin[w] < 0 || end[w] <= begin[w] || !(value[w] > 0) || !std::isfinite(value[w]))
      return set_error(MOAO_ERR_BAD_ARG, "ctx_set_offsets: range " + std::to_string(w) +
                                             " needs 0 <= begin < end and a finite value > 0");
    for (int v = 0; v < w; ++v)
      if (begin[w] < end[v] && begin[v] < end[w])
        return set_error(MOAO_ERR_BAD_ARG, "ctx_set_offsets: ranges overlap");
    o.begin[o.n] = begin[w];
    o.end[o.n] = end[w];
    o.value[o.n] = value[w];
    ++o.n;
  }
  std::lock_guard<std::mutex> lk(c->mu);
  c->offsets = o;
  c->mx_factored_n = -1;
  return MOAO_OK;
}

moao_status moao_ctx_set_offsets_from_tomo(moao_ctx* c, const moao_tomo* tp) {
  if (!c || !tp) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_offsets_from_tomo: null argument");
  const Tomo_struct<double>& t = tp->t;
  std::vector<int> b, e;
  std::vector<double> v;
  const double cst = t.sys.lgsCst;
  if (cst > 0) {
    // Cmm rows: WFS w holds x slopes [base, base + Nsubap) then y slopes; the
    // LGS constant sits on every xx and yy entry of an LGS's own block.
    long base = 0;
    for (int w = 0; w + 1 < t.sys.nW; ++w) {
      const long ns = t.Nsubap[w];
      if (w < t.sys.nLgs) {
        b.push_back((int)base); e.push_back((int)(base + ns)); v.push_back(cst);
        b.push_back((int)(base + ns)); e.push_back((int)(base + 2 * ns)); v.push_back(cst);
      }
      base += 2 * ns;
    }
  }
  return moao_ctx_set_offsets(c, (int)b.size(), b.data(), e.data(), v.data());
}

moao_status moao_ctx_set_factor_format(moao_ctx* c, int format) {
  if (!c || (format != MOAO_FACTOR_BF16X3 && format != MOAO_FACTOR_F16X2))
    return set_error(MOAO_ERR_BAD_ARG, "ctx_set_factor_format: BF16X3 or F16X2");
  std::lock_guard<std::mutex> lk(c->mu);
  c->factor_format = format;
  c->mx_factored_n = -1;
  return MOAO_OK;
}

moao_status moao_ctx_set_lookahead(moao_ctx* c, int sms) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_lookahead: null");
  if (sms < 0 || sms > 64) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_lookahead: 0..64 SMs");
  std::lock_guard<std::mutex> lk(c->mu);
  c->lookahead_sms = sms;
  return MOAO_OK;
}

moao_status moao_ctx_set_accuracy(moao_ctx* c, double target) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_accuracy: null");
  if (!(target >= 0.0)) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_accuracy: target >= 0");
  std::lock_guard<std::mutex> lk(c->mu);
  c->acc_target = target;
  return MOAO_OK;
}

moao_status moao_ctx_set_wait_limit(moao_ctx* c, long long polls) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_wait_limit: null");
  if (polls < 0) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_wait_limit: polls >= 0");
  std::lock_guard<std::mutex> lk(c->mu);
  c->wait_polls = (unsigned long long)polls;
  return MOAO_OK;
}

moao_status moao_ctx_set_gemm_tile(moao_ctx* c, int cfg) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_gemm_tile: null");
  if (cfg < 0 || cfg >= kGemmConfigs) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_gemm_tile: 0..3");
  std::lock_guard<std::mutex> lk(c->mu);
  c->gemm_cfg = cfg;
  return MOAO_OK;
}

moao_status moao_ctx_set_residual(moao_ctx* c, int scheme) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_residual: null");
  if (scheme != 0 && scheme != 1)
    return set_error(MOAO_ERR_BAD_ARG, "ctx_set_residual: 0 (slice products) or 1 (CRT)");
  std::lock_guard<std::mutex> lk(c->mu);
  c->residual_crt = scheme;
  c->mx_factored_n = -1;  // a kept factorisation holds the other scheme's operands
  c->rstate_valid = false;
  return MOAO_OK;
}

moao_status moao_debug_residual(moao_ctx* c, int scheme, long m, long n, const double* R, long ldR,
                                const double* Cmm, long ldCmm, const double* Ctm, long ldCtm,
                                double* E, long ldE) {
  if (!c || !R || !Cmm || !Ctm || !E || m <= 0 || n <= 0 || ldR < m || ldCmm < n || ldCtm < m ||
      ldE < m || (scheme != 0 && scheme != 1))
    return set_error(MOAO_ERR_BAD_ARG, "debug_residual: bad arguments");
  std::lock_guard<std::mutex> lk(c->mu);
  MOAO_CUDA_TRY(cudaSetDevice(c->device));
  return debug_residual(c, scheme, m, n, R, ldR, Cmm, ldCmm, Ctm, ldCtm, E, ldE);
}

int moao_debug_crt_moduli(int ns, long K) { return crt_moduli_for(ns, K); }

moao_status moao_ctx_set_tc_pair(moao_ctx* c, int on) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_tc_pair: null");
  std::lock_guard<std::mutex> lk(c->mu);
  c->tc_pair = on != 0;
  return MOAO_OK;
}

moao_status moao_ctx_set_host_cache(moao_ctx* c, int on) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_host_cache: null");
  std::lock_guard<std::mutex> lk(c->mu);
  c->host_cache = on != 0;
  c->cache_cmm = moao_ctx::HostTile{};
  c->cache_ctm = moao_ctx::HostTile{};
  return MOAO_OK;
}

moao_status moao_ctx_set_lookahead_max(moao_ctx* c, int sms) {
  if (!c) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_lookahead_max: null");
  if (sms < 0 || sms > 120) return set_error(MOAO_ERR_BAD_ARG, "ctx_set_lookahead_max: 0..120 SMs");
  std::lock_guard<std::mutex> lk(c->mu);
  c->lookahead_max = sms;
  return MOAO_OK;
}

moao_status moao_ctx_set_host_precision(moao_ctx* c, moao_prec prec) {
  if (!c || (prec != MOAO_PREC_FP64 && prec != MOAO_PREC_MIXED))
    return set_error(MOAO_ERR_BAD_ARG, "ctx_set_host_precision: FP64 or MIXED");
  c->host_prec = prec;
  return MOAO_OK;
}

moao_status moao_ctx_set_block(moao_ctx* c, int nb) {
  if (!c || nb < 64 || nb % 64 != 0 || nb > 2048)
    return set_error(MOAO_ERR_BAD_ARG, "ctx_set_block: nb must be a multiple of 64 in [64, 2048]");
  std::lock_guard<std::mutex> lk(c->mu);
  c->nb = nb;
  c->mx_factored_n = -1;
  return MOAO_OK;
}

// ---------------------------------------------------------------- matcov
moao_status moao_matcov_tile(moao_ctx* ctx, const moao_tomo* t, double* d_data, int nrows,
                             int ncols, int xoffset, int yoffset, int lda, int type_mat) {
  if (!ctx || !t) return set_error(MOAO_ERR_BAD_ARG, "matcov_tile: null");
  std::lock_guard<std::mutex> lk(ctx->mu);
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  const DevGeometry* g = nullptr;
  MOAO_TRY(device_geometry(ctx, t, &g));
  double elems = (double)nrows * ncols;
  if (type_mat == 1 && xoffset == yoffset && nrows == ncols) elems = 0.5 * nrows * (nrows + 1.0);
  KernelTimer kt(ctx, "matcov", elems);
  return launch_matcov(*g, d_data, nrows, ncols, xoffset, yoffset, lda, type_mat, ctx->stream,
                       &ctx->launches);
}

namespace {

// Copies, column panel by column panel (width w), the part of an nrows x ncols
// column-major tile whose local row r and column c satisfy r >= c - d (d = the
// tile's global row offset minus its global column offset): exactly the
// elements a type-1 (lower) covariance tile writes and the lower factor
// occupies. Each panel [c0, c1) is copied from its first such row down to the
// last row, which includes, inside the panel, the elements above the boundary;
// with corner_only only those first rows (the panel's diagonal block, where
// the untouched elements lie) are copied.
moao_status copy_lower_panels(double* dst, long ldd, const double* src, long lds, long nrows,
                              long ncols, long d, bool corner_only, cudaMemcpyKind kind,
                              cudaStream_t s) {
  const long w = 512;
  for (long c0 = 0; c0 < ncols; c0 += w) {
    const long c1 = std::min(ncols, c0 + w);
    const long r0 = std::max(0L, c0 - d);
    if (r0 >= nrows) break;  // later panels start lower still
    const long r1 = corner_only ? std::min(nrows, std::max(r0, c1 - d)) : nrows;
    if (r1 <= r0) continue;
    MOAO_CUDA_TRY(cudaMemcpy2DAsync(dst + c0 * ldd + r0, sizeof(double) * ldd,
                                    src + c0 * lds + r0, sizeof(double) * lds,
                                    sizeof(double) * (r1 - r0), c1 - c0, kind, s));
  }
  return MOAO_OK;
}

// The caller's elements above the diagonal inside the diagonal blocks of the
// 512-column panels of an n x n matrix (the only upper elements that the lower
// panel copies carry), brought down into dst without touching anything else.
moao_status upload_panel_uppers(double* dst, long ldd, const double* src, long lds, long n,
                                DevBuf& stage, cudaStream_t s, long long* launches) {
  const long w = 512;
  MOAO_TRY(stage.ensure(sizeof(double) * (size_t)w * w));
  for (long c0 = 0; c0 < n; c0 += w) {
    const long b = std::min(w, n - c0);
    MOAO_CUDA_TRY(cudaMemcpy2DAsync(stage.p, sizeof(double) * b, src + c0 * lds + c0,
                                    sizeof(double) * lds, sizeof(double) * b, b,
                                    cudaMemcpyHostToDevice, s));
    upper_of_block_kernel<<<(unsigned)std::min<long>((b * b + 255) / 256, 1024), 256, 0, s>>>(
        dst + c0 * ldd + c0, ldd, stage.as<double>(), b);
    MOAO_CUDA_TRY(cudaGetLastError());
    if (launches) ++*launches;
  }
  return MOAO_OK;
}

}  // namespace

moao_status moao_matcov_tile_host(moao_ctx* ctx, const moao_tomo* t, double* h_data, int nrows,
                                  int ncols, int xoffset, int yoffset, int lda, int type_mat) {
  if (!ctx || !t || !h_data) return set_error(MOAO_ERR_BAD_ARG, "matcov_tile_host: null");
  if (nrows <= 0 || ncols <= 0) return MOAO_OK;
  if (lda < nrows) return set_error(MOAO_ERR_BAD_ARG, "matcov_tile_host: lda < nrows");
  std::lock_guard<std::mutex> lk(ctx->mu);
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  const DevGeometry* g = nullptr;
  MOAO_TRY(device_geometry(ctx, t, &g));
  if (type_mat != 1 && type_mat != 2 && type_mat != 3 && type_mat != 4 && type_mat != 5)
    return set_error(MOAO_ERR_BAD_ARG, "matcov_tile_host: unknown type_mat " +
                                           std::to_string(type_mat));
  const size_t bytes = sizeof(double) * (size_t)nrows * ncols;
  // With the host cache a whole type-3 tile (Ctm) is generated in the Ctm
  // workspace of moao_reconstructor_host, so that a whole Cmm left in ws_tmp
  // survives it; every other tile goes through ws_tmp.
  const bool whole_cmm = type_mat == 1 && xoffset == 0 && yoffset == 0 && nrows == ncols;
  const bool ctm_ws = ctx->host_cache && type_mat == 3 && xoffset == 0 && yoffset == 0;
  DevBuf& buf = ctm_ws ? ctx->ws_host_t : ctx->ws_tmp;
  MOAO_TRY(buf.ensure(bytes));
  double* d = buf.as<double>();
  cudaStream_t s = ctx->stream;
  if (ctm_ws) ctx->cache_ctm = moao_ctx::HostTile{};
  else ctx->cache_cmm = moao_ctx::HostTile{};
  // Column blocks at the WFS boundaries of the columns (types 1 and 3 have WFS
  // slopes as columns and write only inside their own columns; a block holds both
  // slope axes of its WFS, so no pair's stencils are evaluated twice): block b is
  // generated on the context stream while block b - 1 is copied back on the copy
  // stream. Type 5 mirrors into other columns and stays one block.
  std::vector<long> cuts{0};
  if (type_mat == 1 || type_mat == 3) {
    long b = 0;
    const Tomo_struct<double>& tt = t->t;
    for (int w = 0; w + 1 < tt.sys.nW; ++w) {
      b += 2 * tt.Nsubap[w];
      const long c = b - yoffset;
      if (c > 0 && c < ncols) cuts.push_back(c);
    }
  }
  cuts.push_back(ncols);
  if (!ctx->copy) MOAO_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
  while (ctx->copy_ev.size() < cuts.size()) {
    cudaEvent_t e;
    MOAO_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->copy_ev.push_back(e);
  }
  const long dd = (long)xoffset - yoffset;
  for (size_t k = 0; k + 1 < cuts.size(); ++k) {
    const long c0 = cuts[k], w = cuts[k + 1] - c0;
    double* dk = d + c0 * nrows;
    double* hk = h_data + c0 * (long)lda;
    if (type_mat == 1) {
      // A type-1 tile writes only elements on or below the global diagonal; the
      // others keep the caller's values. Only the panels' diagonal blocks (where
      // both kinds meet) go down, and only the written panels come back.
      MOAO_TRY(copy_lower_panels(dk, nrows, hk, lda, nrows, w, dd - c0, true,
                                 cudaMemcpyHostToDevice, s));
    }
    MOAO_TRY(launch_matcov(*g, dk, nrows, (int)w, xoffset, yoffset + (int)c0, nrows, type_mat, s,
                           &ctx->launches));
    MOAO_CUDA_TRY(cudaEventRecord(ctx->copy_ev[k], s));
    MOAO_CUDA_TRY(cudaStreamWaitEvent(ctx->copy, ctx->copy_ev[k], 0));
    if (type_mat == 1) {
      MOAO_TRY(copy_lower_panels(hk, lda, dk, nrows, nrows, w, dd - c0, false,
                                 cudaMemcpyDeviceToHost, ctx->copy));
    } else {
      // every element of the block is written
      MOAO_CUDA_TRY(cudaMemcpy2DAsync(hk, sizeof(double) * lda, dk, sizeof(double) * nrows,
                                      sizeof(double) * nrows, w, cudaMemcpyDeviceToHost,
                                      ctx->copy));
    }
  }
  MOAO_CUDA_TRY(cudaStreamSynchronize(s));
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->copy));
  if (ctx->host_cache && (whole_cmm || ctm_ws)) {
    moao_ctx::HostTile& c = ctm_ws ? ctx->cache_ctm : ctx->cache_cmm;
    c.h = h_data;
    c.ld = lda;
    c.rows = nrows;
    c.cols = ncols;
    c.gen = buf.generation;
  }
  return MOAO_OK;
}

// ---------------------------------------------------------------- host variants
moao_status moao_reconstructor_host(moao_ctx* ctx, long nmeas, long nmeasts, double* Cmm,
                                    long ldCmm, double* Ctm, long ldCtm, long ngal,
                                    moao_solve_report* rep) {
  if (!ctx || !Cmm || !Ctm) return set_error(MOAO_ERR_BAD_ARG, "reconstructor_host: null");
  if (nmeas <= 0 || nmeasts <= 0 || ngal <= 0 || ldCmm < nmeas || ldCtm < nmeasts)
    return set_error(MOAO_ERR_BAD_ARG, "reconstructor_host: bad sizes");
  const size_t tspan = (size_t)nmeas * nmeasts * (ngal - 1) + (size_t)ldCtm * (nmeas - 1) + nmeasts;
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  double *dC = nullptr, *dT = nullptr;
  bool cmm_cached = false, ctm_cached = false;
  {
    // device copies in the context's workspaces (kept for the next call)
    std::lock_guard<std::mutex> lk(ctx->mu);
    MOAO_TRY(ctx->ws_tmp.ensure(sizeof(double) * (size_t)nmeas * nmeas));
    MOAO_TRY(ctx->ws_host_t.ensure(sizeof(double) * tspan));
    dC = ctx->ws_tmp.as<double>();
    dT = ctx->ws_host_t.as<double>();
    if (ctx->host_cache) {
      // what moao_matcov_tile_host generated into these very buffers for these
      // host buffers (the caller promised not to change them since)
      const moao_ctx::HostTile &a = ctx->cache_cmm, &b = ctx->cache_ctm;
      cmm_cached = a.h == Cmm && a.ld == ldCmm && a.rows == nmeas && a.cols == nmeas &&
                   a.gen == ctx->ws_tmp.generation;
      ctm_cached = b.h == Ctm && ngal == 1 && b.ld == ldCtm && ldCtm == nmeasts &&
                   b.rows == nmeasts && b.cols == nmeas && b.gen == ctx->ws_host_t.generation;
    }
    ctx->cache_cmm = moao_ctx::HostTile{};  // the buffers now become the factor and R
    ctx->cache_ctm = moao_ctx::HostTile{};
  }
  cudaStream_t s = ctx->stream;
  if (!ctx->copy) MOAO_CUDA_TRY(cudaStreamCreateWithFlags(&ctx->copy, cudaStreamNonBlocking));
  if (!ctx->inputs_ready)
    MOAO_CUDA_TRY(cudaEventCreateWithFlags(&ctx->inputs_ready, cudaEventDisableTiming));
  // Only the lower triangle of Cmm is read and only its lower triangle becomes
  // the factor: the column panels of the lower part go down and come back (the
  // panels' diagonal blocks carry their upper elements unchanged both ways).
  // Ctm goes down on the copy stream while the factorisation runs (the solves
  // wait for it), and the factor comes back on the copy stream while the solves
  // run.
  // A cached Cmm still takes the caller's elements above the diagonal inside
  // the panels' diagonal blocks (the covariance tile never wrote them, and they
  // go back with the factor's panels); nothing of the lower part is read.
  if (cmm_cached)
    MOAO_TRY(upload_panel_uppers(dC, nmeas, Cmm, ldCmm, nmeas, ctx->ws_corner, s,
                                 &ctx->launches));
  else
    MOAO_TRY(copy_lower_panels(dC, nmeas, Cmm, ldCmm, nmeas, nmeas, 0, false,
                               cudaMemcpyHostToDevice, s));
  if (!ctm_cached)
    MOAO_CUDA_TRY(cudaMemcpyAsync(dT, Ctm, sizeof(double) * tspan, cudaMemcpyHostToDevice,
                                  ctx->copy));
  MOAO_CUDA_TRY(cudaEventRecord(ctx->inputs_ready, ctx->copy));
  ctx->wait_inputs = true;
  ctx->host_factor = Cmm;
  ctx->host_factor_ld = ldCmm;
  const moao_status st =
      moao_reconstructor(ctx, nmeas, nmeasts, dC, nmeas, dT, ldCtm, ngal, ctx->host_prec, rep);
  const bool factor_sent = ctx->factor_done;
  ctx->wait_inputs = false;
  ctx->host_factor = nullptr;
  ctx->factor_done = false;
  // the stream must not run ahead of Ctm's copy on any path (errors included)
  MOAO_CUDA_TRY(cudaStreamWaitEvent(s, ctx->inputs_ready, 0));
  // On a failed factorisation the reference has already overwritten Cmm
  // (partially) and leaves Ctm alone; mirror that.
  if ((st == MOAO_OK || st == MOAO_ERR_NOT_SPD) && !factor_sent)
    MOAO_TRY(copy_lower_panels(Cmm, ldCmm, dC, nmeas, nmeas, nmeas, 0, false,
                               cudaMemcpyDeviceToHost, s));
  if (st == MOAO_OK)
    MOAO_CUDA_TRY(cudaMemcpyAsync(Ctm, dT, sizeof(double) * tspan, cudaMemcpyDeviceToHost, s));
  MOAO_CUDA_TRY(cudaStreamSynchronize(s));
  MOAO_CUDA_TRY(cudaStreamSynchronize(ctx->copy));
  return st;
}

moao_status moao_cee_cvv_host(moao_ctx* ctx, long nmeas, long nmeasts, long nact, double* Cmm,
                              long ldCmm, double* Cpp, long ldCpp, double* Cpm, long ldCpm,
                              double* R, long ldR, double* Dx, long ldDx, double* Cee,
                              long ldCee, double* Cvv, long ldCvv, double* Tmp, long ldTmp) {
  if (!ctx) return set_error(MOAO_ERR_BAD_ARG, "Cee_Cvv_host: null");
  struct Mat { double* h; long ld, m, n; double* d; bool in, out; };
  Mat mats[] = {{Cmm, ldCmm, nmeas, nmeas, nullptr, true, false},
                {Cpp, ldCpp, nmeasts, nmeasts, nullptr, true, true},
                {Cpm, ldCpm, nmeasts, nmeas, nullptr, true, true},
                {R, ldR, nmeasts, nmeas, nullptr, true, false},
                {Dx, ldDx, nact, nmeasts, nullptr, true, false},
                {Cee, ldCee, nmeasts, nmeasts, nullptr, false, true},
                {Cvv, ldCvv, nact, nact, nullptr, false, true},
                {Tmp, ldTmp, nact, nmeasts, nullptr, false, true}};
  for (auto& m : mats)
    if (!m.h || m.ld < std::max(1L, m.m) || m.m < 0 || m.n < 0)
      return set_error(MOAO_ERR_BAD_ARG, "Cee_Cvv_host: bad matrix argument");
  MOAO_CUDA_TRY(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  moao_status st = MOAO_OK;
  for (auto& m : mats) {
    if (cudaMalloc(&m.d, sizeof(double) * std::max(1L, m.m * m.n)) != cudaSuccess) {
      st = set_error(MOAO_ERR_OOM, "Cee_Cvv_host: device allocation");
      break;
    }
    if (m.in && m.m * m.n > 0 &&
        cudaMemcpy2DAsync(m.d, sizeof(double) * m.m, m.h, sizeof(double) * m.ld,
                          sizeof(double) * m.m, m.n, cudaMemcpyHostToDevice, s) != cudaSuccess) {
      st = set_error(MOAO_ERR_CUDA, "Cee_Cvv_host: H2D");
      break;
    }
  }
  if (st == MOAO_OK)
    st = moao_cee_cvv_prec(ctx, nmeas, nmeasts, nact, mats[0].d, std::max(1L, nmeas), mats[1].d,
                           std::max(1L, nmeasts), mats[2].d, std::max(1L, nmeasts), mats[3].d,
                           std::max(1L, nmeasts), mats[4].d, std::max(1L, nact), mats[5].d,
                           std::max(1L, nmeasts), mats[6].d, std::max(1L, nact), mats[7].d,
                           std::max(1L, nact), ctx->host_prec);
  if (st == MOAO_OK)
    for (auto& m : mats)
      if (m.out && m.m * m.n > 0 &&
          cudaMemcpy2DAsync(m.h, sizeof(double) * m.ld, m.d, sizeof(double) * m.m,
                            sizeof(double) * m.m, m.n, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        st = set_error(MOAO_ERR_CUDA, "Cee_Cvv_host: D2H");
  cudaStreamSynchronize(s);
  for (auto& m : mats)
    if (m.d) cudaFree(m.d);
  return st;
}

}  // extern "C"
