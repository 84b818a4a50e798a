// hj_api.cu -- C ABI of the tracking library (include/haissinski_gpu.h).
//
// Host orchestration of the device kernels.  A run is a "bunch": its state
// z/dE stays on the device; per turn the host only enqueues three kernels
// (particle pass, histogram reduction, bins step) whose turn-to-turn state
// (E0, pending kick, turn counter) lives in device memory, so turns never
// wait for the host.
#include <memory>
#include "hj_state.h"

namespace {
const char* kVersion = "haissinski-b200 0.1.0 (sm_100a)";
}  // namespace

namespace hj_impl {

hj_status set_err(hj_ctx* ctx, hj_status code, const char* fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return code;
}




int64_t next_pow2(int64_t n) {
  if (n <= 0) return 1;
  int64_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

int ilog2(int64_t v) {
  int l = 0;
  while ((int64_t(1) << l) < v) ++l;
  return l;
}

// compute_global_std from sums (src/utils.jl:593-605).
double global_std(double s, double s2, int64_t n) {
  if (n <= 1) return 0.0;
  const double nd = (double)n;
  const double mean = s / nd;
  const double var = (s2 / nd) - (mean * mean);
  double sv = var * nd / (double)(n - 1);
  if (!(sv > 0.0)) sv = (sv != sv) ? sv : 0.0;
  return std::sqrt(sv);
}

hj_status ctx_ok(hj_ctx* ctx) {
  if (!ctx) return HJ_ERR_ARG;
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess)
    return set_err(ctx, HJ_ERR_CUDA, "cudaSetDevice(%d): %s", ctx->device, cudaGetErrorString(e));
  ctx->err.clear();
  return HJ_OK;
}

hj_status scratch(hj_ctx* ctx, size_t bytes, void** out) {
  if (bytes > ctx->scratch_bytes) {
    if (ctx->scratch) cudaFree(ctx->scratch);
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    cudaError_t e = cudaMalloc(&ctx->scratch, bytes);
    if (e != cudaSuccess)
      return set_err(ctx, HJ_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes,
                     cudaGetErrorString(e));
    ctx->scratch_bytes = bytes;
  }
  *out = ctx->scratch;
  return HJ_OK;
}


// ---- block cache.  A bunch's buffers come from one device block and one
// pinned block; released blocks are kept (up to a cap) for the next request
// of the same size class, so admitting and retiring bunches of recurring
// sizes allocates nothing.  Size classes: 2^k x {1, 1.25, 1.5, 1.75}.
constexpr size_t kDevCacheCap = size_t(8) << 30;
constexpr size_t kHostCacheCap = size_t(256) << 20;

size_t size_class(size_t b) {
  if (b <= 4096) return 4096;
  const int lg = 63 - __builtin_clzll((unsigned long long)b);
  const size_t step = size_t(1) << (lg - 2);
  return (b + step - 1) / step * step;
}

constexpr size_t kSlabBlockMax = size_t(16) << 20;
constexpr size_t kSlabSize = size_t(256) << 20;

hj_status cache_take(hj_ctx* ctx, bool host, size_t bytes, void** out, size_t* cap) {
  const size_t c = size_class(bytes);
  auto& fl = host ? ctx->host_free : ctx->dev_free;
  auto it = fl.find(c);
  if (it != fl.end()) {
    *out = it->second;
    fl.erase(it);
    if (host || !ctx->carved.count(*out)) (host ? ctx->host_free_bytes : ctx->dev_free_bytes) -= c;
  } else if (!host && c <= kSlabBlockMax) {
    if (ctx->slab_left < c) {
      void* slab = nullptr;
      cudaError_t e = cudaMalloc(&slab, kSlabSize);
      if (e != cudaSuccess) {
        *out = nullptr;
        return set_err(ctx, HJ_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", kSlabSize,
                       cudaGetErrorString(e));
      }
      ctx->dev_slabs.push_back(slab);
      ctx->slab_cur = (char*)slab;
      ctx->slab_left = kSlabSize;
    }
    *out = ctx->slab_cur;                 // size classes are multiples of 256 bytes
    ctx->slab_cur += c;
    ctx->slab_left -= c;
    ctx->carved.insert(*out);
  } else {
    cudaError_t e = host ? cudaMallocHost(out, c) : cudaMalloc(out, c);
    if (e != cudaSuccess) {
      *out = nullptr;
      return set_err(ctx, HJ_ERR_NOMEM, "%s(%zu bytes) failed: %s",
                     host ? "cudaMallocHost" : "cudaMalloc", c, cudaGetErrorString(e));
    }
  }
  *cap = c;
  return HJ_OK;
}

// Returns a block to the cache (or frees it beyond the cap).  No queued work
// may still use it.
void cache_give(hj_ctx* ctx, bool host, void* p, size_t cap) {
  if (!p) return;
  if (!host && ctx->carved.count(p)) {
    ctx->dev_free.insert({cap, p});
    return;
  }
  size_t& held = host ? ctx->host_free_bytes : ctx->dev_free_bytes;
  if (held + cap > (host ? kHostCacheCap : kDevCacheCap)) {
    if (host) cudaFreeHost(p);
    else cudaFree(p);
    return;
  }
  (host ? ctx->host_free : ctx->dev_free).insert({cap, p});
  held += cap;
}

// Frees the kept blocks (carved ones stay for reuse unless `slabs` is set,
// which also frees the slabs: only when no bunch or batch holds a block).
void cache_clear(hj_ctx* ctx, bool slabs) {
  for (auto it = ctx->wake_sets.begin(); it != ctx->wake_sets.end();) {
    if (it->second.refs > 0 && !slabs) {
      ++it;
      continue;
    }
    cache_give(ctx, false, it->second.dev, it->second.cap);
    it = ctx->wake_sets.erase(it);
  }
  std::multimap<size_t, void*> keep;
  for (auto& kv : ctx->dev_free) {
    if (ctx->carved.count(kv.second)) keep.insert(kv);
    else cudaFree(kv.second);
  }
  for (auto& kv : ctx->host_free) cudaFreeHost(kv.second);
  ctx->dev_free.swap(keep);
  ctx->host_free.clear();
  ctx->dev_free_bytes = ctx->host_free_bytes = 0;
  if (slabs) {
    for (void* s : ctx->dev_slabs) cudaFree(s);
    ctx->dev_slabs.clear();
    ctx->carved.clear();
    ctx->dev_free.clear();
    ctx->slab_cur = nullptr;
    ctx->slab_left = 0;
  }
}

// The twiddle table [P] of the bins step, built once per context and P.
hj_status shared_twiddles(hj_ctx* ctx, int P, double2** out) {
  auto it = ctx->twiddles.find(P);
  if (it == ctx->twiddles.end()) {
    std::vector<double> tw(2 * (size_t)P);
    host_twiddles(P, tw.data());
    double2* d = nullptr;
    cudaError_t e = cudaMalloc((void**)&d, sizeof(double2) * P);
    if (e == cudaSuccess)
      e = cudaMemcpy(d, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      if (d) cudaFree(d);
      return set_err(ctx, HJ_ERR_CUDA, "twiddle table: %s", cudaGetErrorString(e));
    }
    it = ctx->twiddles.insert({P, d}).first;
  }
  *out = it->second;
  return HJ_OK;
}


hj_status check_params(hj_ctx* ctx, const hj_params* p) {
  if (!p) return set_err(ctx, HJ_ERR_ARG, "params is NULL");
  if (p->n_turns < 0) return set_err(ctx, HJ_ERR_ARG, "n_turns must be >= 0");
  if (!(p->mass > 0)) return set_err(ctx, HJ_ERR_ARG, "mass must be > 0");
  return HJ_OK;
}

hj_status check_grid(hj_ctx* ctx, const hj_grid* g) {
  if (!g) return set_err(ctx, HJ_ERR_ARG, "grid is NULL");
  if (g->nbins <= 0) return set_err(ctx, HJ_ERR_NBINS, "nbins must be > 0 (got %lld)",
                                    (long long)g->nbins);
  if (!g->centers) return set_err(ctx, HJ_ERR_ARG, "grid.centers is NULL");
  if (!(g->edge_step != 0.0))
    return set_err(ctx, HJ_ERR_ARG, "Bin edges have zero step size.");
  return HJ_OK;
}

// Device sums of the moments kernel, reduced on the host in block order.
void sum_moments(const hj_bunch* b, double m[4]) {
  m[0] = m[1] = m[2] = m[3] = 0.0;
  for (int i = 0; i < b->nblk_m; ++i)
    for (int k = 0; k < 4; ++k) m[k] += b->h_mom[4 * i + k];
}

hj_status read_moments(hj_bunch* b, double m[4]) {
  HJ_CUDA(b->ctx, cudaMemcpyAsync(b->h_mom, b->part_mom, sizeof(double) * 4 * b->nblk_m,
                                  cudaMemcpyDeviceToHost, b->stream));
  HJ_CUDA(b->ctx, cudaStreamSynchronize(b->stream));
  sum_moments(b, m);
  return HJ_OK;
}

hj_status launch_moments(hj_bunch* b, int apply, double* z_out, double* dE_out) {
  FlushArgs f{};
  f.z = b->z;
  f.dE = b->dE;
  f.n = b->n;
  f.ts = b->ts;
  f.potd = b->potd;
  f.B = b->B;
  f.use_wake = b->use_wake;
  f.update_E0 = b->p.update_E0;
  f.c1 = b->c1;
  f.cB = b->cB;
  f.inv_cstep = b->inv_c;
  f.e0 = b->e0;
  f.inv_estep = b->inv_e;
  f.apply = apply;
  f.z_out = z_out;
  f.dE_out = dE_out;
  f.part = b->part_mom;
  HJ_CUDA(b->ctx, launch_flush(f, b->nblk_m, b->stream));
  return HJ_OK;
}

// The sticky status of the turn state already copied to h_ts.
hj_status state_status(hj_bunch* b) {
  int st = b->h_ts->status;
  if (st & (1 << HJ_ERR_NONFINITE))
    return set_err(b->ctx, HJ_ERR_NONFINITE,
                   "non-finite bunch moments detected on the device (turn %lld)",
                   (long long)b->h_ts->turn - 1);
  if (st & (1 << HJ_ERR_ARG))
    return set_err(b->ctx, HJ_ERR_ARG, "host-fed draws do not cover turn %lld",
                   (long long)b->h_ts->turn - 1);
  return HJ_OK;
}

hj_status read_state(hj_bunch* b) {
  HJ_CUDA(b->ctx, cudaMemcpyAsync(b->h_ts, b->ts, sizeof(TurnState), cudaMemcpyDeviceToHost,
                                  b->stream));
  HJ_CUDA(b->ctx, cudaStreamSynchronize(b->stream));
  return state_status(b);
}

// Thread layout of the fused pass when the context does not pin one, from
// timings on B200: four particles per thread x 512 threads, prefetching the
// next group, one 32-bit counter per bin (1e8 particles, 16384 bins, Float64
// normals, both with range-checked deposits, one box: 0.75 ms per pass
// against 0.79 with 16-bit pairs, whose wider hot window does not make up
// for their overflow checks).
int default_pass_layout(int B, int64_t n) {
  (void)B;
  (void)n;
  return 0 | kPassN32;
}

// The library's layout for a request r (-1: the default for B bins).
int auto_pass_layout(int r, int B, int64_t n) {
  return resolve_pass_request(r, default_pass_layout(B, n));
}

void fill_result(hj_bunch* b, const double m[4], hj_result* res) {
  if (!res) return;
  res->sigma_z = global_std(m[0], m[1], b->n);
  res->sigma_E = global_std(m[2], m[3], b->n);
  res->E0 = b->h_ts->cur.E0;
  res->sigma_E0_initial = b->sigma_E0_initial;
  res->sigma_z0_initial = b->sigma_z0_initial;
  res->mean_z = b->n > 0 ? m[0] / (double)b->n : 0.0;
  res->mean_dE = b->n > 0 ? m[2] / (double)b->n : 0.0;
  // a batch member's turns are counted on the device (its turn state was read)
  res->turns = b->batch_member ? b->h_ts->turn - 1 : b->turns_done;
}

cudaError_t set_kernel_attributes(hj_ctx* ctx) {
  cudaError_t e = prepare_track_kernels(ctx->max_smem_optin);
  if (e == cudaSuccess) e = prepare_wake_kernels(ctx->max_smem_optin);
  return e;
}

}  // namespace hj_impl

// ====================================================================== context

int hj::ctx_device(const hj_ctx* ctx) { return ctx->device; }

hj_status hj::ctx_set_error(hj_ctx* ctx, hj_status code, const char* msg) {
  if (ctx) ctx->err = msg;
  return code;
}

extern "C" const char* hj_version(void) { return kVersion; }

extern "C" const char* hj_status_string(hj_status s) {
  switch (s) {
    case HJ_OK: return "HJ_OK";
    case HJ_ERR_ARG: return "HJ_ERR_ARG";
    case HJ_ERR_NBINS: return "HJ_ERR_NBINS";
    case HJ_ERR_WAKE_PARAM: return "HJ_ERR_WAKE_PARAM";
    case HJ_ERR_CUDA: return "HJ_ERR_CUDA";
    case HJ_ERR_NOMEM: return "HJ_ERR_NOMEM";
    case HJ_ERR_TOO_LARGE: return "HJ_ERR_TOO_LARGE";
    case HJ_ERR_EMPTY: return "HJ_ERR_EMPTY";
    case HJ_ERR_NONFINITE: return "HJ_ERR_NONFINITE";
    case HJ_ERR_TIMEOUT: return "HJ_ERR_TIMEOUT";
    case HJ_ERR_NO_DEVICE: return "HJ_ERR_NO_DEVICE";
    case HJ_ERR_STATE: return "HJ_ERR_STATE";
    case HJ_ERR_FULL: return "HJ_ERR_FULL";
    default: return "HJ_ERR_UNKNOWN";
  }
}

extern "C" hj_status hj_create(int32_t device, hj_ctx** out) {
  if (!out) return HJ_ERR_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return HJ_ERR_NO_DEVICE;
  if (device < 0 || device >= count) return HJ_ERR_NO_DEVICE;
  if (cudaSetDevice(device) != cudaSuccess) return HJ_ERR_CUDA;
  hj_ctx* ctx = new hj_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&ctx->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (set_kernel_attributes(ctx) != cudaSuccess) {
    delete ctx;
    return HJ_ERR_CUDA;
  }
  *out = ctx;
  return HJ_OK;
}

static void ctx_free(hj_ctx* ctx) {
  cudaSetDevice(ctx->device);
  if (ctx->scratch) cudaFree(ctx->scratch);
  cache_clear(ctx, true);
  for (auto& kv : ctx->twiddles) cudaFree(kv.second);
  delete ctx;
}

extern "C" void hj_destroy(hj_ctx* ctx) {
  if (!ctx || ctx->closing) return;
  if (ctx->live_objects > 0) {   // freed by the last bunch or batch destroyed
    ctx->closing = true;
    return;
  }
  ctx_free(ctx);
}

void hj_impl::ctx_retain(hj_ctx* ctx) { ctx->live_objects += 1; }

void hj_impl::ctx_release(hj_ctx* ctx) {
  if (--ctx->live_objects == 0 && ctx->closing) ctx_free(ctx);
}

extern "C" const char* hj_last_error(const hj_ctx* ctx) { return ctx ? ctx->err.c_str() : ""; }

extern "C" hj_status hj_trim(hj_ctx* ctx) {
  HJ_TRY(ctx_ok(ctx));
  HJ_CUDA(ctx, cudaDeviceSynchronize());
  cache_clear(ctx);
  return HJ_OK;
}

extern "C" hj_status hj_set_pass_layout(hj_ctx* ctx, int32_t layout) {
  if (!ctx) return HJ_ERR_ARG;
  if (!pass_request_valid(layout))
    return set_err(ctx, HJ_ERR_ARG,
                   "pass layout must be -1 (automatic), %d (automatic, single-precision normals), "
                   "0..%d or 8..%d, plus %d for single-precision normals",
                   kPassAutoFast, kNumPassCfgs - 1, kPassN32 + kNumPassCfgs - 1, kPassFastNormals);
  ctx->pass_layout = layout;
  return HJ_OK;
}

// ====================================================================== bunch

extern "C" void hj_bunch_destroy(hj_bunch* b) {
  if (!b) return;
  if (!b->ctx) {                          // failed before it was tied to a context
    delete b;
    return;
  }
  cudaSetDevice(b->ctx->device);
  cudaStreamSynchronize(b->stream);       // nothing queued still uses the blocks
  cache_give(b->ctx, false, b->arena, b->arena_cap);
  cache_give(b->ctx, true, b->harena, b->harena_cap);
  if (b->wset) b->wset->refs -= 1;
  cache_give(b->ctx, false, b->tables, b->tables_cap);
  if (b->d_sums) cudaFree(b->d_sums);
  if (b->d_log) cudaFree(b->d_log);
  for (cudaEvent_t e : b->events) cudaEventDestroy(e);
  hj_ctx* ctx = b->ctx;
  const bool held = b->holds_ctx;
  delete b;
  if (held) ctx_release(ctx);
}

// Creation of a bunch in two halves, so that a batch can admit many bunches
// with one synchronisation: bunch_create_begin validates, lays out the
// buffers and enqueues the initial moments and their copy to the host;
// bunch_create_end (after the stream has reached them) builds the grid, the
// wake tables, the RF table and the turn state.
// chunk > 0: a batch member, whose partial slots are its chunks of `chunk`
// particles (the batch's chunk table) instead of one per block of the grid;
// cfg >= 0 pins the pass layout.
hj_status hj_impl::bunch_create_begin(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                                      const hj_params* params, const hj_wake* wake,
                                      int64_t nbins, const hj_grid* grid, uint64_t seed,
                                      void* stream, hj_bunch* b, int64_t chunk, int cfg) {
  b->ctx = ctx;
  if (!b->holds_ctx) {
    ctx_retain(ctx);
    b->holds_ctx = true;
  }
  b->stream = (cudaStream_t)stream;
  b->z = d_z;
  b->dE = d_dE;
  b->n = n;
  b->p = *params;
  b->seed = seed;
  b->use_wake = params->use_wakefield ? 1 : 0;
  if (wake) b->w = *wake;
  else hj_wake_reference(params, &b->w);
  b->qe_mode = params->use_excitation ? QE_PHILOX : QE_OFF;

  if (b->use_wake) {
    const int64_t B = grid ? grid->nbins : nbins;
    if (B <= 0) return set_err(ctx, HJ_ERR_NBINS, "Buffer nbins invalid (must be > 0).");
    if (B > kMaxBins)
      return set_err(ctx, HJ_ERR_TOO_LARGE, "nbins = %lld exceeds the supported %lld",
                     (long long)B, (long long)kMaxBins);
    if (b->w.ctau <= 0) return set_err(ctx, HJ_ERR_WAKE_PARAM, "Wake parameter cτ must be positive.");
    if (params->pipe_radius <= 0)
      return set_err(ctx, HJ_ERR_WAKE_PARAM, "Wake parameter pipe_radius must be positive.");
    if (n == 0)
      return set_err(ctx, HJ_ERR_EMPTY, "wakefield with zero particles: log10(0) in the particle factor");
    if (grid) HJ_TRY(check_grid(ctx, grid));
    b->B = (int)B;
  }

  // sizes of every buffer, then one device and one pinned block for all
  b->nblk_m = (int)std::min<int64_t>(std::max<int64_t>((n + 4095) / 4096, 1),
                                     (int64_t)ctx->num_sms * 4);
  if (b->use_wake) {
    b->P = (int)next_pow2(2 * (int64_t)b->B);            // src/evolution.jl:265
    b->M = b->P / 2;
    b->H = b->M / 2;
    b->logH = b->H >= 1 ? ilog2(b->H) : 0;
  }
  b->cfg = cfg >= 0 ? cfg : auto_pass_layout(ctx->pass_layout, b->B, n);
  if (chunk > 0) {
    b->batch_member = true;
    b->nblk = (int)std::max<int64_t>((n + chunk - 1) / chunk, 1);
  } else {
    const int bps = track_blocks_per_sm(b->B, b->qe_mode, b->use_wake, b->cfg);
    b->nblk = track_grid_size(n, b->B, ctx->num_sms, bps, b->cfg);
  }
  {
    const size_t B = (size_t)b->B, nb = (size_t)b->nblk;
    Carve c;
    const size_t o_mom = c.add<double>(4 * (size_t)b->nblk_m);
    const size_t o_ts = c.add<TurnState>(1);
    const size_t o_sum = c.add<double>((size_t)kNumSums * nb);
    const size_t o_rf = c.add<double2>(kRfTableSize);
    // per block and warp, the staging queue of the particles whose Float64
    // normal takes the slow path (kDeferStage indices)
    const bool defer = b->qe_mode == QE_PHILOX && !(b->cfg & kPassFastNormals);
    const size_t o_dq =
        defer ? c.add<int64_t>(nb * (size_t)(pass_cfg_threads(b->cfg) / 32) * kDeferStage) : 0;
    size_t o[6] = {};
    if (b->use_wake) {
      // pot, potd, hist and hist_spill are adjacent: one memset zeroes them
      o[0] = c.add<double>(B);                                   // pot
      o[1] = c.add<double2>(B + 1);                              // potd
      o[2] = c.add<unsigned long long>(3 * B + 2);               // hist
      o[3] = c.add<unsigned long long>(3 * B + 2);               // hist_spill
      b->zero_bytes = c.off - o[0];
      o[4] = c.add<uint32_t>(nb * B);                            // part_cnt
      o[5] = c.add<unsigned long long>(nb * (B + 1));            // part_cic
    }
    HJ_TRY(cache_take(ctx, false, c.off, &b->arena, &b->arena_cap));
    char* a = (char*)b->arena;
    b->part_mom = (double*)(a + o_mom);
    b->ts = (TurnState*)(a + o_ts);
    b->part_sum = (double*)(a + o_sum);
    b->rf_table = (double2*)(a + o_rf);
    b->defer_q = defer ? (int64_t*)(a + o_dq) : nullptr;
    if (b->use_wake) {
      b->pot = (double*)(a + o[0]);
      b->potd = (double2*)(a + o[1]);
      b->hist = (unsigned long long*)(a + o[2]);
      b->hist_spill = (unsigned long long*)(a + o[3]);
      b->part_cnt = (uint32_t*)(a + o[4]);
      b->part_cic = (unsigned long long*)(a + o[5]);
    }
    Carve hc;
    const size_t h_mom = hc.add<double>(4 * (size_t)b->nblk_m);
    const size_t h_ts = hc.add<TurnState>(1);
    const size_t h_rf = hc.add<double>(2 * (size_t)kRfTableSize);
    HJ_TRY(cache_take(ctx, true, hc.off, &b->harena, &b->harena_cap));
    b->h_mom = (double*)((char*)b->harena + h_mom);
    b->h_ts = (TurnState*)((char*)b->harena + h_ts);
    b->h_rf = (double*)((char*)b->harena + h_rf);
  }

  // Initial spreads, src/evolution.jl:247-249: enqueued here, read in
  // bunch_create_end
  HJ_TRY(launch_moments(b, 0, nullptr, nullptr));
  HJ_CUDA(ctx, cudaMemcpyAsync(b->h_mom, b->part_mom, sizeof(double) * 4 * b->nblk_m,
                               cudaMemcpyDeviceToHost, b->stream));
  return HJ_OK;
}

hj_status hj_impl::bunch_create_end(hj_ctx* ctx, hj_bunch* b, const hj_grid* grid,
                                    const hj_checkpoint* cp) {
  const int64_t n = b->n;
  const hj_params* params = &b->p;
  double m[4];
  sum_moments(b, m);
  b->sigma_z0_initial = cp ? cp->sigma_z0_initial : global_std(m[0], m[1], n);
  b->sigma_E0_initial = cp ? cp->sigma_E0_initial : global_std(m[2], m[3], n);

  if (b->use_wake) {
    const int B = b->B;
    b->centers.resize(B);
    hj_grid g{};
    hj_ctx::WakeSet* cached = nullptr;
    std::array<uint64_t, 8> key{};
    if (grid) {
      std::memcpy(b->centers.data(), grid->centers, sizeof(double) * B);
      g = *grid;
    } else {
      const double kv[7] = {b->sigma_z0_initial, b->w.half_width_sigmas, b->w.wake_factor,
                            b->w.wake_sqrt, b->w.ctau, b->w.sin_coef, b->w.delta_std};
      key[0] = (uint64_t)B;
      std::memcpy(key.data() + 1, kv, sizeof(kv));
      auto it = ctx->wake_sets.find(key);
      if (it != ctx->wake_sets.end()) {
        cached = &it->second;
        cached->used = ++ctx->wake_clock;
        b->centers = cached->centers;
        g.nbins = B;
        g.edge_first = cached->e0;
        g.edge_last = cached->eN;
        g.edge_step = cached->estep;
      } else {
        HJ_TRY(hj_make_grid(b->sigma_z0_initial, b->w.half_width_sigmas, B, b->centers.data(),
                            &g));
      }
    }
    b->e0 = g.edge_first;
    b->eN = g.edge_last;
    b->estep = g.edge_step;
    b->inv_e = 1.0 / g.edge_step;                        // src/utils.jl:378
    b->c1 = b->centers[0];
    b->cB = b->centers[B - 1];
    if (B >= 2) {
      const double step = (b->cB - b->c1) / (double)(B - 1);  // src/wakefield.jl:41-42
      b->inv_c = 1.0 / step;
      const double u = (b->cB - b->c1) * b->inv_c;          // src/wakefield.jl:81-91
      const double fl = std::floor(u);
      const int64_t idx1 = std::min<int64_t>(std::max<int64_t>((int64_t)fl + 1, 1), B - 1);
      b->hi_idx = (int)(idx1 - 1);
      b->hi_w = u - fl;
    }
    HJ_TRY(shared_twiddles(ctx, b->P, &b->twP));
    const size_t wbytes = sizeof(double) * B, fbytes = sizeof(double2) * ((size_t)b->M + 1);
    void* blk = nullptr;
    if (cached) {
      blk = cached->dev;
    } else {
      // W, λ and FFT(W) of this grid in one block of the cache, read-only for
      // every bunch; kept in wake_sets for the next bunch when the grid was
      // built here, else private to this bunch
      size_t cap = 0;
      HJ_TRY(cache_take(ctx, false, 2 * wbytes + fbytes, &blk, &cap));
      double* W = (double*)blk;
      std::vector<double> hW(B), hl(B);
      host_wake_tables(b->centers.data(), B, b->w, hW.data(), hl.data());
      cudaError_t e = cudaMemcpyAsync(W, hW.data(), wbytes, cudaMemcpyHostToDevice, b->stream);
      if (e == cudaSuccess)
        e = cudaMemcpyAsync(W + B, hl.data(), wbytes, cudaMemcpyHostToDevice, b->stream);
      void* xg = nullptr;
      hj_status s = HJ_OK;
      if (e == cudaSuccess && b->H >= 4) {
        s = scratch(ctx, sizeof(double2) * (size_t)b->M, &xg);
        if (s == HJ_OK)
          e = launch_wake_spectrum(W, B, b->P, b->M, b->H, b->logH, b->twP, (double2*)xg,
                                   (double2*)((char*)blk + 2 * wbytes), b->stream);
      }
      cudaError_t e2 = cudaStreamSynchronize(b->stream);   // host vectors, scratch
      if (s == HJ_OK && (e != cudaSuccess || e2 != cudaSuccess))
        s = set_err(ctx, HJ_ERR_CUDA, "wake tables: %s",
                    cudaGetErrorString(e != cudaSuccess ? e : e2));
      if (s != HJ_OK) {
        cache_give(ctx, false, blk, cap);
        return s;
      }
      if (!grid) {
        constexpr size_t kWakeSets = 8;
        if (ctx->wake_sets.size() >= kWakeSets) {   // the least recently used free set goes
          auto lru = ctx->wake_sets.end();
          for (auto it = ctx->wake_sets.begin(); it != ctx->wake_sets.end(); ++it)
            if (it->second.refs == 0 && (lru == ctx->wake_sets.end() || it->second.used < lru->second.used))
              lru = it;
          if (lru != ctx->wake_sets.end()) {
            cache_give(ctx, false, lru->second.dev, lru->second.cap);
            ctx->wake_sets.erase(lru);
          }
        }
        if (ctx->wake_sets.size() < kWakeSets) {
          hj_ctx::WakeSet ws;
          ws.centers = b->centers;
          ws.e0 = g.edge_first;
          ws.eN = g.edge_last;
          ws.estep = g.edge_step;
          ws.used = ++ctx->wake_clock;
          ws.dev = blk;
          ws.cap = cap;
          cached = &ctx->wake_sets.insert({key, std::move(ws)}).first->second;
        }
      }
      if (!cached) {
        b->tables = blk;
        b->tables_cap = cap;
      }
    }
    if (cached) {
      cached->refs += 1;
      b->wset = cached;
    }
    b->W = (double*)blk;
    b->lam = b->W + B;
    b->Wf = (double2*)((char*)blk + 2 * wbytes);
    HJ_CUDA(ctx, cudaMemsetAsync(b->pot, 0, b->zero_bytes, b->stream));   // pot potd hist ovf
  }

  // RF table, staged in the bunch's pinned block
  host_rf_table(params->voltage, params->phi_s, kRfTableSize, b->h_rf);
  b->rf_Vs = b->h_rf[0];
  HJ_CUDA(ctx, cudaMemcpyAsync(b->rf_table, b->h_rf, sizeof(double) * 2 * kRfTableSize,
                               cudaMemcpyHostToDevice, b->stream));

  TurnState t{};
  t.cur = make_turn_scalars(cp ? cp->E0 : params->E0, *params, b->sigma_E0_initial);
  t.pending = 0;
  t.pending_mean = 0.0;
  t.turn = cp ? cp->turn : 1;
  b->turns_done = cp ? cp->turn - 1 : 0;
  t.turns_left = INT64_MAX;   // a plain bunch runs until it is finished
  t.status = 0;
  *b->h_ts = t;
  // staged in pinned memory that lives as long as the bunch; later work on
  // the stream is ordered after the copy, host reads of h_ts synchronise first
  // (a batch member's state goes to the batch's array instead)
  if (!b->batch_member)
    HJ_CUDA(ctx, cudaMemcpyAsync(b->ts, b->h_ts, sizeof(TurnState), cudaMemcpyHostToDevice,
                                 b->stream));
  return HJ_OK;
}

hj_status hj_impl::bunch_create_impl(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                                     const hj_params* params, const hj_wake* wake,
                                     int64_t nbins, const hj_grid* grid, uint64_t seed,
                                     void* stream, hj_bunch* b, int64_t chunk, int cfg) {
  HJ_TRY(bunch_create_begin(ctx, d_z, d_dE, n, params, wake, nbins, grid, seed, stream, b,
                            chunk, cfg));
  HJ_CUDA(ctx, cudaStreamSynchronize(b->stream));
  return bunch_create_end(ctx, b, grid);
}

extern "C" hj_status hj_bunch_create(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                                     const hj_params* params, const hj_wake* wake,
                                     int64_t nbins, const hj_grid* grid, uint64_t seed,
                                     void* stream, hj_bunch** out) {
  HJ_TRY(ctx_ok(ctx));
  if (!out) return set_err(ctx, HJ_ERR_ARG, "out is NULL");
  *out = nullptr;
  HJ_TRY(check_params(ctx, params));
  if (n < 0) return set_err(ctx, HJ_ERR_ARG, "Number of particles must be non-negative. Got %lld.", (long long)n);
  if (n > 0 && (!d_z || !d_dE)) return set_err(ctx, HJ_ERR_ARG, "particle arrays are NULL");
  if ((((uintptr_t)d_z) | ((uintptr_t)d_dE)) & 31)
    return set_err(ctx, HJ_ERR_ARG, "device particle arrays must be 32-byte aligned");
  if (n == 0 && !params->use_wakefield)
    return set_err(ctx, HJ_ERR_ARG, "a resident bunch needs at least one particle");
  hj_bunch* b = new hj_bunch();
  hj_status s = bunch_create_impl(ctx, d_z, d_dE, n, params, wake, nbins, grid, seed, stream, b);
  if (s != HJ_OK) {
    hj_bunch_destroy(b);
    return s;
  }
  *out = b;
  return HJ_OK;
}

extern "C" hj_status hj_bunch_set_draws(hj_bunch* b, const double* d_draws, int64_t first_turn,
                                        int64_t turns) {
  if (!b) return HJ_ERR_ARG;
  if (d_draws && turns <= 0) return set_err(b->ctx, HJ_ERR_ARG, "turns must be > 0");
  b->draws = d_draws;
  b->draws_first = first_turn;
  b->draws_turns = turns;
  if (!b->p.use_excitation) b->qe_mode = QE_OFF;
  else b->qe_mode = d_draws ? QE_DRAWS : QE_PHILOX;
  return HJ_OK;
}

// Arguments of the fused pass and of the bins step of bunch b.
void hj_impl::fill_turn_args(const hj_bunch* b, PassArgs& a, BinsArgs& g) {
  a = PassArgs{};
  a.z = b->z;
  a.dE = b->dE;
  a.n = b->n;
  a.ts = b->ts;
  a.potd = b->potd;
  a.zig = (b->qe_mode == QE_PHILOX && !(b->cfg & kPassFastNormals)) ? 1 : 0;
  if (b->use_wake) {
    const PassWindows w = track_windows(b->B, b->cfg, a.zig != 0);
    a.win = w.kick;
    a.hwin = w.hot;
  }
  a.B = b->B;
  a.use_wake = b->use_wake;
  a.e0 = b->e0;
  a.eN = b->eN;
  a.inv_estep = b->inv_e;
  a.c1 = b->c1;
  a.cB = b->cB;
  a.inv_cstep = b->inv_c;
  a.V = b->p.voltage;
  a.phi_s = b->p.phi_s;
  {
    const long double kPiL = 3.141592653589793238462643383279502884L;
    const long double h = 2.0L * kPiL / (long double)kRfTableSize;
    a.rf_table = b->rf_table;
    a.Vs = b->rf_Vs;
    a.rf_inv_h = (double)(1.0L / h);
    a.rf_h_hi = (double)h;
    a.rf_h_lo = (double)(h - (long double)a.rf_h_hi);
    a.philox = philox_keys(b->seed);
  }
  a.inv_mass = 1.0 / b->p.mass;
  a.alpha_c = b->p.alpha_c;
  a.two_pi_h = kTwoPi * (double)b->p.harmonic;
  a.update_eta = b->p.update_eta;
  a.update_E0 = b->p.update_E0;
  a.sr = b->p.SR_damping;
  a.qe_mode = b->qe_mode;
  a.cfg = b->cfg;
  a.seed = b->seed;
  a.draws = b->draws;
  a.draws_first_turn = b->draws_first;
  a.draws_turns = b->draws_turns;
  a.part_cnt = b->part_cnt;
  a.part_cic = b->part_cic;
  a.part_sum = b->part_sum;
  a.hist_out = b->hist;
  a.hist_spill = b->hist_spill;

  g = BinsArgs{};
  g.ts = b->ts;
  g.part_sum = b->shard ? b->d_sums : b->part_sum;
  g.nblk = b->shard ? 1 : b->nblk;
  g.n = b->shard ? b->n_global : b->n;
  g.params = b->p;
  g.sigma_E0_initial = b->sigma_E0_initial;
  g.population = b->w.population;
  g.use_wake = b->use_wake;
  g.B = b->B;
  g.P = b->P;
  g.M = b->M;
  g.H = b->H;
  g.logH = b->logH;
  g.cnt = b->hist;
  g.cic = b->hist ? b->hist + b->B : nullptr;
  g.lam = b->lam;
  g.Wf = b->Wf;
  g.twP = b->twP;
  g.pot = b->pot;
  g.potd = b->potd;
  g.hi_idx = b->hi_idx;
  g.hi_w = b->hi_w;
  g.W = b->W;
  g.conv_only = 0;

  a.n_parts = b->nblk;
  a.pair_offset = b->first_particle / 2;
  a.defer_q = b->defer_q;
}

extern "C" hj_status hj_bunch_advance(hj_bunch* b, int64_t turns) {
  if (!b) return HJ_ERR_ARG;
  hj_ctx* ctx = b->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (turns < 0) return set_err(ctx, HJ_ERR_ARG, "turns must be >= 0");
  PassArgs a;
  BinsArgs g;
  fill_turn_args(b, a, g);

  for (int64_t t = 0; t < turns; ++t) {
    cudaEvent_t ev[3] = {nullptr, nullptr, nullptr};
    if (b->profiling) {
      while (b->events.size() < b->events_used + 3) {
        cudaEvent_t e;
        HJ_CUDA(ctx, cudaEventCreate(&e));
        b->events.push_back(e);
      }
      for (int k = 0; k < 3; ++k) ev[k] = b->events[b->events_used + k];
      b->events_used += 3;
      HJ_CUDA(ctx, cudaEventRecord(ev[0], b->stream));
    }
    HJ_CUDA(ctx, launch_track_pass(a, b->nblk, b->stream));
    if (b->profiling) HJ_CUDA(ctx, cudaEventRecord(ev[1], b->stream));
    if (b->use_wake)
      HJ_CUDA(ctx, launch_hist_reduce(b->part_cnt, b->part_cic, b->nblk, b->B, b->hist, false,
                                      b->stream, b->hist_spill));
    HJ_CUDA(ctx, launch_bins(g, b->stream));
    if (b->profiling) {
      HJ_CUDA(ctx, cudaEventRecord(ev[2], b->stream));
      b->profiled_turns += 1;
      b->profiled_launches += b->use_wake ? 3 : 2;
    }
    if (b->log_every > 0 && (b->turns_done + t + 1) % b->log_every == 0) {
      const int64_t rec = kLogHeader + (b->log_density ? b->B : 0);
      HJ_TRY(launch_moments(b, 1, nullptr, nullptr));
      HJ_CUDA(ctx, launch_log_record(b->part_mom, b->nblk_m, b->n, b->ts,
                                     b->log_density ? b->hist : nullptr, b->B,
                                     b->d_log + (b->log_count % b->log_capacity) * rec,
                                     b->stream));
      b->log_count += 1;
      if (b->profiling) b->profiled_launches += 2;
    }
  }
  b->turns_done += turns;
  return HJ_OK;
}

extern "C" hj_status hj_bunch_set_profiling(hj_bunch* b, int32_t enable) {
  if (!b) return HJ_ERR_ARG;
  HJ_TRY(ctx_ok(b->ctx));
  b->profiling = enable != 0;
  b->events_used = 0;
  b->profiled_turns = 0;
  b->profiled_launches = 0;
  return HJ_OK;
}

extern "C" hj_status hj_bunch_read_profile(hj_bunch* b, double* out4) {
  if (!b || !out4) return HJ_ERR_ARG;
  HJ_TRY(ctx_ok(b->ctx));
  HJ_CUDA(b->ctx, cudaStreamSynchronize(b->stream));
  double pass = 0.0, bins = 0.0;
  for (size_t i = 0; i + 3 <= b->events_used; i += 3) {
    float a = 0.f, c = 0.f;
    HJ_CUDA(b->ctx, cudaEventElapsedTime(&a, b->events[i], b->events[i + 1]));
    HJ_CUDA(b->ctx, cudaEventElapsedTime(&c, b->events[i + 1], b->events[i + 2]));
    pass += a;
    bins += c;
  }
  out4[0] = pass;
  out4[1] = bins;
  out4[2] = (double)b->profiled_turns;
  out4[3] = (double)b->profiled_launches;
  return HJ_OK;
}

extern "C" hj_status hj_bunch_observe(hj_bunch* b, double* d_z_out, double* d_dE_out,
                                      hj_result* res) {
  if (!b) return HJ_ERR_ARG;
  HJ_TRY(ctx_ok(b->ctx));
  HJ_TRY(launch_moments(b, 1, d_z_out, d_dE_out));
  double m[4];
  HJ_TRY(read_moments(b, m));
  HJ_TRY(read_state(b));
  fill_result(b, m, res);
  return HJ_OK;
}

extern "C" hj_status hj_bunch_finish(hj_bunch* b, hj_result* res) {
  if (!b) return HJ_ERR_ARG;
  HJ_TRY(ctx_ok(b->ctx));
  HJ_TRY(launch_moments(b, 1, b->z, b->dE));
  // nothing is pending any more: the next pass must see a zero kick table
  const int32_t zero = 0;
  HJ_CUDA(b->ctx, cudaMemcpyAsync(&b->ts->pending, &zero, sizeof(int32_t),
                                  cudaMemcpyHostToDevice, b->stream));
  if (b->potd)
    HJ_CUDA(b->ctx, cudaMemsetAsync(b->potd, 0, sizeof(double2) * ((size_t)b->B + 1), b->stream));
  double m[4];
  HJ_TRY(read_moments(b, m));
  HJ_TRY(read_state(b));
  fill_result(b, m, res);
  return HJ_OK;
}

extern "C" hj_status hj_bunch_histogram(hj_bunch* b, int64_t* counts_host) {
  if (!b || !counts_host) return HJ_ERR_ARG;
  HJ_TRY(ctx_ok(b->ctx));
  if (!b->use_wake) return set_err(b->ctx, HJ_ERR_STATE, "bunch has no wakefield histogram");
  HJ_CUDA(b->ctx, cudaMemcpyAsync(counts_host, b->hist, sizeof(int64_t) * b->B,
                                  cudaMemcpyDeviceToHost, b->stream));
  HJ_CUDA(b->ctx, cudaStreamSynchronize(b->stream));
  return HJ_OK;
}

extern "C" hj_status hj_bunch_potential(hj_bunch* b, double* pot_host) {
  if (!b || !pot_host) return HJ_ERR_ARG;
  HJ_TRY(ctx_ok(b->ctx));
  if (!b->use_wake) return set_err(b->ctx, HJ_ERR_STATE, "bunch has no wake potential");
  HJ_CUDA(b->ctx, cudaMemcpyAsync(pot_host, b->pot, sizeof(double) * b->B,
                                  cudaMemcpyDeviceToHost, b->stream));
  HJ_CUDA(b->ctx, cudaStreamSynchronize(b->stream));
  return HJ_OK;
}

// ====================================================================== whole loop

static hj_status evolve_empty(hj_ctx* ctx, const hj_params* p, hj_result* out) {
  if (p->use_wakefield)
    return set_err(ctx, HJ_ERR_EMPTY, "wakefield with zero particles: log10(0) in the particle factor");
  if (out) {
    std::memset(out, 0, sizeof(*out));
    out->E0 = p->E0;
    // MPI branch: mean = 0/0 per turn (src/evolution.jl:426)
    if (p->update_E0 && p->n_turns > 0) out->E0 = p->E0 + 0.0 / 0.0;
    out->turns = p->n_turns;
  }
  return HJ_OK;
}

extern "C" hj_status hj_evolve_device(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                                      const hj_params* params, const hj_wake* wake,
                                      int64_t nbins, const hj_grid* grid,
                                      const double* d_qe_draws, uint64_t seed, void* stream,
                                      hj_result* out) {
  HJ_TRY(ctx_ok(ctx));
  HJ_TRY(check_params(ctx, params));
  if (n < 0) return set_err(ctx, HJ_ERR_ARG, "Number of particles must be non-negative. Got %lld.", (long long)n);
  if (n == 0) return evolve_empty(ctx, params, out);
  hj_bunch* b = nullptr;
  HJ_TRY(hj_bunch_create(ctx, d_z, d_dE, n, params, wake, nbins, grid, seed, stream, &b));
  hj_status s = HJ_OK;
  if (d_qe_draws) s = hj_bunch_set_draws(b, d_qe_draws, 1, params->n_turns);
  if (s == HJ_OK) s = hj_bunch_advance(b, params->n_turns);
  if (s == HJ_OK) s = hj_bunch_finish(b, out);
  hj_bunch_destroy(b);
  return s;
}

extern "C" hj_status hj_evolve(hj_ctx* ctx, double* z, double* dE, int64_t n,
                               const hj_params* params, const hj_wake* wake, int64_t nbins,
                               const hj_grid* grid, const double* qe_draws, uint64_t seed,
                               hj_result* out) {
  HJ_TRY(ctx_ok(ctx));
  HJ_TRY(check_params(ctx, params));
  if (n < 0) return set_err(ctx, HJ_ERR_ARG, "Number of particles must be non-negative. Got %lld.", (long long)n);
  if (n == 0) return evolve_empty(ctx, params, out);
  if (!z || !dE) return set_err(ctx, HJ_ERR_ARG, "particle arrays are NULL");
  double *d_z = nullptr, *d_dE = nullptr, *d_draws = nullptr;
  // the particle arrays: one block of the context's cache, kept for the next call
  void* blk = nullptr;
  size_t blk_cap = 0;
  const size_t half = align_up(sizeof(double) * (size_t)n);
  hj_status s = cache_take(ctx, false, 2 * half, &blk, &blk_cap);
  if (s == HJ_OK) {
    d_z = (double*)blk;
    d_dE = (double*)((char*)blk + half);
  }
  const bool draws = qe_draws && params->use_excitation && params->n_turns > 0;
  if (s == HJ_OK && draws) s = dalloc(ctx, &d_draws, (size_t)n * (size_t)params->n_turns);
  cudaStream_t st = ctx->stream;
  if (s == HJ_OK) {
    cudaError_t e = cudaMemcpyAsync(d_z, z, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_dE, dE, sizeof(double) * n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && draws)
      e = cudaMemcpyAsync(d_draws, qe_draws, sizeof(double) * n * params->n_turns,
                          cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) s = set_err(ctx, HJ_ERR_CUDA, "host->device copy failed: %s", cudaGetErrorString(e));
  }
  if (s == HJ_OK)
    s = hj_evolve_device(ctx, d_z, d_dE, n, params, wake, nbins, grid, d_draws, seed, st, out);
  if (s == HJ_OK) {
    cudaError_t e = cudaMemcpyAsync(z, d_z, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dE, d_dE, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) s = set_err(ctx, HJ_ERR_CUDA, "device->host copy failed: %s", cudaGetErrorString(e));
  }
  cudaStreamSynchronize(st);
  cache_give(ctx, false, blk, blk_cap);
  if (d_draws) cudaFree(d_draws);
  return s;
}

// ====================================================================== single steps

namespace {
// Copy n doubles of host arrays into the context scratch; returns device pointers.
hj_status stage(hj_ctx* ctx, int64_t n, int k, double** dev, const double* const* host) {
  void* base = nullptr;
  const size_t one = align_up(sizeof(double) * (size_t)(n > 0 ? n : 1));
  HJ_TRY(scratch(ctx, one * k, &base));
  for (int i = 0; i < k; ++i) {
    dev[i] = (double*)((char*)base + one * i);
    if (host[i] && n > 0)
      HJ_CUDA(ctx, cudaMemcpyAsync(dev[i], host[i], sizeof(double) * n, cudaMemcpyHostToDevice,
                                   ctx->stream));
  }
  return HJ_OK;
}

hj_status unstage(hj_ctx* ctx, int64_t n, double* host, const double* dev) {
  if (n > 0)
    HJ_CUDA(ctx, cudaMemcpyAsync(host, dev, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  HJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return HJ_OK;
}
}  // namespace

extern "C" hj_status hj_rf_kick(hj_ctx* ctx, double voltage, double sin_phis, double rf_factor,
                                double phi_s, const double* z, double* dE, int64_t n) {
  HJ_TRY(ctx_ok(ctx));
  if (n < 0 || (n > 0 && (!z || !dE))) return set_err(ctx, HJ_ERR_ARG, "bad particle arrays");
  if (n == 0) return HJ_OK;
  double* d[2];
  const double* h[2] = {z, dE};
  HJ_TRY(stage(ctx, n, 2, d, h));
  HJ_CUDA(ctx, launch_rf_kick(voltage, sin_phis, rf_factor, phi_s, d[0], d[1], n, ctx->stream));
  return unstage(ctx, n, dE, d[1]);
}

extern "C" hj_status hj_quantum_excitation(hj_ctx* ctx, double E0, double radius,
                                           double sigma_E0, const double* draws, uint64_t seed,
                                           int64_t turn, double* dE, int64_t n) {
  HJ_TRY(ctx_ok(ctx));
  if (n < 0 || (n > 0 && !dE)) return set_err(ctx, HJ_ERR_ARG, "bad particle arrays");
  if (n == 0) return HJ_OK;
  const double t = E0 / 1e9;
  const double dU = 4 * 8.85e-5 * (t * t * t) / radius;   // src/quantum_excitation.jl:58
  const double om = 1 - dU;
  const double excitation = std::sqrt(1 - om * om) * sigma_E0;  // :59
  double* d[2];
  const double* h[2] = {dE, draws};
  HJ_TRY(stage(ctx, n, 2, d, h));
  HJ_CUDA(ctx, launch_qe(excitation, draws ? d[1] : nullptr, seed, turn, d[0], n, ctx->stream));
  return unstage(ctx, n, dE, d[0]);
}

extern "C" hj_status hj_synchrotron_radiation(hj_ctx* ctx, double E0, double radius, double* dE,
                                              int64_t n) {
  HJ_TRY(ctx_ok(ctx));
  if (n < 0 || (n > 0 && !dE)) return set_err(ctx, HJ_ERR_ARG, "bad particle arrays");
  if (n == 0) return HJ_OK;
  const double t = E0 / 1e9;
  const double dU = 4 * 8.85e-5 * (t * t * t) / radius;  // src/synchrotron_radiation.jl:44
  const double damping = 1 - dU;                         // :45
  double* d[1];
  const double* h[1] = {dE};
  HJ_TRY(stage(ctx, n, 1, d, h));
  HJ_CUDA(ctx, launch_sr(damping, d[0], n, ctx->stream));
  return unstage(ctx, n, dE, d[0]);
}

extern "C" hj_status hj_phase_advance(hj_ctx* ctx, int32_t update_eta, double E0, double mass,
                                      double alpha_c, int64_t harmonic, double phi_s,
                                      double freq_rf, const double* dE, double* z, int64_t n) {
  HJ_TRY(ctx_ok(ctx));
  if (n < 0 || (n > 0 && (!z || !dE))) return set_err(ctx, HJ_ERR_ARG, "bad particle arrays");
  if (n == 0) return HJ_OK;
  hj_params p{};
  p.mass = mass;
  p.alpha_c = alpha_c;
  p.harmonic = harmonic;
  p.phi_s = phi_s;
  p.freq_rf = freq_rf;
  p.radius = 1.0;
  const TurnScalars s = make_turn_scalars(E0, p, 0.0);
  double* d[2];
  const double* h[2] = {z, dE};
  HJ_TRY(stage(ctx, n, 2, d, h));
  HJ_CUDA(ctx, launch_phase_advance(update_eta, s, 1.0 / mass, alpha_c,
                                    kTwoPi * (double)harmonic, phi_s, d[1], d[0], n,
                                    ctx->stream));
  return unstage(ctx, n, z, d[0]);
}

extern "C" hj_status hj_gaussian(hj_ctx* ctx, uint64_t seed, int64_t turn, int64_t n,
                                 double* out) {
  HJ_TRY(ctx_ok(ctx));
  if (n < 0 || (n > 0 && !out)) return set_err(ctx, HJ_ERR_ARG, "bad output array");
  if (n == 0) return HJ_OK;
  double* d[1];
  const double* h[1] = {nullptr};
  HJ_TRY(stage(ctx, n, 1, d, h));
  HJ_CUDA(ctx, launch_gaussian(seed, turn, n, d[0], ctx->stream));
  return unstage(ctx, n, out, d[0]);
}

extern "C" hj_status hj_normal_tables(double* out, int64_t cap) {
  if (!out || cap < HJ_NORMAL_TABLES_SIZE) return HJ_ERR_ARG;
  std::unique_ptr<NormalTables> tp(new NormalTables);   // 48 KB: not on the stack
  const NormalTables& t = *tp;
  host_normal_tables(tp.get());
  double* o = out;
  for (int i = 0; i < kZigLayers; ++i) {
    *o++ = t.xd[i][0];
    *o++ = t.xd[i][1];
  }
  for (int i = 0; i <= kZigLayers; ++i) *o++ = t.f[i];
  *o++ = t.r;
  *o++ = t.v;
  return o - out == HJ_NORMAL_TABLES_SIZE ? HJ_OK : HJ_ERR_STATE;
}

namespace {
// Device histogram of z on `grid` into dcnt (u64 counts), using scratch after `off` bytes.
hj_status device_histogram(hj_ctx* ctx, const double* d_z, int64_t n, const hj_grid* grid,
                           unsigned long long* dcnt, uint32_t* part, int nblk) {
  const int B = (int)grid->nbins;
  HJ_CUDA(ctx, launch_histogram_only(d_z, n, B, grid->edge_first, grid->edge_last,
                                     1.0 / grid->edge_step, part, nblk, ctx->stream));
  HJ_CUDA(ctx, launch_hist_reduce(part, nullptr, nblk, B, dcnt, true, ctx->stream));
  return HJ_OK;
}

int hist_blocks(hj_ctx* ctx, int64_t n) {
  int64_t g = (n + 8191) / 8192;
  if (g < 1) g = 1;
  if (g > ctx->num_sms * 2) g = ctx->num_sms * 2;
  return (int)g;
}

struct ConvBuffers {
  double* W;
  double* lam;
  double2* twP;
  double2* Wf;
  double2* Xg;
  double2* zE;
  double* pot;
  unsigned long long* cnt;
};

// Potential at the centers from device counts (conv_only bins kernel).
hj_status device_conv(hj_ctx* ctx, const hj_grid* grid, const hj_wake* wake, double current,
                      ConvBuffers& cb) {
  const int B = (int)grid->nbins;
  const int P = (int)next_pow2(2 * (int64_t)B), M = P / 2, H = M / 2;
  const int logH = H >= 1 ? ilog2(H) : 0;
  std::vector<double> W(B), lam(B), tw(2 * (size_t)P);
  host_wake_tables(grid->centers, B, *wake, W.data(), lam.data());
  host_twiddles(P, tw.data());
  HJ_CUDA(ctx, cudaMemcpyAsync(cb.W, W.data(), sizeof(double) * B, cudaMemcpyHostToDevice, ctx->stream));
  HJ_CUDA(ctx, cudaMemcpyAsync(cb.lam, lam.data(), sizeof(double) * B, cudaMemcpyHostToDevice, ctx->stream));
  HJ_CUDA(ctx, cudaMemcpyAsync(cb.twP, tw.data(), sizeof(double) * tw.size(), cudaMemcpyHostToDevice, ctx->stream));
  if (H >= 4)
    HJ_CUDA(ctx, launch_wake_spectrum(cb.W, B, P, M, H, logH, cb.twP, cb.Xg, cb.Wf, ctx->stream));
  BinsArgs g{};
  g.use_wake = 1;
  g.B = B;
  g.P = P;
  g.M = M;
  g.H = H;
  g.logH = logH;
  g.cnt = cb.cnt;
  g.cic = nullptr;
  g.lam = cb.lam;
  g.Wf = cb.Wf;
  g.twP = cb.twP;
  g.Xg = cb.Xg;
  g.zE = cb.zE;
  g.pot = cb.pot;
  g.W = cb.W;
  g.conv_only = 1;
  g.conv_current = current;
  HJ_CUDA(ctx, launch_bins(g, ctx->stream));
  HJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // host tables go out of scope
  return HJ_OK;
}

// Carve the conv buffers (and extra doubles) out of the context scratch.
hj_status conv_scratch(hj_ctx* ctx, int B, size_t extra_doubles, int extra_arrays,
                       int64_t part_words, ConvBuffers& cb, double** extra,
                       uint32_t** part) {
  const int P = (int)next_pow2(2 * (int64_t)B), M = P / 2, H = std::max(M / 2, 1);
  size_t sizes[] = {align_up(sizeof(double) * B),     align_up(sizeof(double) * B),
                    align_up(sizeof(double2) * P),    align_up(sizeof(double2) * (M + 1)),
                    align_up(sizeof(double2) * M),    align_up(sizeof(double2) * H),
                    align_up(sizeof(double) * B),     align_up(sizeof(uint64_t) * B),
                    align_up(sizeof(uint32_t) * (size_t)std::max<int64_t>(part_words, 1))};
  size_t total = 0;
  for (size_t s : sizes) total += s;
  const size_t ex = align_up(sizeof(double) * std::max<size_t>(extra_doubles, 1));
  total += ex * extra_arrays;
  void* base = nullptr;
  HJ_TRY(scratch(ctx, total, &base));
  char* p = (char*)base;
  cb.W = (double*)p; p += sizes[0];
  cb.lam = (double*)p; p += sizes[1];
  cb.twP = (double2*)p; p += sizes[2];
  cb.Wf = (double2*)p; p += sizes[3];
  cb.Xg = (double2*)p; p += sizes[4];
  cb.zE = (double2*)p; p += sizes[5];
  cb.pot = (double*)p; p += sizes[6];
  cb.cnt = (unsigned long long*)p; p += sizes[7];
  *part = (uint32_t*)p; p += sizes[8];
  for (int i = 0; i < extra_arrays; ++i) {
    extra[i] = (double*)p;
    p += ex;
  }
  return HJ_OK;
}
}  // namespace

extern "C" hj_status hj_histogram(hj_ctx* ctx, const double* z, int64_t n, const hj_grid* grid,
                                  int64_t* counts) {
  HJ_TRY(ctx_ok(ctx));
  HJ_TRY(check_grid(ctx, grid));
  if (n < 0 || (n > 0 && !z) || !counts) return set_err(ctx, HJ_ERR_ARG, "bad arrays");
  if (grid->nbins * (int64_t)sizeof(uint32_t) > (int64_t)ctx->max_smem_optin)
    return set_err(ctx, HJ_ERR_TOO_LARGE, "nbins = %lld too large for the shared-memory histogram",
                   (long long)grid->nbins);
  const int B = (int)grid->nbins;
  const int nblk = hist_blocks(ctx, n);
  ConvBuffers cb{};
  double* ex[1];
  uint32_t* part = nullptr;
  HJ_TRY(conv_scratch(ctx, B, (size_t)n, 1, (int64_t)nblk * B, cb, ex, &part));
  if (n > 0)
    HJ_CUDA(ctx, cudaMemcpyAsync(ex[0], z, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  HJ_TRY(device_histogram(ctx, ex[0], n, grid, cb.cnt, part, nblk));
  HJ_CUDA(ctx, cudaMemcpyAsync(counts, cb.cnt, sizeof(int64_t) * B, cudaMemcpyDeviceToHost, ctx->stream));
  HJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return HJ_OK;
}

extern "C" hj_status hj_wake_potential(hj_ctx* ctx, const int64_t* counts, const hj_grid* grid,
                                       const hj_wake* wake, double current, double* pot) {
  HJ_TRY(ctx_ok(ctx));
  HJ_TRY(check_grid(ctx, grid));
  if (!counts || !wake || !pot) return set_err(ctx, HJ_ERR_ARG, "bad arrays");
  if (grid->nbins > kMaxBins)
    return set_err(ctx, HJ_ERR_TOO_LARGE, "nbins = %lld exceeds the supported %lld",
                   (long long)grid->nbins, (long long)kMaxBins);
  if (wake->ctau <= 0) return set_err(ctx, HJ_ERR_WAKE_PARAM, "Wake parameter cτ must be positive.");
  const int B = (int)grid->nbins;
  for (int i = 0; i < B; ++i)
    if (counts[i] < 0) return set_err(ctx, HJ_ERR_ARG, "negative bin count");
  ConvBuffers cb{};
  uint32_t* part = nullptr;
  HJ_TRY(conv_scratch(ctx, B, 0, 0, 0, cb, nullptr, &part));
  HJ_CUDA(ctx, cudaMemcpyAsync(cb.cnt, counts, sizeof(int64_t) * B, cudaMemcpyHostToDevice, ctx->stream));
  HJ_TRY(device_conv(ctx, grid, wake, current, cb));
  HJ_CUDA(ctx, cudaMemcpyAsync(pot, cb.pot, sizeof(double) * B, cudaMemcpyDeviceToHost, ctx->stream));
  HJ_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return HJ_OK;
}

extern "C" hj_status hj_apply_wakefield(hj_ctx* ctx, const double* z, double* dE, int64_t n,
                                        const hj_wake* wake, double current, double sigma_z,
                                        const hj_grid* grid) {
  (void)sigma_z;  // unused by the reference's MPI branch as well
  HJ_TRY(ctx_ok(ctx));
  HJ_TRY(check_grid(ctx, grid));
  if (n < 0 || (n > 0 && (!z || !dE)) || !wake) return set_err(ctx, HJ_ERR_ARG, "bad arrays");
  if (grid->nbins > kMaxBins)
    return set_err(ctx, HJ_ERR_TOO_LARGE, "nbins = %lld exceeds the supported %lld",
                   (long long)grid->nbins, (long long)kMaxBins);
  if (wake->ctau <= 0) return set_err(ctx, HJ_ERR_WAKE_PARAM, "Wake parameter cτ must be positive.");
  const int B = (int)grid->nbins;
  const int nblk = hist_blocks(ctx, n);
  ConvBuffers cb{};
  double* ex[2];
  uint32_t* part = nullptr;
  HJ_TRY(conv_scratch(ctx, B, (size_t)n, 2, (int64_t)nblk * B, cb, ex, &part));
  if (n > 0) {
    HJ_CUDA(ctx, cudaMemcpyAsync(ex[0], z, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
    HJ_CUDA(ctx, cudaMemcpyAsync(ex[1], dE, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  }
  HJ_TRY(device_histogram(ctx, ex[0], n, grid, cb.cnt, part, nblk));
  HJ_TRY(device_conv(ctx, grid, wake, current, cb));
  if (n > 0) {
    const double c1 = grid->centers[0], cB = grid->centers[B - 1];
    const double inv_c = B >= 2 ? 1.0 / ((cB - c1) / (double)(B - 1)) : 0.0;
    HJ_CUDA(ctx, launch_interp_kick(ex[0], ex[1], n, cb.pot, B, c1, cB, inv_c, ctx->stream));
  }
  return unstage(ctx, n, dE, ex[1]);
}
