// hj_batch.cu -- batches of independent bunches (hj_batch_*): one particle
// pool, one turn-state array, per turn one batched pass over a chunk table,
// one merge of the chunk partials and one batched bins step; turn blocks
// replayed from a CUDA graph.
#include "hj_ranges.h"
#include "hj_state.h"

// ====================================================================== batches
//
// A batch holds hj_bunch objects whose particles live in one pool and whose
// turn state lives in one device array (slot per bunch), so a poll is one
// copy.  Per turn: k_batch_pass over the chunk table, k_batch_reduce, and
// k_batch_bins (one 2-CTA cluster per bunch); the kernels read the bunch
// tables and the live counts from device memory and are launched over the
// batch's capacity, so a captured graph stays valid as bunches come and go.
// A bunch's chunking depends only on its own size and the batch's chunk size,
// so its sums -- and its results -- do not depend on the other bunches.

struct BatchMember {
  int64_t id = 0;
  hj_bunch* b = nullptr;
  int64_t start = 0, cap = 0;   // pool range [start, start + cap)
  int slot = 0;                 // index into the turn-state array
  int64_t turns = 0;
};

struct hj_batch {
  hj_ctx* ctx = nullptr;
  bool holds_ctx = false;                      // counted in ctx->live_objects
  cudaStream_t stream = nullptr;
  int cfg = 0;
  int64_t chunk = 65536;
  int max_bunches = 0, max_B = 0, max_H = 0, max_chunks = 0;
  // launch widths: the live counts rounded up to a power of two (a captured
  // graph is re-captured only when the live counts outgrow them)
  int grid_chunks = 0, grid_bunches = 0, grid_items = 0;
  int wake = -1, qe = -1;                      // fixed by the first bunch
  int64_t pool_n = 0;
  double* pool_z = nullptr;
  double* pool_dE = nullptr;
  hj_ranges::Ranges free_ranges;               // free pool ranges (first fit)
  std::vector<BatchMember> members;            // dense: index = device table slot
  std::vector<int> free_slots;
  int64_t next_id = 1;
  TurnState* d_ts = nullptr;                   // [max_bunches]
  TurnState* h_ts = nullptr;                   // pinned copy for polls
  PassArgs* d_pass = nullptr;
  BinsArgs* d_bins = nullptr;
  BatchChunk* d_chunks = nullptr;
  BatchChunk* d_items = nullptr;               // merge table: groups of a bunch's partial slots
  int32_t* d_counts = nullptr;                 // [0] chunks, [1] bunches, [2] merge items,
                                               // [3] the resident pass's chunk queue
  bool resident = false;                       // the pass: resident blocks on a chunk queue
  int resident_blocks = 0;                     // their number (SMs x blocks per SM)
  PassArgs* h_pass = nullptr;                  // pinned staging
  BinsArgs* h_bins = nullptr;
  BatchChunk* h_chunks = nullptr;
  BatchChunk* h_items = nullptr;
  int32_t* h_counts = nullptr;
  // the buffers above are carved from one device and one pinned cached block
  void* arena = nullptr;
  size_t arena_cap = 0;
  void* harena = nullptr;
  size_t harena_cap = 0;
  bool dirty = true;
  int bins_ctas = 2;                           // CTAs per bunch in the bins step
  int graph_turns = 16;
  cudaGraphExec_t graph = nullptr;
  int64_t turns_enqueued = 0;
};

namespace {

hj_status batch_alloc_range(hj_batch* bt, int64_t n, int64_t* start, int64_t* cap) {
  return hj_ranges::take(bt->free_ranges, n, start, cap) ? HJ_OK : HJ_ERR_FULL;
}

void batch_free_range(hj_batch* bt, int64_t start, int64_t cap) {
  hj_ranges::give(bt->free_ranges, start, cap);
}

int64_t batch_largest_free(const hj_batch* bt) { return hj_ranges::largest(bt->free_ranges); }

// Rebuild and upload the device tables (bunch arguments, chunk table, counts).
hj_status batch_upload(hj_batch* bt) {
  hj_ctx* ctx = bt->ctx;
  HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));   // staging buffers are free again
  int nch = 0;
  const int nb = (int)bt->members.size();
  for (int k = 0; k < nb; ++k) {
    hj_bunch* b = bt->members[k].b;
    fill_turn_args(b, bt->h_pass[k], bt->h_bins[k]);
    for (int c = 0; c < b->nblk; ++c) {
      BatchChunk ch;
      ch.first = (int64_t)c * bt->chunk;
      ch.count = std::min<int64_t>(bt->chunk, b->n - ch.first);
      ch.bunch = k;
      ch.part = c;
      if (nch >= bt->max_chunks) return set_err(ctx, HJ_ERR_STATE, "batch chunk table overflow");
      bt->h_chunks[nch++] = ch;
    }
  }
  // full chunks first, then the partial ones largest first: the last wave of
  // blocks is made of the shortest chunks
  std::stable_sort(bt->h_chunks, bt->h_chunks + nch,
                   [](const BatchChunk& x, const BatchChunk& y) { return x.count > y.count; });
  // merge table: each bunch's partial slots in groups of kMergeGroup
  constexpr int kMergeGroup = 4;
  int nit = 0;
  for (int k = 0; k < nb; ++k) {
    const int np = bt->members[k].b->nblk;
    for (int p0 = 0; p0 < np; p0 += kMergeGroup) {
      if (nit >= bt->max_chunks) return set_err(ctx, HJ_ERR_STATE, "batch merge table overflow");
      BatchChunk it;
      it.first = p0;
      it.count = std::min(kMergeGroup, np - p0);
      it.bunch = k;
      it.part = 0;
      bt->h_items[nit++] = it;
    }
  }
  bt->h_counts[0] = nch;
  bt->h_counts[1] = nb;
  bt->h_counts[2] = nit;
  if (nch > bt->grid_chunks || nb > bt->grid_bunches || nit > bt->grid_items) {
    bt->grid_chunks = std::max(bt->grid_chunks, (int)std::min<int64_t>(next_pow2(nch), bt->max_chunks));
    bt->grid_bunches = std::max(bt->grid_bunches, (int)std::min<int64_t>(next_pow2(nb), bt->max_bunches));
    bt->grid_items = std::max(bt->grid_items, (int)std::min<int64_t>(next_pow2(nit), bt->max_chunks));
    if (bt->graph) {
      cudaGraphExecDestroy(bt->graph);
      bt->graph = nullptr;
    }
  }
  if (nb > 0) {
    HJ_CUDA(ctx, cudaMemcpyAsync(bt->d_pass, bt->h_pass, sizeof(PassArgs) * nb,
                                 cudaMemcpyHostToDevice, bt->stream));
    HJ_CUDA(ctx, cudaMemcpyAsync(bt->d_bins, bt->h_bins, sizeof(BinsArgs) * nb,
                                 cudaMemcpyHostToDevice, bt->stream));
  }
  if (nch > 0)
    HJ_CUDA(ctx, cudaMemcpyAsync(bt->d_chunks, bt->h_chunks, sizeof(BatchChunk) * nch,
                                 cudaMemcpyHostToDevice, bt->stream));
  if (nit > 0)
    HJ_CUDA(ctx, cudaMemcpyAsync(bt->d_items, bt->h_items, sizeof(BatchChunk) * nit,
                                 cudaMemcpyHostToDevice, bt->stream));
  HJ_CUDA(ctx, cudaMemcpyAsync(bt->d_counts, bt->h_counts, sizeof(int32_t) * 3,
                               cudaMemcpyHostToDevice, bt->stream));
  bt->dirty = false;
  return HJ_OK;
}

hj_status batch_launch_turn(hj_batch* bt) {
  hj_ctx* ctx = bt->ctx;
  HJ_CUDA(ctx, launch_batch_pass(bt->d_pass, bt->d_chunks, bt->d_counts, bt->grid_chunks,
                                 bt->max_B, bt->wake, bt->qe, bt->cfg,
                                 bt->resident ? bt->d_counts + 3 : nullptr, bt->resident_blocks,
                                 bt->stream));
  if (bt->wake)
    HJ_CUDA(ctx, launch_batch_reduce(bt->d_pass, bt->d_items, bt->d_counts + 2, bt->grid_items,
                                     bt->max_B, bt->stream));
  HJ_CUDA(ctx, launch_batch_bins(bt->d_bins, bt->d_counts + 1, bt->grid_bunches, bt->max_H,
                                 bt->bins_ctas, bt->stream));
  return HJ_OK;
}

hj_status batch_capture(hj_batch* bt) {
  hj_ctx* ctx = bt->ctx;
  cudaGraph_t g = nullptr;
  HJ_CUDA(ctx, cudaStreamBeginCapture(bt->stream, cudaStreamCaptureModeThreadLocal));
  hj_status s = HJ_OK;
  for (int t = 0; t < bt->graph_turns && s == HJ_OK; ++t) s = batch_launch_turn(bt);
  cudaError_t e = cudaStreamEndCapture(bt->stream, &g);
  if (s != HJ_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess)
    return set_err(ctx, HJ_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&bt->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess)
    return set_err(ctx, HJ_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
  return HJ_OK;
}

int batch_find(const hj_batch* bt, int64_t id) {
  for (size_t k = 0; k < bt->members.size(); ++k)
    if (bt->members[k].id == id) return (int)k;
  return -1;
}

}  // namespace

extern "C" void hj_batch_destroy(hj_batch* bt) {
  if (!bt) return;
  if (!bt->ctx) {
    delete bt;
    return;
  }
  cudaSetDevice(bt->ctx->device);
  if (bt->stream) cudaStreamSynchronize(bt->stream);
  for (auto& m : bt->members) {
    m.b->ts = nullptr;   // lives in the batch's array
    hj_bunch_destroy(m.b);
  }
  if (bt->graph) cudaGraphExecDestroy(bt->graph);
  cache_give(bt->ctx, false, bt->arena, bt->arena_cap);
  cache_give(bt->ctx, true, bt->harena, bt->harena_cap);
  if (bt->stream) cudaStreamDestroy(bt->stream);
  hj_ctx* ctx = bt->ctx;
  const bool held = bt->holds_ctx;
  delete bt;
  if (held) ctx_release(ctx);
}

static hj_status batch_create_impl(hj_ctx* ctx, int64_t pool_particles, int32_t max_bunches,
                                   int32_t max_nbins, int64_t chunk, int32_t layout,
                                   hj_batch* bt) {
  bt->ctx = ctx;
  ctx_retain(ctx);
  bt->holds_ctx = true;
  bt->chunk = chunk;
  bt->max_bunches = max_bunches;
  bt->max_B = max_nbins;
  const int64_t P = next_pow2(2 * (int64_t)max_nbins);
  bt->max_H = (int)std::max<int64_t>(P / 4, 4);
  bt->bins_ctas = batch_bins_ctas(bt->max_H, max_bunches, ctx->num_sms);
  bt->cfg = auto_pass_layout(layout, max_nbins, pool_particles);
  bt->pool_n = (pool_particles + 3) / 4 * 4;
  bt->max_chunks = (int)std::min<int64_t>(bt->pool_n / chunk + max_bunches + 1, INT32_MAX);
  HJ_CUDA(ctx, cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking));
  // the pool and the tables: one device and one pinned block of the context's cache
  const size_t nb = (size_t)max_bunches, nc = (size_t)bt->max_chunks;
  Carve c;
  const size_t o_z = c.add<double>((size_t)bt->pool_n), o_e = c.add<double>((size_t)bt->pool_n);
  const size_t o_ts = c.add<TurnState>(nb), o_pass = c.add<PassArgs>(nb);
  const size_t o_bins = c.add<BinsArgs>(nb), o_ch = c.add<BatchChunk>(nc);
  const size_t o_it = c.add<BatchChunk>(nc), o_cnt = c.add<int32_t>(4);
  HJ_TRY(cache_take(ctx, false, c.off, &bt->arena, &bt->arena_cap));
  char* a = (char*)bt->arena;
  bt->pool_z = (double*)(a + o_z);
  bt->pool_dE = (double*)(a + o_e);
  bt->d_ts = (TurnState*)(a + o_ts);
  bt->d_pass = (PassArgs*)(a + o_pass);
  bt->d_bins = (BinsArgs*)(a + o_bins);
  bt->d_chunks = (BatchChunk*)(a + o_ch);
  bt->d_items = (BatchChunk*)(a + o_it);
  bt->d_counts = (int32_t*)(a + o_cnt);
  Carve h;
  const size_t p_ts = h.add<TurnState>(nb), p_pass = h.add<PassArgs>(nb);
  const size_t p_bins = h.add<BinsArgs>(nb), p_ch = h.add<BatchChunk>(nc);
  const size_t p_it = h.add<BatchChunk>(nc), p_cnt = h.add<int32_t>(3);
  HJ_TRY(cache_take(ctx, true, h.off, &bt->harena, &bt->harena_cap));
  char* q = (char*)bt->harena;
  bt->h_ts = (TurnState*)(q + p_ts);
  bt->h_pass = (PassArgs*)(q + p_pass);
  bt->h_bins = (BinsArgs*)(q + p_bins);
  bt->h_chunks = (BatchChunk*)(q + p_ch);
  bt->h_items = (BatchChunk*)(q + p_it);
  bt->h_counts = (int32_t*)(q + p_cnt);
  HJ_CUDA(ctx, cudaMemsetAsync(bt->d_counts, 0, sizeof(int32_t) * 4, bt->stream));
  HJ_CUDA(ctx, cudaMemsetAsync(bt->d_ts, 0, sizeof(TurnState) * max_bunches, bt->stream));
  bt->free_ranges.push_back({0, bt->pool_n});
  for (int s = max_bunches - 1; s >= 0; --s) bt->free_slots.push_back(s);
  HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));
  return HJ_OK;
}

extern "C" hj_status hj_batch_create(hj_ctx* ctx, int64_t pool_particles, int32_t max_bunches,
                                     int32_t max_nbins, int64_t chunk_particles,
                                     int32_t layout, hj_batch** out) {
  HJ_TRY(ctx_ok(ctx));
  if (!out) return set_err(ctx, HJ_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (pool_particles <= 0 || max_bunches <= 0)
    return set_err(ctx, HJ_ERR_ARG, "pool_particles and max_bunches must be positive");
  if (max_nbins <= 0) return set_err(ctx, HJ_ERR_NBINS, "Buffer nbins invalid (must be > 0).");
  if (max_nbins > kMaxBins)
    return set_err(ctx, HJ_ERR_TOO_LARGE, "max_nbins = %d exceeds the supported %lld",
                   max_nbins, (long long)kMaxBins);
  if (chunk_particles == 0) chunk_particles = 65536;
  if (chunk_particles < 4 || chunk_particles % 4 || chunk_particles > kMaxBlockParticles)
    return set_err(ctx, HJ_ERR_ARG, "chunk_particles must be a positive multiple of 4, at most %lld",
                   (long long)kMaxBlockParticles);
  if (!pass_request_valid(layout))
    return set_err(ctx, HJ_ERR_ARG,
                   "pass layout must be -1 (automatic), %d (automatic, single-precision normals), "
                   "0..%d or 8..%d, plus %d for single-precision normals",
                   kPassAutoFast, kNumPassCfgs - 1, kPassN32 + kNumPassCfgs - 1, kPassFastNormals);
  hj_batch* bt = new hj_batch();
  hj_status s = batch_create_impl(ctx, pool_particles, max_bunches, max_nbins, chunk_particles,
                                  layout, bt);
  if (s != HJ_OK) {
    hj_batch_destroy(bt);
    return s;
  }
  *out = bt;
  return HJ_OK;
}

extern "C" hj_status hj_batch_set_resident(hj_batch* bt, int32_t on) {
  if (!bt) return HJ_ERR_ARG;
  if (bt->graph) {
    HJ_CUDA(bt->ctx, cudaStreamSynchronize(bt->stream));
    cudaGraphExecDestroy(bt->graph);
    bt->graph = nullptr;
  }
  bt->resident = on != 0;
  return HJ_OK;
}

extern "C" hj_status hj_batch_set_graph_turns(hj_batch* bt, int32_t turns) {
  if (!bt) return HJ_ERR_ARG;
  if (turns < 0) return set_err(bt->ctx, HJ_ERR_ARG, "graph turns must be >= 0");
  if (bt->graph) {
    HJ_CUDA(bt->ctx, cudaStreamSynchronize(bt->stream));
    cudaGraphExecDestroy(bt->graph);
    bt->graph = nullptr;
  }
  bt->graph_turns = turns;
  return HJ_OK;
}

// z, dE != NULL: copy them into the pool; else generate independent
// Gaussians (σ_z, σ_E) from init_seed in place.
// Admission in two halves (see bunch_create_begin): the first checks the
// bunch, reserves its slot and pool range, fills its particles and enqueues
// its initial moments; the second, after the stream has reached them,
// completes the bunch and makes it a member.
struct PendingAdd {
  hj_bunch* b = nullptr;
  int64_t start = 0, cap = 0, turns = 0;
  int slot = -1;
};

static void batch_add_abort(hj_batch* bt, PendingAdd& p) {
  if (p.b) hj_bunch_destroy(p.b);
  if (p.cap) batch_free_range(bt, p.start, p.cap);
  if (p.slot >= 0) bt->free_slots.push_back(p.slot);
  p = PendingAdd{};
}

static hj_status batch_add_begin(hj_batch* bt, const double* z, const double* dE, int64_t n,
                                 const hj_params* params, const hj_wake* wake, int64_t nbins,
                                 uint64_t seed, int64_t turns, double sigma_z, double sigma_E,
                                 uint64_t init_seed, PendingAdd* out) {
  hj_ctx* ctx = bt->ctx;
  HJ_TRY(check_params(ctx, params));
  if (n <= 0) return set_err(ctx, HJ_ERR_ARG, "a batch bunch needs at least one particle");
  if (turns < 0) return set_err(ctx, HJ_ERR_ARG, "turns must be >= 0");
  const int wake_on = params->use_wakefield ? 1 : 0;
  const int qe = params->use_excitation ? QE_PHILOX : QE_OFF;
  if ((bt->wake >= 0 && bt->wake != wake_on) || (bt->qe >= 0 && bt->qe != qe))
    return set_err(ctx, HJ_ERR_ARG,
                   "all bunches of a batch share the wakefield and quantum-excitation switches");
  if (wake_on && nbins > bt->max_B)
    return set_err(ctx, HJ_ERR_FULL, "nbins = %lld exceeds the batch's %d",
                   (long long)nbins, bt->max_B);
  if (bt->free_slots.empty()) return set_err(ctx, HJ_ERR_FULL, "the batch's bunch slots are full");
  PendingAdd p;
  if (batch_alloc_range(bt, n, &p.start, &p.cap) != HJ_OK)
    return set_err(ctx, HJ_ERR_FULL, "no free pool range of %lld particles", (long long)n);
  p.slot = bt->free_slots.back();
  bt->free_slots.pop_back();
  p.turns = turns;
  double* dz = bt->pool_z + p.start;
  double* de = bt->pool_dE + p.start;
  cudaError_t e;
  if (z) {
    e = cudaMemcpyAsync(dz, z, sizeof(double) * n, cudaMemcpyDefault, bt->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(de, dE, sizeof(double) * n, cudaMemcpyDefault, bt->stream);
  } else {
    e = launch_gaussian_bunch(init_seed, n, 0.0, sigma_z, 0.0, sigma_E, dz, de, bt->stream);
  }
  if (e != cudaSuccess) {
    batch_add_abort(bt, p);
    return set_err(ctx, HJ_ERR_CUDA, "copying the bunch into the pool failed: %s",
                   cudaGetErrorString(e));
  }
  p.b = new hj_bunch();
  hj_status s = bunch_create_begin(ctx, dz, de, n, params, wake, nbins, nullptr, seed,
                                   (void*)bt->stream, p.b, bt->chunk, bt->cfg);
  if (s == HJ_OK && p.b->nblk > bt->max_chunks) s = set_err(ctx, HJ_ERR_FULL, "chunk table full");
  if (s != HJ_OK) {
    batch_add_abort(bt, p);
    return s;
  }
  if (bt->resident_blocks == 0 || bt->wake != wake_on || bt->qe != qe)
    bt->resident_blocks = ctx->num_sms * batch_blocks_per_sm(bt->max_B, qe, wake_on, bt->cfg);
  bt->wake = wake_on;
  bt->qe = qe;
  *out = p;
  return HJ_OK;
}

static hj_status batch_add_end(hj_batch* bt, PendingAdd& p, int64_t* id_out) {
  hj_ctx* ctx = bt->ctx;
  hj_status s = bunch_create_end(ctx, p.b, nullptr);
  if (s != HJ_OK) {
    batch_add_abort(bt, p);
    return s;
  }
  // move the turn state into the batch's array, with this bunch's turn budget
  hj_bunch* b = p.b;
  b->h_ts->turns_left = p.turns;
  b->ts = bt->d_ts + p.slot;         // the arena's own TurnState stays unused
  cudaError_t e = cudaMemcpyAsync(b->ts, b->h_ts, sizeof(TurnState), cudaMemcpyHostToDevice,
                                  bt->stream);   // ordered before the next turn's kernels
  if (e != cudaSuccess) {
    batch_add_abort(bt, p);
    return set_err(ctx, HJ_ERR_CUDA, "turn state upload failed: %s", cudaGetErrorString(e));
  }
  BatchMember m;
  m.id = bt->next_id++;
  m.b = b;
  m.start = p.start;
  m.cap = p.cap;
  m.slot = p.slot;
  m.turns = p.turns;
  bt->members.push_back(m);
  bt->dirty = true;
  *id_out = m.id;
  p = PendingAdd{};
  return HJ_OK;
}

static hj_status batch_add_impl(hj_batch* bt, const double* z, const double* dE, int64_t n,
                                const hj_params* params, const hj_wake* wake, int64_t nbins,
                                uint64_t seed, int64_t turns, int64_t* id_out, double sigma_z,
                                double sigma_E, uint64_t init_seed) {
  if (!bt) return HJ_ERR_ARG;
  hj_ctx* ctx = bt->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (!id_out) return set_err(ctx, HJ_ERR_ARG, "id_out is NULL");
  *id_out = 0;
  HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));
  PendingAdd p;
  HJ_TRY(batch_add_begin(bt, z, dE, n, params, wake, nbins, seed, turns, sigma_z, sigma_E,
                         init_seed, &p));
  cudaError_t e = cudaStreamSynchronize(bt->stream);
  if (e != cudaSuccess) {
    batch_add_abort(bt, p);
    return set_err(ctx, HJ_ERR_CUDA, "%s", cudaGetErrorString(e));
  }
  return batch_add_end(bt, p, id_out);
}

extern "C" hj_status hj_batch_add(hj_batch* bt, const double* z, const double* dE, int64_t n,
                                  const hj_params* params, const hj_wake* wake, int64_t nbins,
                                  uint64_t seed, int64_t turns, int64_t* id_out) {
  if (bt && (!z || !dE)) return set_err(bt->ctx, HJ_ERR_ARG, "particle arrays are NULL");
  return batch_add_impl(bt, z, dE, n, params, wake, nbins, seed, turns, id_out, 0.0, 0.0, 0);
}

extern "C" hj_status hj_batch_add_gaussian(hj_batch* bt, int64_t n, double sigma_z,
                                           double sigma_E, uint64_t init_seed,
                                           const hj_params* params, const hj_wake* wake,
                                           int64_t nbins, uint64_t seed, int64_t turns,
                                           int64_t* id_out) {
  if (bt && !(sigma_z >= 0.0 && sigma_E >= 0.0))
    return set_err(bt->ctx, HJ_ERR_ARG, "spreads must be non-negative");
  return batch_add_impl(bt, nullptr, nullptr, n, params, wake, nbins, seed, turns, id_out,
                        sigma_z, sigma_E, init_seed);
}

extern "C" hj_status hj_batch_add_many(hj_batch* bt, int32_t count, const double* const* z,
                                       const double* const* dE, const int64_t* n,
                                       const hj_params* params, const hj_wake* wakes,
                                       const int64_t* nbins, const uint64_t* seeds,
                                       const int64_t* turns, int64_t* ids_out,
                                       int32_t* n_added) {
  if (!bt) return HJ_ERR_ARG;
  hj_ctx* ctx = bt->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (!n_added) return set_err(ctx, HJ_ERR_ARG, "n_added is NULL");
  *n_added = 0;
  if (count < 0) return set_err(ctx, HJ_ERR_ARG, "count must be >= 0");
  if (count > 0 && (!z || !dE || !n || !params || !nbins || !seeds || !turns || !ids_out))
    return set_err(ctx, HJ_ERR_ARG, "an argument array is NULL");
  HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));
  std::vector<PendingAdd> pend;
  pend.reserve(count);
  hj_status first = HJ_OK;
  std::string first_msg;
  for (int k = 0; k < count; ++k) {
    PendingAdd p;
    hj_status s = (!z[k] || !dE[k])
                      ? set_err(ctx, HJ_ERR_ARG, "particle arrays of bunch %d are NULL", k)
                      : batch_add_begin(bt, z[k], dE[k], n[k], &params[k],
                                        wakes ? &wakes[k] : nullptr, nbins[k], seeds[k],
                                        turns[k], 0.0, 0.0, 0, &p);
    if (s != HJ_OK) {
      first = s;
      first_msg = ctx->err;
      break;
    }
    pend.push_back(p);
  }
  cudaError_t e = cudaStreamSynchronize(bt->stream);
  if (e != cudaSuccess) {
    for (auto& p : pend) batch_add_abort(bt, p);
    return set_err(ctx, HJ_ERR_CUDA, "%s", cudaGetErrorString(e));
  }
  for (size_t k = 0; k < pend.size(); ++k) {
    hj_status s = batch_add_end(bt, pend[k], &ids_out[k]);
    if (s != HJ_OK) {
      for (size_t j = k + 1; j < pend.size(); ++j) batch_add_abort(bt, pend[j]);
      *n_added = (int32_t)k;
      return s;
    }
  }
  *n_added = (int32_t)pend.size();
  if (first != HJ_OK) ctx->err = first_msg;
  return first;
}

extern "C" hj_status hj_batch_take_many(hj_batch* bt, int32_t count, const int64_t* ids,
                                        double* const* z_out, double* const* dE_out,
                                        hj_result* res, double* corr_out) {
  if (!bt) return HJ_ERR_ARG;
  hj_ctx* ctx = bt->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (count < 0 || (count > 0 && !ids)) return set_err(ctx, HJ_ERR_ARG, "bad id list");
  std::vector<hj_bunch*> bs(count);
  for (int k = 0; k < count; ++k) {
    const int j = batch_find(bt, ids[k]);
    if (j < 0) return set_err(ctx, HJ_ERR_ARG, "no bunch %lld in the batch", (long long)ids[k]);
    for (int q = 0; q < k; ++q)
      if (ids[q] == ids[k]) return set_err(ctx, HJ_ERR_ARG, "bunch %lld listed twice", (long long)ids[k]);
    bs[k] = bt->members[j].b;
  }
  // one round trip for all: pending kick and re-centring in place, moments,
  // turn state, copies out, and every slot's state set to "no turns left"
  TurnState dead{};
  dead.turns_left = 0;
  for (int k = 0; k < count; ++k) {
    hj_bunch* b = bs[k];
    HJ_TRY(launch_moments(b, 1, b->z, b->dE));
    HJ_CUDA(ctx, cudaMemcpyAsync(b->h_mom, b->part_mom, sizeof(double) * 4 * b->nblk_m,
                                 cudaMemcpyDeviceToHost, bt->stream));
    HJ_CUDA(ctx, cudaMemcpyAsync(b->h_ts, b->ts, sizeof(TurnState), cudaMemcpyDeviceToHost,
                                 bt->stream));
    if (z_out && z_out[k])
      HJ_CUDA(ctx, cudaMemcpyAsync(z_out[k], b->z, sizeof(double) * b->n, cudaMemcpyDefault,
                                   bt->stream));
    if (dE_out && dE_out[k])
      HJ_CUDA(ctx, cudaMemcpyAsync(dE_out[k], b->dE, sizeof(double) * b->n, cudaMemcpyDefault,
                                   bt->stream));
    HJ_CUDA(ctx, cudaMemcpyAsync(b->ts, &dead, sizeof(TurnState), cudaMemcpyHostToDevice,
                                 bt->stream));
  }
  HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));
  hj_status st = HJ_OK;
  std::vector<double> mean_z(count), mean_e(count);
  for (int k = 0; k < count; ++k) {
    hj_bunch* b = bs[k];
    double m[4];
    sum_moments(b, m);
    hj_status s = state_status(b);
    if (st == HJ_OK) st = s;
    if (res) fill_result(b, m, &res[k]);
    mean_z[k] = m[0] / (double)b->n;
    mean_e[k] = m[2] / (double)b->n;
  }
  if (corr_out) {
    // cor(z, ΔE) of the final particles (the second pass of hj_correlation,
    // about the means above), partial sums in the moments' buffers
    for (int k = 0; k < count; ++k) {
      hj_bunch* b = bs[k];
      HJ_CUDA(ctx, launch_cor_parts(b->z, b->dE, b->n, mean_z[k], mean_e[k], 1, b->part_mom,
                                    b->nblk_m, bt->stream));
      HJ_CUDA(ctx, cudaMemcpyAsync(b->h_mom, b->part_mom, sizeof(double) * 3 * b->nblk_m,
                                   cudaMemcpyDeviceToHost, bt->stream));
    }
    HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));
    for (int k = 0; k < count; ++k) {
      hj_bunch* b = bs[k];
      double sxx = 0.0, syy = 0.0, sxy = 0.0;
      for (int q = 0; q < b->nblk_m; ++q) {
        sxx += b->h_mom[3 * q];
        syy += b->h_mom[3 * q + 1];
        sxy += b->h_mom[3 * q + 2];
      }
      const double r = sxy / (std::sqrt(sxx) * std::sqrt(syy));
      corr_out[k] = r != r ? r : std::min(1.0, std::max(-1.0, r));
    }
  }
  for (int k = 0; k < count; ++k) {
    const int j = batch_find(bt, ids[k]);
    BatchMember m = bt->members[j];
    m.b->ts = nullptr;
    hj_bunch_destroy(m.b);
    batch_free_range(bt, m.start, m.cap);
    bt->free_slots.push_back(m.slot);
    bt->members[j] = bt->members.back();
    bt->members.pop_back();
  }
  bt->dirty = true;
  return st;
}

extern "C" hj_status hj_gaussian_bunch(hj_ctx* ctx, uint64_t init_seed, int64_t n,
                                       double sigma_z, double sigma_E, double* d_z,
                                       double* d_dE, void* stream) {
  HJ_TRY(ctx_ok(ctx));
  if (n < 0 || (n > 0 && (!d_z || !d_dE))) return set_err(ctx, HJ_ERR_ARG, "bad particle arrays");
  if (!(sigma_z >= 0.0 && sigma_E >= 0.0)) return set_err(ctx, HJ_ERR_ARG, "spreads must be non-negative");
  if (n == 0) return HJ_OK;
  HJ_CUDA(ctx, launch_gaussian_bunch(init_seed, n, 0.0, sigma_z, 0.0, sigma_E, d_z, d_dE,
                                     (cudaStream_t)stream));
  return HJ_OK;
}

extern "C" hj_status hj_batch_advance(hj_batch* bt, int64_t turns) {
  if (!bt) return HJ_ERR_ARG;
  hj_ctx* ctx = bt->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (turns < 0) return set_err(ctx, HJ_ERR_ARG, "turns must be >= 0");
  if (bt->members.empty() || turns == 0) return HJ_OK;
  if (bt->dirty) HJ_TRY(batch_upload(bt));
  int64_t t = 0;
  if (bt->graph_turns > 0 && turns >= bt->graph_turns) {
    if (!bt->graph) HJ_TRY(batch_capture(bt));
    for (; t + bt->graph_turns <= turns; t += bt->graph_turns)
      HJ_CUDA(ctx, cudaGraphLaunch(bt->graph, bt->stream));
  }
  for (; t < turns; ++t) HJ_TRY(batch_launch_turn(bt));
  bt->turns_enqueued += turns;
  return HJ_OK;
}

extern "C" hj_status hj_batch_poll(hj_batch* bt, int64_t* ids, int32_t cap, int32_t* n_done) {
  if (!bt || !n_done || (cap > 0 && !ids)) return HJ_ERR_ARG;
  hj_ctx* ctx = bt->ctx;
  HJ_TRY(ctx_ok(ctx));
  *n_done = 0;
  HJ_CUDA(ctx, cudaMemcpyAsync(bt->h_ts, bt->d_ts, sizeof(TurnState) * bt->max_bunches,
                               cudaMemcpyDeviceToHost, bt->stream));
  HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));
  for (auto& m : bt->members) {
    if (bt->h_ts[m.slot].turns_left <= 0 && *n_done < cap) ids[(*n_done)++] = m.id;
  }
  return HJ_OK;
}

extern "C" hj_status hj_batch_take(hj_batch* bt, int64_t id, double* z_out, double* dE_out,
                                   hj_result* res) {
  if (!bt) return HJ_ERR_ARG;
  hj_ctx* ctx = bt->ctx;
  HJ_TRY(ctx_ok(ctx));
  const int k = batch_find(bt, id);
  if (k < 0) return set_err(ctx, HJ_ERR_ARG, "no bunch %lld in the batch", (long long)id);
  BatchMember m = bt->members[k];
  hj_bunch* b = m.b;
  // one round trip: pending kick and re-centring applied in place, moments
  // and turn state read, particles copied out, and the slot's state set to
  // "no turns left" for the kernels
  HJ_TRY(launch_moments(b, 1, b->z, b->dE));
  HJ_CUDA(ctx, cudaMemcpyAsync(b->h_mom, b->part_mom, sizeof(double) * 4 * b->nblk_m,
                               cudaMemcpyDeviceToHost, bt->stream));
  HJ_CUDA(ctx, cudaMemcpyAsync(b->h_ts, b->ts, sizeof(TurnState), cudaMemcpyDeviceToHost,
                               bt->stream));
  if (z_out)
    HJ_CUDA(ctx, cudaMemcpyAsync(z_out, b->z, sizeof(double) * b->n, cudaMemcpyDefault, bt->stream));
  if (dE_out)
    HJ_CUDA(ctx, cudaMemcpyAsync(dE_out, b->dE, sizeof(double) * b->n, cudaMemcpyDefault,
                                 bt->stream));
  TurnState dead{};
  dead.turns_left = 0;
  HJ_CUDA(ctx, cudaMemcpyAsync(b->ts, &dead, sizeof(TurnState), cudaMemcpyHostToDevice,
                               bt->stream));
  HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));
  double mom[4];
  sum_moments(b, mom);
  hj_status st = state_status(b);
  fill_result(b, mom, res);
  b->ts = nullptr;
  hj_bunch_destroy(b);
  batch_free_range(bt, m.start, m.cap);
  bt->free_slots.push_back(m.slot);
  bt->members[k] = bt->members.back();
  bt->members.pop_back();
  bt->dirty = true;
  return st;
}

extern "C" hj_status hj_batch_histogram(hj_batch* bt, int64_t id, int64_t* counts_host) {
  if (!bt || !counts_host) return HJ_ERR_ARG;
  hj_ctx* ctx = bt->ctx;
  HJ_TRY(ctx_ok(ctx));
  const int k = batch_find(bt, id);
  if (k < 0) return set_err(ctx, HJ_ERR_ARG, "no bunch %lld in the batch", (long long)id);
  const hj_bunch* b = bt->members[k].b;
  if (!b->use_wake) return set_err(ctx, HJ_ERR_STATE, "bunch has no wakefield histogram");
  HJ_CUDA(ctx, cudaMemcpyAsync(counts_host, b->hist, sizeof(int64_t) * b->B,
                               cudaMemcpyDeviceToHost, bt->stream));
  HJ_CUDA(ctx, cudaStreamSynchronize(bt->stream));
  return HJ_OK;
}

extern "C" hj_status hj_batch_stats(hj_batch* bt, int64_t* out4) {
  if (!bt || !out4) return HJ_ERR_ARG;
  out4[0] = (int64_t)bt->members.size();
  out4[1] = batch_largest_free(bt);
  out4[2] = (int64_t)bt->free_slots.size();
  out4[3] = bt->turns_enqueued;
  return HJ_OK;
}
