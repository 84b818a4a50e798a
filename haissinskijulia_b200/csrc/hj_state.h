// hj_state.h -- state and helpers shared by the C-ABI sources (hj_api.cu:
// context, bunches, whole runs and single steps; hj_batch.cu: batches;
// hj_extra.cu: shards, turn log, generate_particles, correlation).  Not part
// of the public ABI.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <unordered_set>
#include <vector>

#include "hj_host.h"
#include "hj_internal.h"

using namespace hj;

struct hj_ctx {
  int device = 0;
  int num_sms = 148;
  int max_smem_optin = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  int pass_layout = -1;   // -1: chosen per bunch
  // released blocks kept for reuse, by size class (device / pinned host)
  std::multimap<size_t, void*> dev_free, host_free;
  size_t dev_free_bytes = 0, host_free_bytes = 0;
  // device blocks up to kSlabBlockMax are carved from large slabs (a
  // cudaMalloc of a megabyte costs ~0.6 ms); carved blocks are reused through
  // dev_free and released with their slabs by hj_destroy
  std::vector<void*> dev_slabs;
  char* slab_cur = nullptr;
  size_t slab_left = 0;
  std::unordered_set<void*> carved;
  // twiddle tables of the bins step by FFT length P, shared by all bunches
  std::map<int, double2*> twiddles;
  // grids and wake tables built from an initial σ_z, by the bit patterns of
  // (nbins, σ_z0, half width, F, s, cτ, sin coefficient, δ width): bunches
  // of a scan start from the same particles and share them
  struct WakeSet {
    std::vector<double> centers;
    double e0 = 0, eN = 0, estep = 0;
    void* dev = nullptr;            // W[B] | λ[B] | FFT(W)[M+1], a block of the cache
    size_t cap = 0;
    uint64_t used = 0;
    int refs = 0;                   // bunches reading the tables (read-only)
  };
  std::map<std::array<uint64_t, 8>, WakeSet> wake_sets;
  uint64_t wake_clock = 0;
  // Bunches and batches alive on this context.  hj_destroy with some alive
  // only marks the context closing; the last of them to be destroyed frees it,
  // so objects may be destroyed in any order (e.g. by a garbage collector).
  int64_t live_objects = 0;
  bool closing = false;
};

struct hj_bunch {
  hj_ctx* ctx = nullptr;
  bool holds_ctx = false;   // counted in ctx->live_objects
  cudaStream_t stream = nullptr;
  double* z = nullptr;
  double* dE = nullptr;
  int64_t n = 0;
  hj_params p{};
  hj_wake w{};
  int use_wake = 0;
  int B = 0, P = 0, M = 0, H = 0, logH = 0;
  double e0 = 0, eN = 0, estep = 0, inv_e = 0, c1 = 0, cB = 0, inv_c = 0;
  // interpolation the reference applies to every z >= cB (src/wakefield.jl:80-102):
  // u = (cB - c1)/Δc, cell clamp(floor(u), 0, B-2), weight u - floor(u)
  int hi_idx = 0;
  double hi_w = 0;
  std::vector<double> centers;
  double sigma_E0_initial = 0, sigma_z0_initial = 0;
  uint64_t seed = 0;
  int qe_mode = QE_OFF;
  const double* draws = nullptr;
  int64_t draws_first = 0, draws_turns = 0;
  int nblk = 1, nblk_m = 1;
  // a shard of a bunch split over processes: its particles are
  // [first_particle, first_particle + n) of n_global; the bins step reads the
  // exchanged totals (d_sums, hist) instead of this shard's partials
  bool shard = false;
  int64_t n_global = 0, first_particle = 0;
  double* d_sums = nullptr;
  // turn log: a record every log_every turns into a ring of log_capacity
  int64_t log_every = 0, log_capacity = 0, log_count = 0;
  int log_density = 0;
  double* d_log = nullptr;
  int64_t turns_done = 0;
  // device buffers
  TurnState* ts = nullptr;
  double* pot = nullptr;
  double2* potd = nullptr;              // [B+1] kick table (cell j: pot[j-1], step)
  int cfg = 0;                          // thread layout of the fused pass
  unsigned long long* hist = nullptr;   // counts[B] | cell counts[B+1] | cell Σw·2^24 [B+1]
  double* lam = nullptr;
  double* W = nullptr;
  double2* Wf = nullptr;
  double2* twP = nullptr;
  uint32_t* part_cnt = nullptr;
  int64_t* defer_q = nullptr;             // [nblk][warps][kDeferStage] (Float64 normals)
  unsigned long long* part_cic = nullptr;
  unsigned long long* hist_spill = nullptr;   // [3B+2] the pass's deposits outside its hot
                                              // window and beyond its 16-bit counters
  double2* rf_table = nullptr;             // [kRfTableSize] RF kick table of the pass
  double rf_Vs = 0;                        // its entry 0: V sin ϕs
  double* part_sum = nullptr;
  double* part_mom = nullptr;
  double* h_mom = nullptr;    // pinned
  TurnState* h_ts = nullptr;  // pinned
  double* h_rf = nullptr;     // pinned staging of the RF table
  // the buffers above are carved from one device block and one pinned block
  // of the context's cache; twP is the context's shared table; W, lam and Wf
  // point into a wake set shared with other bunches (wset) or a private block
  // (tables); pot, potd, hist and hist_spill are the first zero_bytes of the
  // arena's histogram part
  hj_ctx::WakeSet* wset = nullptr;
  bool batch_member = false;
  void* tables = nullptr;
  size_t tables_cap = 0;
  size_t zero_bytes = 0;
  void* arena = nullptr;
  size_t arena_cap = 0;
  void* harena = nullptr;
  size_t harena_cap = 0;
  // profiling: three events per profiled turn (before pass, after pass, after bins)
  bool profiling = false;
  std::vector<cudaEvent_t> events;
  size_t events_used = 0;
  int64_t profiled_turns = 0;
  int64_t profiled_launches = 0;
};

#define HJ_CUDA(ctx, call)                                                            \
  do {                                                                                \
    cudaError_t e_ = (call);                                                          \
    if (e_ != cudaSuccess)                                                            \
      return set_err((ctx), e_ == cudaErrorMemoryAllocation ? HJ_ERR_NOMEM : HJ_ERR_CUDA, \
                     "%s failed: %s", #call, cudaGetErrorString(e_));                 \
  } while (0)

#define HJ_TRY(expr)             \
  do {                           \
    hj_status s_ = (expr);       \
    if (s_ != HJ_OK) return s_;  \
  } while (0)

namespace hj_impl {

inline size_t align_up(size_t v) { return (v + 255) & ~size_t(255); }

// Offsets of the buffers carved from one block (each 256-byte aligned).
struct Carve {
  size_t off = 0;
  template <class T>
  size_t add(size_t count) {
    const size_t o = off;
    off = align_up(off + sizeof(T) * (count ? count : 1));
    return o;
  }
};

hj_status set_err(hj_ctx* ctx, hj_status code, const char* fmt, ...);
hj_status ctx_ok(hj_ctx* ctx);
// Count an object in ctx->live_objects / drop it (the last drop of a closing
// context frees the context).
void ctx_retain(hj_ctx* ctx);
void ctx_release(hj_ctx* ctx);

template <typename T>
hj_status dalloc(hj_ctx* ctx, T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    *p = nullptr;
    return set_err(ctx, HJ_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", count * sizeof(T),
                   cudaGetErrorString(e));
  }
  return HJ_OK;
}

int64_t next_pow2(int64_t n);
int ilog2(int64_t v);
// compute_global_std from global sums (src/utils.jl:593-605), on the host
double global_std(double s, double s2, int64_t n);
// The context's reusable scratch block (grows; one user at a time).
hj_status scratch(hj_ctx* ctx, size_t bytes, void** out);

// Block cache (see hj_api.cu): blocks by size class, small device blocks
// carved from slabs.
size_t size_class(size_t b);
hj_status cache_take(hj_ctx* ctx, bool host, size_t bytes, void** out, size_t* cap);
void cache_give(hj_ctx* ctx, bool host, void* p, size_t cap);
void cache_clear(hj_ctx* ctx, bool slabs = false);
hj_status shared_twiddles(hj_ctx* ctx, int P, double2** out);

hj_status check_params(hj_ctx* ctx, const hj_params* p);
hj_status check_grid(hj_ctx* ctx, const hj_grid* g);

// Moments of a bunch: per-block sums on the device, summed on the host in
// block order.
void sum_moments(const hj_bunch* b, double m[4]);
hj_status read_moments(hj_bunch* b, double m[4]);
hj_status launch_moments(hj_bunch* b, int apply, double* z_out, double* dE_out);
hj_status state_status(hj_bunch* b);
hj_status read_state(hj_bunch* b);
int default_pass_layout(int B, int64_t n);
int auto_pass_layout(int r, int B, int64_t n);
void fill_result(hj_bunch* b, const double m[4], hj_result* res);
cudaError_t set_kernel_attributes(hj_ctx* ctx);

// Creation of a bunch in two halves around one synchronisation of its stream
// (hj_api.cu); chunk > 0: a batch member with chunks of `chunk` particles;
// cfg >= 0 pins the pass layout.
hj_status bunch_create_begin(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                             const hj_params* params, const hj_wake* wake, int64_t nbins,
                             const hj_grid* grid, uint64_t seed, void* stream, hj_bunch* b,
                             int64_t chunk = 0, int cfg = -1);
// cp: continue from a checkpoint (its turn, E0 and initial spreads)
hj_status bunch_create_end(hj_ctx* ctx, hj_bunch* b, const hj_grid* grid,
                           const hj_checkpoint* cp = nullptr);
hj_status bunch_create_impl(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                            const hj_params* params, const hj_wake* wake, int64_t nbins,
                            const hj_grid* grid, uint64_t seed, void* stream, hj_bunch* b,
                            int64_t chunk = 0, int cfg = -1);
// Arguments of the fused pass and of the bins step of bunch b.
void fill_turn_args(const hj_bunch* b, PassArgs& a, BinsArgs& g);

}  // namespace hj_impl

using namespace hj_impl;
