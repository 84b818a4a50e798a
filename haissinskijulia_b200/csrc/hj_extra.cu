// hj_extra.cu -- shards of a bunch over processes (the reference's MPI
// mode), the turn log, generate_particles on the device, and the
// correlation of the emittance figure of merit.
#include "hj_state.h"

// ====================================================================== shards
//
// A bunch split over processes (one GPU each), the reference's MPI mode
// (src/evolution.jl:206-212 with use_mpi): every rank tracks its particles;
// once per turn the ranks sum the merged histograms and the pass's sums
// (exchange buffers, B*3+2 u64 and kNumSums doubles) -- one all-reduce -- and
// every rank runs the bins step on the totals, so all ranks keep the same
// potential and E0.  The Philox draws of particle i of a shard are those of
// particle first_particle + i of the whole bunch.

extern "C" hj_status hj_bunch_create_shard(hj_ctx* ctx, double* d_z, double* d_dE,
                                           int64_t n_local, int64_t first_particle,
                                           int64_t n_global, const hj_params* params,
                                           const hj_wake* wake, const hj_grid* grid,
                                           uint64_t seed, void* stream, hj_bunch** out) {
  HJ_TRY(ctx_ok(ctx));
  if (!out) return set_err(ctx, HJ_ERR_ARG, "out is NULL");
  *out = nullptr;
  HJ_TRY(check_params(ctx, params));
  if (!params->use_wakefield || !grid)
    return set_err(ctx, HJ_ERR_ARG, "a shard needs the wakefield on and the shared bin grid");
  if (n_local <= 0 || first_particle < 0 || (first_particle & 1) ||
      first_particle + n_local > n_global)
    return set_err(ctx, HJ_ERR_ARG,
                   "shard [%lld, %lld) of %lld particles: non-empty, inside, even start",
                   (long long)first_particle, (long long)(first_particle + n_local),
                   (long long)n_global);
  if (!d_z || !d_dE || ((((uintptr_t)d_z) | ((uintptr_t)d_dE)) & 31))
    return set_err(ctx, HJ_ERR_ARG, "device particle arrays must be non-NULL and 32-byte aligned");
  hj_bunch* b = new hj_bunch();
  hj_status s = bunch_create_impl(ctx, d_z, d_dE, n_local, params, wake, grid->nbins, grid,
                                  seed, stream, b);
  if (s == HJ_OK) s = dalloc(ctx, &b->d_sums, kNumSums);
  if (s != HJ_OK) {
    hj_bunch_destroy(b);
    return s;
  }
  b->shard = true;
  b->n_global = n_global;
  b->first_particle = first_particle;
  *out = b;
  return HJ_OK;
}

extern "C" hj_status hj_bunch_local_moments(hj_bunch* b, double* out4) {
  if (!b || !out4) return HJ_ERR_ARG;
  HJ_TRY(ctx_ok(b->ctx));
  HJ_TRY(launch_moments(b, 1, nullptr, nullptr));
  return read_moments(b, out4);
}

extern "C" hj_status hj_bunch_set_global_moments(hj_bunch* b, const double* sums4) {
  if (!b || !sums4) return HJ_ERR_ARG;
  hj_ctx* ctx = b->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (b->turns_done != 0) return set_err(ctx, HJ_ERR_STATE, "global moments are set before the first turn");
  const int64_t n = b->shard ? b->n_global : b->n;
  b->sigma_z0_initial = global_std(sums4[0], sums4[1], n);
  b->sigma_E0_initial = global_std(sums4[2], sums4[3], n);
  HJ_TRY(read_state(b));
  b->h_ts->cur = make_turn_scalars(b->p.E0, b->p, b->sigma_E0_initial);
  HJ_CUDA(ctx, cudaMemcpyAsync(b->ts, b->h_ts, sizeof(TurnState), cudaMemcpyHostToDevice,
                               b->stream));
  HJ_CUDA(ctx, cudaStreamSynchronize(b->stream));
  return HJ_OK;
}

extern "C" hj_status hj_bunch_pass(hj_bunch* b) {
  if (!b) return HJ_ERR_ARG;
  hj_ctx* ctx = b->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (!b->shard) return set_err(ctx, HJ_ERR_STATE, "hj_bunch_pass is for shards (use hj_bunch_advance)");
  PassArgs a;
  BinsArgs g;
  fill_turn_args(b, a, g);
  HJ_CUDA(ctx, launch_track_pass(a, b->nblk, b->stream));
  HJ_CUDA(ctx, launch_hist_reduce(b->part_cnt, b->part_cic, b->nblk, b->B, b->hist, false,
                                  b->stream, b->hist_spill));
  HJ_CUDA(ctx, launch_sum_parts(b->part_sum, b->nblk, b->d_sums, b->stream));
  return HJ_OK;
}

extern "C" hj_status hj_bunch_exchange_buffers(hj_bunch* b, uint64_t** d_counts,
                                               int64_t* n_counts, double** d_sums,
                                               int64_t* n_sums) {
  if (!b || !d_counts || !n_counts || !d_sums || !n_sums) return HJ_ERR_ARG;
  if (!b->shard) return set_err(b->ctx, HJ_ERR_STATE, "not a shard");
  *d_counts = (uint64_t*)b->hist;
  *n_counts = 3 * (int64_t)b->B + 2;
  *d_sums = b->d_sums;
  *n_sums = kNumSums;
  return HJ_OK;
}

extern "C" hj_status hj_bunch_bins(hj_bunch* b) {
  if (!b) return HJ_ERR_ARG;
  hj_ctx* ctx = b->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (!b->shard) return set_err(ctx, HJ_ERR_STATE, "hj_bunch_bins is for shards (use hj_bunch_advance)");
  PassArgs a;
  BinsArgs g;
  fill_turn_args(b, a, g);
  HJ_CUDA(ctx, launch_bins(g, b->stream));
  b->turns_done += 1;
  return HJ_OK;
}

// ====================================================================== checkpoint / resume
//
// A host snapshot of (z, ΔE, E0, turn, initial spreads) is enough to continue
// a run: the Philox draws are keyed by (seed, particle, turn), the grid and
// the excitation amplitude by the initial spreads.

extern "C" hj_status hj_bunch_checkpoint(hj_bunch* b, double* d_z_out, double* d_dE_out,
                                         hj_checkpoint* out) {
  if (!b) return HJ_ERR_ARG;
  hj_ctx* ctx = b->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (!out || !d_z_out || !d_dE_out) return set_err(ctx, HJ_ERR_ARG, "output pointers are NULL");
  if (b->shard || b->batch_member)
    return set_err(ctx, HJ_ERR_STATE, "checkpoints are taken of whole resident bunches");
  HJ_TRY(launch_moments(b, 1, d_z_out, d_dE_out));
  double m[4];
  HJ_TRY(read_moments(b, m));
  HJ_TRY(read_state(b));
  out->turn = b->h_ts->turn;
  out->E0 = b->h_ts->cur.E0;
  out->sigma_E0_initial = b->sigma_E0_initial;
  out->sigma_z0_initial = b->sigma_z0_initial;
  return HJ_OK;
}

extern "C" hj_status hj_bunch_resume(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                                     const hj_params* params, const hj_wake* wake,
                                     int64_t nbins, const hj_grid* grid, uint64_t seed,
                                     const hj_checkpoint* cp, void* stream, hj_bunch** out) {
  HJ_TRY(ctx_ok(ctx));
  if (!out) return set_err(ctx, HJ_ERR_ARG, "out is NULL");
  *out = nullptr;
  if (!cp || cp->turn < 1) return set_err(ctx, HJ_ERR_ARG, "a checkpoint with turn >= 1 is needed");
  HJ_TRY(check_params(ctx, params));
  if (n <= 0 || !d_z || !d_dE) return set_err(ctx, HJ_ERR_ARG, "particle arrays are empty or NULL");
  if ((((uintptr_t)d_z) | ((uintptr_t)d_dE)) & 31)
    return set_err(ctx, HJ_ERR_ARG, "device particle arrays must be 32-byte aligned");
  hj_bunch* b = new hj_bunch();
  hj_status s = bunch_create_begin(ctx, d_z, d_dE, n, params, wake, nbins, grid, seed, stream, b);
  if (s == HJ_OK) {
    cudaError_t e = cudaStreamSynchronize(b->stream);
    s = e == cudaSuccess ? bunch_create_end(ctx, b, grid, cp)
                         : set_err(ctx, HJ_ERR_CUDA, "%s", cudaGetErrorString(e));
  }
  if (s != HJ_OK) {
    hj_bunch_destroy(b);
    return s;
  }
  *out = b;
  return HJ_OK;
}

// ====================================================================== turn log

extern "C" hj_status hj_bunch_set_log(hj_bunch* b, int64_t every, int64_t capacity,
                                      int32_t density) {
  if (!b) return HJ_ERR_ARG;
  hj_ctx* ctx = b->ctx;
  HJ_TRY(ctx_ok(ctx));
  if (every < 0 || (every > 0 && capacity <= 0))
    return set_err(ctx, HJ_ERR_ARG, "log every >= 0 turns into capacity > 0 records");
  if (density && !b->use_wake) return set_err(ctx, HJ_ERR_STATE, "no line density without the wakefield");
  HJ_CUDA(ctx, cudaStreamSynchronize(b->stream));
  if (b->d_log) cudaFree(b->d_log);
  b->d_log = nullptr;
  b->log_every = every;
  b->log_capacity = capacity;
  b->log_density = density ? 1 : 0;
  b->log_count = 0;
  if (every > 0)
    HJ_TRY(dalloc(ctx, &b->d_log, (size_t)capacity * (kLogHeader + (b->log_density ? b->B : 0))));
  return HJ_OK;
}

extern "C" hj_status hj_bunch_read_log(hj_bunch* b, double* out, int64_t max_records,
                                       int64_t* n_records) {
  if (!b || !n_records || (max_records > 0 && !out)) return HJ_ERR_ARG;
  hj_ctx* ctx = b->ctx;
  HJ_TRY(ctx_ok(ctx));
  *n_records = 0;
  if (!b->d_log) return HJ_OK;
  const int64_t rec = kLogHeader + (b->log_density ? b->B : 0);
  const int64_t held = std::min(b->log_count, b->log_capacity);
  const int64_t n = std::min(held, max_records);
  // the n most recent records, oldest first
  for (int64_t k = 0; k < n; ++k) {
    const int64_t idx = (b->log_count - n + k) % b->log_capacity;
    HJ_CUDA(ctx, cudaMemcpyAsync(out + k * rec, b->d_log + idx * rec, sizeof(double) * rec,
                                 cudaMemcpyDeviceToHost, b->stream));
  }
  HJ_CUDA(ctx, cudaStreamSynchronize(b->stream));
  *n_records = n;
  return HJ_OK;
}

// ====================================================================== generate_particles

namespace {
// compute_std (src/utils.jl:531-544) of a device array: two passes, per-block
// sums added on the host in block order.
hj_status device_compute_std(hj_ctx* ctx, const double* x, int64_t n, double* part, int grid,
                             cudaStream_t st, double* out) {
  std::vector<double> h(grid);
  HJ_CUDA(ctx, launch_std_parts(x, n, 0.0, 0, part, grid, st));
  HJ_CUDA(ctx, cudaMemcpyAsync(h.data(), part, sizeof(double) * grid, cudaMemcpyDeviceToHost, st));
  HJ_CUDA(ctx, cudaStreamSynchronize(st));
  double s = 0.0;
  for (double v : h) s += v;
  const double mu = s / (double)n;
  HJ_CUDA(ctx, launch_std_parts(x, n, mu, 1, part, grid, st));
  HJ_CUDA(ctx, cudaMemcpyAsync(h.data(), part, sizeof(double) * grid, cudaMemcpyDeviceToHost, st));
  HJ_CUDA(ctx, cudaStreamSynchronize(st));
  double s2 = 0.0;
  for (double v : h) s2 += v;
  const double var = s2 / (double)(n - 1);
  *out = std::sqrt(std::max(0.0, var));
  return HJ_OK;
}
}  // namespace

extern "C" hj_status hj_generate_particles(hj_ctx* ctx, double mu_z, double mu_E, double sigma_z,
                                           double sigma_E, int64_t n, uint64_t seed,
                                           double* d_z, double* d_dE, void* stream,
                                           double* actual_sigma_E, double* actual_sigma_z) {
  HJ_TRY(ctx_ok(ctx));
  if (!actual_sigma_E || !actual_sigma_z) return set_err(ctx, HJ_ERR_ARG, "output spreads are NULL");
  if (!(sigma_z >= 0.0 && sigma_E >= 0.0)) return set_err(ctx, HJ_ERR_ARG, "spreads must be non-negative");
  cudaStream_t st = (cudaStream_t)stream;
  if (n <= 0) {                                   // src/evolution.jl:47-53
    *actual_sigma_E = 0.0;
    *actual_sigma_z = 0.0;
    return HJ_OK;
  }
  if (!d_z || !d_dE) return set_err(ctx, HJ_ERR_ARG, "particle arrays are NULL");
  *actual_sigma_E = sigma_E;
  *actual_sigma_z = sigma_z;
  if (n < 2) {                                    // :62-67, independent draws, input spreads
    HJ_CUDA(ctx, launch_gaussian_bunch(seed, n, mu_z, sigma_z, mu_E, sigma_E, d_z, d_dE, st));
    HJ_CUDA(ctx, cudaStreamSynchronize(st));
    return HJ_OK;
  }
  const int grid = (int)std::min<int64_t>((n + 1023) / 1024, 4 * (int64_t)ctx->num_sms);
  double* dev = nullptr;
  HJ_TRY(dalloc(ctx, &dev, (size_t)grid + 3));
  hj_status s = HJ_OK;
  do {
    // covariance of a sample of min(n, 10000) independent draws (:69-81)
    const int64_t S = std::min<int64_t>(n, 10000);
    double c[3];
    cudaError_t e = launch_gen_sample_cov(seed, S, mu_z, sigma_z, mu_E, sigma_E, dev + grid, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(c, dev + grid, sizeof(c), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
      s = set_err(ctx, HJ_ERR_CUDA, "covariance sample failed: %s", cudaGetErrorString(e));
      break;
    }
    double a = std::max(1e-18, c[0]), b = c[2], d = std::max(1e-18, c[1]);
    // positive semi-definite guard (:88-93): eigmin of [[a, b], [b, d]]
    const double min_eig = 0.5 * (a + d) - std::sqrt(0.25 * (a - d) * (a - d) + b * b);
    if (min_eig < 1e-12) {
      const double add = std::max(0.0, 1e-12 - min_eig);
      a += add;
      d += add;
    }
    // MvNormal draw (:95-116): mu + L eps, L the lower Cholesky factor of the covariance
    const double l00 = std::sqrt(a), l10 = b / l00, l11 = std::sqrt(std::max(0.0, d - l10 * l10));
    e = launch_gen_correlated(seed, n, mu_z, mu_E, l00, l10, l11, d_z, d_dE, st);
    if (e != cudaSuccess) {
      s = set_err(ctx, HJ_ERR_CUDA, "bunch draw failed: %s", cudaGetErrorString(e));
      break;
    }
    // actual spreads, compute_std (:119-121)
    s = device_compute_std(ctx, d_z, n, dev, grid, st, actual_sigma_z);
    if (s == HJ_OK) s = device_compute_std(ctx, d_dE, n, dev, grid, st, actual_sigma_E);
  } while (false);
  cudaFree(dev);
  return s;
}

// ====================================================================== correlation

// cor(particles.coordinates.z, particles.coordinates.ΔE) of EmittanceFoM
// (src/parameter_sensitivity/figures_of_merit.jl:42, Julia's Statistics.cor):
// two passes over the device arrays (means, then centred sums Sxx, Syy, Sxy),
// per-block sums added on the host in block order, r = Sxy/(√Sxx √Syy)
// clamped to [-1, 1].
extern "C" hj_status hj_correlation(hj_ctx* ctx, const double* d_x, const double* d_y, int64_t n,
                                    void* stream, double* out) {
  HJ_TRY(ctx_ok(ctx));
  if (!out) return set_err(ctx, HJ_ERR_ARG, "out is NULL");
  if (n <= 0) return set_err(ctx, HJ_ERR_ARG, "correlation only defined for non-empty vectors");
  if (!d_x || !d_y) return set_err(ctx, HJ_ERR_ARG, "arrays are NULL");
  cudaStream_t st = (cudaStream_t)stream;
  const int grid = (int)std::min<int64_t>((n + 4095) / 4096, 4 * (int64_t)ctx->num_sms);
  void* base = nullptr;
  HJ_TRY(scratch(ctx, sizeof(double) * 3 * (size_t)grid, &base));
  double* part = (double*)base;
  std::vector<double> h(3 * (size_t)grid);
  double s[2][3] = {};
  double mx = 0.0, my = 0.0;
  for (int pass = 0; pass < 2; ++pass) {
    HJ_CUDA(ctx, launch_cor_parts(d_x, d_y, n, mx, my, pass, part, grid, st));
    HJ_CUDA(ctx, cudaMemcpyAsync(h.data(), part, sizeof(double) * h.size(),
                                 cudaMemcpyDeviceToHost, st));
    HJ_CUDA(ctx, cudaStreamSynchronize(st));
    for (int b = 0; b < grid; ++b)
      for (int k = 0; k < 3; ++k) s[pass][k] += h[3 * (size_t)b + k];
    mx = s[0][0] / (double)n;
    my = s[0][1] / (double)n;
  }
  const double r = s[1][2] / (std::sqrt(s[1][0]) * std::sqrt(s[1][1]));
  *out = r != r ? r : std::min(1.0, std::max(-1.0, r));
  return HJ_OK;
}
