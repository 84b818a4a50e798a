/*
 * haissinski_gpu.h -- C ABI of the B200 (sm_100a) longitudinal tracking library.
 *
 * The reference (HaissinskiJulia, module StochasticHaissinski) exposes its
 * per-turn tracking loop as Julia methods; it has no FFI of its own.  This
 * header is the drop-in boundary a Julia `ccall` (or Python ctypes) binds:
 * plain pointers, sizes and POD structs, no CUDA or torch types.
 *
 * Every entry point below names the reference interface it replaces.
 * Conventions shared by all calls:
 *   - particle state is structure-of-arrays Float64: z[n] in metres and dE[n]
 *     in eV, exactly `particles.coordinates.z` / `particles.coordinates.ΔE`
 *     of the reference's StructArray{Particle{Float64}}
 *     (src/data_structures.jl:26-42);
 *   - functions without `_device` in their name take HOST pointers, copy to
 *     the GPU, run, and copy results back (in-place semantics like the
 *     reference's mutating `!` methods);
 *   - every call returns an hj_status; HJ_OK is 0.  The message of the last
 *     failure on a context is available from hj_last_error().
 *   - a context is bound to one device and is not re-entrant: use one
 *     context per host thread.  Several contexts may share a GPU.
 */
#ifndef HAISSINSKI_GPU_H
#define HAISSINSKI_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t hj_status;

enum {
  HJ_OK = 0,
  HJ_ERR_ARG = 1,          /* invalid argument (null pointer, negative size, ...) */
  HJ_ERR_NBINS = 2,        /* nbins <= 0: src/evolution.jl:264, src/utils.jl:155-157 */
  HJ_ERR_WAKE_PARAM = 3,   /* ctau <= 0 or pipe_radius <= 0: src/evolution.jl:277-278 */
  HJ_ERR_CUDA = 4,         /* a CUDA runtime call failed (message has the CUDA error) */
  HJ_ERR_NOMEM = 5,        /* device allocation failed */
  HJ_ERR_TOO_LARGE = 6,    /* a size exceeds what the library supports */
  HJ_ERR_EMPTY = 7,        /* zero particles with the wakefield on: the reference's
                              log10(0) particle-factor path raises (src/evolution.jl:377-379) */
  HJ_ERR_NONFINITE = 8,    /* a NaN/Inf appeared in the bunch moments */
  HJ_ERR_TIMEOUT = 9,      /* a bounded device-side wait gave up */
  HJ_ERR_NO_DEVICE = 10,   /* no CUDA device, or device index out of range */
  HJ_ERR_STATE = 11,       /* call out of order (e.g. advance after finish) */
  HJ_ERR_FULL = 12         /* a batch has no room for the bunch now (slots, particle
                              pool or bins): retire finished bunches and retry */
};

/*
 * Simulation parameters: field for field the reference's
 * SimulationParameters (src/data_structures.jl:81-97), Float64 instantiation.
 */
typedef struct hj_params {
  double E0;            /* reference energy [eV] */
  double mass;          /* particle mass [eV/c^2] */
  double voltage;       /* RF voltage [V] */
  int64_t harmonic;     /* RF harmonic number */
  double radius;        /* bending radius used by SR damping / quantum excitation [m] */
  double pipe_radius;   /* beam pipe radius [m] (enters the reference wake constants) */
  double alpha_c;       /* momentum compaction */
  double phi_s;         /* synchronous phase [rad] */
  double freq_rf;       /* RF frequency [Hz] */
  int64_t n_turns;      /* turns to track */
  uint8_t use_wakefield;
  uint8_t update_eta;
  uint8_t update_E0;
  uint8_t SR_damping;
  uint8_t use_excitation;
  uint8_t _pad[3];
} hj_params;

/*
 * Wake model and intensity.  The reference hard-codes these inside
 * longitudinal_evolve! (src/evolution.jl:270-280 and :377-386);
 * hj_wake_reference() fills exactly those values.  The extra fields let a
 * caller describe a broadband resonator and a bunch population.
 *
 *   W(c) = 0                                          for c > 0
 *   W(c) = F * exp(c/ctau) * (cos(s c) + sin_coef * sin(s c))   for c <= 0
 * (src/wakefield.jl:115-118 with sin_coef = 0).
 */
typedef struct hj_wake {
  double wake_factor;        /* F */
  double wake_sqrt;          /* s [1/m] */
  double ctau;               /* c*tau [m] */
  double sin_coef;           /* 0 in reference mode */
  double population;         /* > 0: replaces the reference's particle_factor; 0: reference formula */
  double half_width_sigmas;  /* bins span +-half_width_sigmas * sigma_z0_initial; reference 7.5 */
  double delta_std;          /* width of the pointwise Gaussian weight delta(); reference 0.15 */
} hj_wake;

/*
 * Uniform bin grid.  In the reference, edges = range(-w, w, length=nbins+1)
 * and centers = (edges[1:end-1] + edges[2:end]) ./ 2 (src/evolution.jl:270-274).
 * The histogram uses edge_first, edge_last and step(edges)
 * (src/utils.jl:367-380); the wake table and the interpolation use the
 * centers (src/wakefield.jl:39-42, :194-196).  A Julia caller passes the
 * values of its own ranges so that bins agree bit for bit.
 */
typedef struct hj_grid {
  int64_t nbins;
  double edge_first;
  double edge_last;
  double edge_step;
  const double* centers;     /* nbins values, host memory */
} hj_grid;

/* Return tuple of longitudinal_evolve! (src/evolution.jl:470) plus diagnostics. */
typedef struct hj_result {
  double sigma_E;            /* final sample std of dE */
  double sigma_z;            /* final sample std of z */
  double E0;                 /* final reference energy */
  double sigma_E0_initial;   /* src/evolution.jl:248 */
  double sigma_z0_initial;   /* src/evolution.jl:249 */
  double mean_z;             /* final centroid of z */
  double mean_dE;            /* final centroid of dE */
  int64_t turns;             /* turns tracked so far */
} hj_result;

typedef struct hj_ctx hj_ctx;
typedef struct hj_bunch hj_bunch;
typedef struct hj_batch hj_batch;

/* ---------------------------------------------------------------- context */

/* Library version string. */
const char* hj_version(void);
/* Human-readable name of a status code. */
const char* hj_status_string(hj_status s);
/* Create a context on CUDA device `device`.  No reference counterpart (the
 * reference allocates per call in create_simulation_buffers, src/utils.jl:147). */
hj_status hj_create(int32_t device, hj_ctx** out);
/* Free the context.  After this call the handle must not be passed to any
 * entry point.  Bunches and batches keep their context alive: with some still
 * alive, hj_destroy only marks the context closing, they keep working (a
 * batch still admits bunches), and the last of them to be destroyed frees it,
 * so objects may be destroyed in any order, as a garbage collector does. */
void hj_destroy(hj_ctx* ctx);
/* Message of the last failure on this context ("" if none). */
const char* hj_last_error(const hj_ctx* ctx);
/* A context keeps, for reuse, the device and pinned blocks of finished
 * bunches and of hj_evolve's particle arrays (up to 8 GB device, 256 MB
 * pinned) and the last 8 bin grids with their wake tables built from an
 * initial sigma_z (bunches of a scan start from the same particles), so that
 * admitting bunches of recurring sizes allocates and recomputes nothing.
 * Blocks up to 16 MB are carved from 256 MB slabs, which the context keeps
 * until hj_destroy.  hj_trim frees the other kept blocks now (hj_destroy
 * frees everything).  No reference counterpart. */
hj_status hj_trim(hj_ctx* ctx);
/* Thread layout of the fused particle pass for bunches created afterwards on
 * this context: -1 = chosen by the library (default), 0 = 4 particles per
 * thread x 512 threads, 1 = 2 x 1024, 2 = 2 x 768 (each with the next group
 * prefetched), 3 = 2 x 512 without prefetch, 4 = 2 x 512 with prefetch at
 * two blocks per SM, 5 = 4 x 256 with prefetch at two blocks per SM; plus 8
 * (8..13): the same layout with one 32-bit shared-memory counter per bin
 * instead of two 16-bit ones per word (no overflow check; the default).  The
 * pass keeps its per-block bin counters, cell words and kick-table entries in
 * shared memory for the cells around the bunch's last mean position, as many
 * as fit (all of them up to 8192 bins), and deposits the rest with global
 * integer atomics.  Plus 16 (16..29, or 23 for the library's choice): the
 * quantum-excitation normals of the fused pass are formed in single precision
 * (a Box-Muller transform of Philox words 0-1, 24-bit uniforms, tails cut at
 * 6σ, about 12 % faster per pass at 16384 bins) instead of the default
 * Float64 ziggurat; hj_gaussian and the single-step kernels stay in double
 * precision.  Results do not depend on the layout beyond floating-point
 * summation order (and the normals' precision); bin counts are the same.  No
 * reference counterpart. */
hj_status hj_set_pass_layout(hj_ctx* ctx, int32_t layout);

/* ---------------------------------------------------------------- set-up helpers */

/* Fill the reference's hard-coded wake: kp = 30, Z0 = 120*pi, ctau = 4e-3,
 * F = Z0*c/(pi*pipe_radius), s = sqrt(2 kp / pipe_radius)
 * (src/evolution.jl:276-280), particle_factor intensity, +-7.5 sigma bins,
 * delta_std = 0.15 (src/wakefield.jl:204). */
hj_status hj_wake_reference(const hj_params* p, hj_wake* out);

/* Broadband resonator (shunt impedance Rs [Ohm], quality factor Q, resonant
 * frequency fr [Hz]) expressed in the reference's wake form:
 * ctau = c/alpha, s = omega_bar/c, F = 2 alpha Rs, sin_coef = +alpha/omega_bar
 * (the -(alpha/omega_bar) sin(omega_bar tau) term of the resonator wake with
 * c = -c tau), alpha = omega_r/(2Q), omega_bar = sqrt(omega_r^2 - alpha^2).  No reference counterpart (the reference has only
 * the hard-coded form above). */
hj_status hj_wake_resonator(double Rs, double Q, double fr, double population,
                            double half_width_sigmas, hj_wake* out);

/* Build the uniform grid for nbins bins over +-half_width_sigmas*sigma_z0
 * (width floor 1e-6 m when 7.5 sigma < 1e-9, src/evolution.jl:270-272).
 * Each edge and center is the correctly rounded value of its exact rational
 * position.  `centers` (nbins doubles) is caller storage and is referenced by
 * the returned grid. */
hj_status hj_make_grid(double sigma_z0, double half_width_sigmas, int64_t nbins,
                       double* centers, hj_grid* out);

/* ---------------------------------------------------------------- whole loop */

/*
 * Drop-in for
 *   longitudinal_evolve!(particles, params, buffers, comm, use_mpi) -> (σ_E, σ_z, E0)
 * (src/evolution.jl:206-212, returns at :470), MPI-branch semantics at any
 * rank count (the only branch that runs with the wakefield on).
 *   z, dE      host arrays of n Float64, updated in place;
 *   wake       NULL -> hj_wake_reference(params);
 *   nbins      bin count (length(buffers.λ) in the reference);
 *   grid       NULL -> grid built on the device's sigma_z0_initial with
 *              hj_make_grid; non-NULL -> used as given (nbins must match);
 *   qe_draws   NULL -> on-device Philox-4x32-10 / ziggurat Gaussians keyed by
 *              (seed, particle, turn); non-NULL -> host array of
 *              n_turns*n standard normals, turn-major, used in place of
 *              randn! (src/quantum_excitation.jl:36);
 *   out        receives (sigma_E, sigma_z, E0) and diagnostics.
 */
hj_status hj_evolve(hj_ctx* ctx, double* z, double* dE, int64_t n,
                    const hj_params* params, const hj_wake* wake, int64_t nbins,
                    const hj_grid* grid, const double* qe_draws, uint64_t seed,
                    hj_result* out);

/* Same as hj_evolve on DEVICE arrays, enqueued on `stream` (a cudaStream_t,
 * NULL = legacy default stream); returns after the final moments are read. */
hj_status hj_evolve_device(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                           const hj_params* params, const hj_wake* wake, int64_t nbins,
                           const hj_grid* grid, const double* d_qe_draws, uint64_t seed,
                           void* stream, hj_result* out);

/* ---------------------------------------------------------------- resident bunch */

/*
 * A bunch whose state stays on the device between calls (the reference
 * keeps the state in the caller's StructArray across the turn loop,
 * src/evolution.jl:295-456).  create() computes the initial spreads
 * (src/evolution.jl:245-253) and the wake set-up (:261-281); advance()
 * enqueues turns without host synchronisation; observe() writes the
 * turn-boundary state to caller DEVICE buffers without disturbing the
 * bunch; finish() completes the last turn and returns the final tuple.
 * d_z/d_dE are caller-owned device arrays that must outlive the bunch.
 */
hj_status hj_bunch_create(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                          const hj_params* params, const hj_wake* wake, int64_t nbins,
                          const hj_grid* grid, uint64_t seed, void* stream,
                          hj_bunch** out);
/* Host-fed draws for the following turns: device array of turns*n normals,
 * turn-major; turn t of the bunch reads row (t - first_turn).  NULL switches
 * back to on-device Philox. */
hj_status hj_bunch_set_draws(hj_bunch* b, const double* d_draws, int64_t first_turn,
                             int64_t turns);
/* Enqueue `turns` more turns on the bunch's stream. */
hj_status hj_bunch_advance(hj_bunch* b, int64_t turns);
/* Turn-boundary state (all pending kicks applied) into d_z_out/d_dE_out
 * (device, n each; either may be NULL), plus moments and E0 in *res. */
hj_status hj_bunch_observe(hj_bunch* b, double* d_z_out, double* d_dE_out, hj_result* res);
/* Apply the pending wake kick and E0 re-centring of the last turn in place
 * and return the final tuple (src/evolution.jl:458-470). */
hj_status hj_bunch_finish(hj_bunch* b, hj_result* res);
/* Device-time profiling of the turns enqueued while enabled: CUDA events are
 * recorded on the bunch's stream around each particle pass and each bins
 * step (histogram reduction + convolution + E0 update).  enable = 0 stops
 * and clears.  No reference counterpart (the reference times whole calls
 * with BenchmarkTools, tests/benchmark_total.jl:343-369). */
hj_status hj_bunch_set_profiling(hj_bunch* b, int32_t enable);
/* out[0] = particle-pass milliseconds, out[1] = bins-step milliseconds,
 * out[2] = turns profiled, out[3] = kernel launches profiled.
 * Synchronises the bunch's stream. */
hj_status hj_bunch_read_profile(hj_bunch* b, double* out4);
/* Turn log: every `every` turns of hj_bunch_advance, one record of the state
 * after that turn -- [turn, E0, σ_z, σ_E, mean z, mean ΔE, wake current,
 * particles in the bins], then the nbins line-density counts when density != 0
 * -- written on the device into a ring of `capacity` records (no host round
 * trip; costs one moments pass over the particles per record).  every = 0
 * stops.  The reference keeps per-turn observables in BeamTurn
 * (src/data_structures.jl:52-54, src/utils.jl:42-50). */
hj_status hj_bunch_set_log(hj_bunch* b, int64_t every, int64_t capacity, int32_t density);
/* Copies the most recent min(held, max_records) records, oldest first, into
 * out (8 [+ nbins] doubles each); *n_records = how many. */
hj_status hj_bunch_read_log(hj_bunch* b, double* out, int64_t max_records, int64_t* n_records);
/* Checkpoint of a resident bunch at a turn boundary: what, with its
 * particles, lets another bunch (another process, a later job) continue the
 * run -- the next turn's number, E0, and the initial spreads that fix the
 * quantum-excitation amplitude and the bin grid; with the same seed the
 * Philox draws continue unchanged, since they are keyed by (seed, particle,
 * turn).  No reference counterpart (the reference keeps no checkpoint). */
typedef struct hj_checkpoint {
  int64_t turn;              /* number of the next turn (turns done + 1) */
  double E0;
  double sigma_E0_initial;
  double sigma_z0_initial;
} hj_checkpoint;
/* The particles at the turn boundary (the pending kick and re-centring
 * applied, as hj_bunch_observe gives them) into device arrays d_z_out,
 * d_dE_out, and the checkpoint.  The bunch itself runs on unchanged. */
hj_status hj_bunch_checkpoint(hj_bunch* b, double* d_z_out, double* d_dE_out, hj_checkpoint* out);
/* A resident bunch continuing from a checkpoint: as hj_bunch_create, with
 * d_z, d_dE the checkpointed particles and the turn counter, E0 and initial
 * spreads (hence the grid, when grid is NULL) taken from *cp. */
hj_status hj_bunch_resume(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n,
                          const hj_params* params, const hj_wake* wake, int64_t nbins,
                          const hj_grid* grid, uint64_t seed, const hj_checkpoint* cp,
                          void* stream, hj_bunch** out);
/* Line density of the last completed turn: integer bin counts (nbins). */
hj_status hj_bunch_histogram(hj_bunch* b, int64_t* counts_host);
/* Potential at the bin centers from the last completed turn (nbins). */
hj_status hj_bunch_potential(hj_bunch* b, double* pot_host);
void hj_bunch_destroy(hj_bunch* b);

/* ---------------------------------------------------------------- shards
 * One bunch split over processes, one GPU each -- the reference's MPI mode
 * (longitudinal_evolve! with use_mpi, src/evolution.jl:206-212; the exchange
 * sites of src/wakefield.jl:186-345 and src/evolution.jl:408-426).  Per turn:
 * hj_bunch_pass on every rank, a SUM all-reduce across ranks of the two
 * exchange buffers (u64 counts, double sums) on the shard's stream, then
 * hj_bunch_bins on every rank.  No reference counterpart for the split calls. */

/* Particles [first_particle, first_particle + n_local) of a bunch of n_global
 * (first_particle even; the Philox draws are the whole bunch's).  The grid
 * must be the same on every rank.  Before the first turn, sum
 * hj_bunch_local_moments over the ranks and pass the totals to
 * hj_bunch_set_global_moments. */
hj_status hj_bunch_create_shard(hj_ctx* ctx, double* d_z, double* d_dE, int64_t n_local,
                                int64_t first_particle, int64_t n_global,
                                const hj_params* params, const hj_wake* wake,
                                const hj_grid* grid, uint64_t seed, void* stream,
                                hj_bunch** out);
/* out = (Σz, Σz², ΣdE, ΣdE²) of this bunch's particles (pending kick applied,
 * state unchanged).  Synchronises the stream. */
hj_status hj_bunch_local_moments(hj_bunch* b, double* out4);
/* Initial spreads σ_z0, σ_E0 from the moments summed over all shards. */
hj_status hj_bunch_set_global_moments(hj_bunch* b, const double* sums4);
/* This turn's particle pass on the shard; fills the exchange buffers. */
hj_status hj_bunch_pass(hj_bunch* b);
/* Device buffers to SUM across ranks between hj_bunch_pass and hj_bunch_bins. */
hj_status hj_bunch_exchange_buffers(hj_bunch* b, uint64_t** d_counts, int64_t* n_counts,
                                    double** d_sums, int64_t* n_sums);
/* This turn's bins step from the exchanged totals. */
hj_status hj_bunch_bins(hj_bunch* b);

/* ---------------------------------------------------------------- batches
 * Many independent bunches -- each with its own particle count, RF voltage,
 * intensity, bins, seed and number of turns -- advanced together: every turn
 * is one particle-pass launch over a chunk table of all live bunches, one
 * histogram merge and one bins-step launch with a two-CTA cluster per bunch.
 * Blocks of K turns replay a captured CUDA graph.  A bunch's results do not
 * depend on which other bunches share the batch.  No reference counterpart:
 * the reference runs parameter points one after another
 * (src/parameter_sensitivity/scan.jl:182-184). */

/* A batch on ctx's device with its own stream: a particle pool of
 * pool_particles (16 B each), up to max_bunches bunches of up to max_nbins
 * bins, chunk_particles particles per block of the pass (a multiple of 4, at
 * most 2^20 - 8, what a block's packed cell counters can count; 0 = 65536)
 * and pass layout `layout` (-1 = the default for max_nbins; values as for
 * hj_set_pass_layout). */
hj_status hj_batch_create(hj_ctx* ctx, int64_t pool_particles, int32_t max_bunches,
                          int32_t max_nbins, int64_t chunk_particles, int32_t layout,
                          hj_batch** out);
void hj_batch_destroy(hj_batch* bt);
/* The batched pass's launch: on != 0 runs resident blocks, one per SM slot,
 * that take chunks of the chunk table from a device-side queue (an atomic
 * counter reset every turn) until the table is exhausted -- one persistent
 * launch per turn over the ragged table; 0 (the default) launches one block
 * per chunk, which the hardware scheduler hands out to free SMs as well and
 * which compiles without the queue loop's register spills.  Results are the
 * same either way (a chunk's slot and arithmetic do not depend on its
 * block).  No reference counterpart. */
hj_status hj_batch_set_resident(hj_batch* bt, int32_t on);
/* Turns per captured CUDA graph (0 = launch every turn directly; default 16). */
hj_status hj_batch_set_graph_turns(hj_batch* bt, int32_t turns);
/* Admit a bunch: z, dE (host or device, n each) are copied into the pool;
 * params/wake/nbins/seed as for hj_bunch_create (the wakefield must be on);
 * it runs `turns` turns.  *id_out names it.  HJ_ERR_FULL: no room now. */
hj_status hj_batch_add(hj_batch* bt, const double* z, const double* dE, int64_t n,
                       const hj_params* params, const hj_wake* wake, int64_t nbins,
                       uint64_t seed, int64_t turns, int64_t* id_out);
/* As hj_batch_add, with the bunch generated on the device: independent
 * Gaussians z ~ N(0, sigma_z), dE ~ N(0, sigma_E) (hj_gaussian_bunch). */
hj_status hj_batch_add_gaussian(hj_batch* bt, int64_t n, double sigma_z, double sigma_E,
                                uint64_t init_seed, const hj_params* params,
                                const hj_wake* wake, int64_t nbins, uint64_t seed,
                                int64_t turns, int64_t* id_out);
/* Admit up to `count` bunches in order with one synchronisation: bunch k has
 * particles z[k], dE[k] (host or device, copied), n[k], params[k], wakes[k]
 * (wakes NULL: the reference wake of each params), nbins[k], seeds[k] and
 * turns[k]; ids_out[k] receives its id.  Stops at the first bunch that cannot
 * be admitted and returns that bunch's status (HJ_ERR_FULL when the batch has
 * no room); *n_added bunches, the first ones, were admitted either way. */
hj_status hj_batch_add_many(hj_batch* bt, int32_t count, const double* const* z,
                            const double* const* dE, const int64_t* n, const hj_params* params,
                            const hj_wake* wakes, const int64_t* nbins, const uint64_t* seeds,
                            const int64_t* turns, int64_t* ids_out, int32_t* n_added);
/* Enqueue `turns` turns of every live bunch (a bunch stops at its own count). */
hj_status hj_batch_advance(hj_batch* bt, int64_t turns);
/* Wait for the enqueued turns; ids[0..*n_done-1] = bunches that have run all
 * their turns and are not taken yet (at most cap). */
hj_status hj_batch_poll(hj_batch* bt, int64_t* ids, int32_t cap, int32_t* n_done);
/* Finish bunch `id` (pending kick and re-centring applied), copy its (z, dE)
 * to z_out/dE_out (host or device, either may be NULL), fill *res, and free
 * its slot and pool range. */
hj_status hj_batch_take(hj_batch* bt, int64_t id, double* z_out, double* dE_out,
                        hj_result* res);
/* hj_batch_take for `count` bunches with one synchronisation (two with
 * corr_out): z_out/dE_out (NULL, or arrays of per-bunch destinations, entries
 * may be NULL), res[count] (or NULL), and corr_out[count] (or NULL): the
 * correlation cor(z, ΔE) of each bunch's final particles, as hj_correlation
 * computes it (for EmittanceFoM, src/parameter_sensitivity/figures_of_merit.jl:42). */
hj_status hj_batch_take_many(hj_batch* bt, int32_t count, const int64_t* ids,
                             double* const* z_out, double* const* dE_out, hj_result* res,
                             double* corr_out);
/* out[0] live bunches, out[1] free pool particles (largest free range),
 * out[2] free slots, out[3] turns enqueued so far. */
hj_status hj_batch_stats(hj_batch* bt, int64_t* out4);
/* The bin counts of bunch `id`'s last completed turn (the histogram of z
 * after that turn's drift, calculate_local_histogram! src/utils.jl:351-401)
 * into counts_host[nbins], after the enqueued turns complete. */
hj_status hj_batch_histogram(hj_batch* bt, int64_t id, int64_t* counts_host);

/* ---------------------------------------------------------------- single steps (host buffers) */

/* rf_kick!(voltage, sin_ϕs, rf_factor, ϕs, particles, buffers)
 * (src/rf_kick.jl:18-25, body :84-87): dE += V (sin(-z k + ϕs) - sin ϕs). */
hj_status hj_rf_kick(hj_ctx* ctx, double voltage, double sin_phis, double rf_factor,
                     double phi_s, const double* z, double* dE, int64_t n);

/* quantum_excitation!(E0, radius, σ_E0, buffers, particles)
 * (src/quantum_excitation.jl:24-30, :58-71).  draws: host array of n normals
 * or NULL for Philox(seed, particle, turn). */
hj_status hj_quantum_excitation(hj_ctx* ctx, double E0, double radius, double sigma_E0,
                                const double* draws, uint64_t seed, int64_t turn,
                                double* dE, int64_t n);

/* synchrotron_radiation!(E0, radius, particles, buffers)
 * (src/synchrotron_radiation.jl:12-17, :44-56): dE *= 1 - 4*8.85e-5*(E0/1e9)^3/radius. */
hj_status hj_synchrotron_radiation(hj_ctx* ctx, double E0, double radius, double* dE,
                                   int64_t n);

/* Phase advance of longitudinal_evolve!: update_eta != 0 is the inline loop
 * at src/evolution.jl:331-344; update_eta == 0 is apply_phase_advance!
 * (src/evolution.jl:143-167, skipped for non-physical beta0/E0/rf_factor). */
hj_status hj_phase_advance(hj_ctx* ctx, int32_t update_eta, double E0, double mass,
                           double alpha_c, int64_t harmonic, double phi_s,
                           double freq_rf, const double* dE, double* z, int64_t n);

/* calculate_local_histogram! (src/utils.jl:351-401): counts[nbins] of z. */
hj_status hj_histogram(hj_ctx* ctx, const double* z, int64_t n, const hj_grid* grid,
                       int64_t* counts);

/* The convolution of apply_wakefield_inplace! (MPI branch,
 * src/wakefield.jl:186-327): potential at the bin centers from integer
 * counts, pot = Re(IFFT(FFT(W) FFT(delta*counts/sum(counts)) * current)). */
hj_status hj_wake_potential(hj_ctx* ctx, const int64_t* counts, const hj_grid* grid,
                            const hj_wake* wake, double current, double* pot);

/* Same potential as hj_wake_potential, on DEVICE buffers, with no allocation.
 * No counterpart in the reference.  For callers that cannot call cudaMalloc:
 * those whose device memory is all owned by another allocator (a framework's
 * pool, a fixed arena sized at start-up), and latency-critical loops, since
 * cudaMalloc/cudaFree can synchronise the device.  It calls no
 * cudaMalloc/cudaFree and keeps its FFT tables and work space in one static
 * device array of about 1.4 MB that every GPU loading the library holds
 * until exit.  Limit: nbins <= 16384 (HJ_ERR_TOO_LARGE beyond).
 *   d_counts  device array of nbins non-negative bin counts;
 *   grid      host struct and host centres (copied into the static array);
 *   d_pot     device array of nbins doubles, written on `stream`.
 * The work is enqueued on `stream` (a cudaStream_t, NULL = legacy default
 * stream) and is complete when that stream is.  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) and keeps it
 * for the life of the process; make that first call before any stream
 * capture, and do not reset the device (cudaDeviceReset) while the library
 * is in use.  All calls share the array: calls whose work overlaps on the GPU
 * race, so serialise them.  The caller's current device is restored on
 * return. */
hj_status hj_wake_potential_noalloc(hj_ctx* ctx, const int64_t* d_counts, const hj_grid* grid,
                                    const hj_wake* wake, double current, double* d_pot,
                                    void* stream);

/* apply_wakefield_inplace!(particles, buffers, wake_factor, wake_sqrt, cτ,
 * current, sigma_z, bin_edges, bin_centers, comm, use_mpi=true)
 * (src/wakefield.jl:137-345): histogram, convolution, interpolation
 * (src/wakefield.jl:22-105) and dE -= potential.  sigma_z is accepted for
 * signature parity and, as in the reference's MPI branch, unused. */
hj_status hj_apply_wakefield(hj_ctx* ctx, const double* z, double* dE, int64_t n,
                             const hj_wake* wake, double current, double sigma_z,
                             const hj_grid* grid);

/* A bunch of independent Gaussians on the device: d_z[i] = sigma_z * N0,
 * d_dE[i] = sigma_E * N1 with (N0, N1) the Philox-4x32-10 / ziggurat pair of
 * particle i under init_seed (a stream apart from the quantum-excitation
 * draws).  Enqueued on `stream`.  The reference draws its bunches with
 * Distributions.jl on the host (generate_particles, src/evolution.jl:42-133,
 * with a covariance estimate; the benchmark configurations use independent
 * Gaussians). */
hj_status hj_gaussian_bunch(hj_ctx* ctx, uint64_t init_seed, int64_t n, double sigma_z,
                            double sigma_E, double* d_z, double* d_dE, void* stream);

/* generate_particles(μ_z, μ_E, σ_z, σ_E, num_particles, ...)
 * (src/evolution.jl:42-133) on the device: the covariance of a sample of
 * min(n, 10000) independent Gaussians, its positive-definite guard, then n
 * correlated draws mu + L eps (L its Cholesky factor) into d_z, d_dE, and the
 * actual spreads by the two-pass compute_std (src/utils.jl:531-544).  Draws
 * are Philox-4x32-10 / ziggurat normals under `seed` (the reference's come from
 * Julia's default RNG).  n <= 0: spreads 0; n = 1: one independent draw and
 * the input spreads, as the reference returns them. */
hj_status hj_generate_particles(hj_ctx* ctx, double mu_z, double mu_E, double sigma_z,
                                double sigma_E, int64_t n, uint64_t seed, double* d_z,
                                double* d_dE, void* stream, double* actual_sigma_E,
                                double* actual_sigma_z);

/* cor(particles.coordinates.z, particles.coordinates.ΔE), the correlation
 * EmittanceFoM computes (src/parameter_sensitivity/figures_of_merit.jl:42), of
 * two device arrays of n doubles: Pearson r from two passes (means, then the
 * centred sums), clamped to [-1, 1]; NaN when a spread is zero.  n <= 0 is
 * HJ_ERR_ARG, as cor rejects empty vectors.  Synchronises `stream`. */
hj_status hj_correlation(hj_ctx* ctx, const double* d_x, const double* d_y, int64_t n,
                         void* stream, double* out);

/* The Float64 standard normals used for quantum excitation: out[i] = the
 * N(0,1) draw of particle i at `turn` under `seed` (Philox-4x32-10 of
 * (pair i/2, turn) keyed by the 64-bit seed, 64 bits per normal, a 2048-layer
 * ziggurat whose rare slow path draws further Philox words keyed by
 * (pair, turn, attempt); turns below 2^56).  No reference counterpart (the
 * reference calls randn!, src/quantum_excitation.jl:36, whose algorithm is
 * also a ziggurat). */
hj_status hj_gaussian(hj_ctx* ctx, uint64_t seed, int64_t turn, int64_t n, double* out);

/* The ziggurat's tables, for restatements of it (no reference counterpart;
 * host only, no context): out[HJ_NORMAL_TABLES_SIZE] = 2048 pairs (X_i, D_i)
 * (layer i's width and its fast-acceptance bound 1 + ceil(2^52 X_{i+1}/X_i)
 * 2^-52, X_2048 = 0), the 2049 values f(X_i) = exp(-X_i^2/2), r = X_1 (the
 * tail's start) and v (the layers' common area).  cap <
 * HJ_NORMAL_TABLES_SIZE is HJ_ERR_ARG. */
#define HJ_NORMAL_TABLES_SIZE 6147
hj_status hj_normal_tables(double* out, int64_t cap);

#ifdef __cplusplus
}
#endif

#endif /* HAISSINSKI_GPU_H */
