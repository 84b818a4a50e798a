/*
 * oracle.h -- CPU restatement of HaissinskiJulia's longitudinal_evolve! turn
 * loop.  TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg as the checker / CPU timing reference.
 * The product path (haissinskijulia_b200) never links or calls it.
 *
 * Parity status: UNPINNED against the reference itself.  The reference is
 * Julia (not installed in this environment) and ships no golden vectors,
 * known-answer tests or fixtures for this path (its tests/loop_benchmark.jl
 * only cross-checks its own loop variants at rtol 1e-12).  The restatement is
 * checked against independent high-precision restatements of each step
 * formula (tests/golden/make_golden.py) and against a direct long-double
 * convolution for the FFT step.
 *
 * Every function cites the reference file:line it follows.  The parameter
 * structs are the library's POD structs (include/haissinski_gpu.h) so the
 * oracle and the GPU path read identical inputs.
 */
#ifndef HJ_ORACLE_H
#define HJ_ORACLE_H

#include <stdint.h>
#include "../include/haissinski_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* src/constants.jl:5-7 */
#define OR_SPEED_LIGHT 299792458.0
#define OR_MASS_ELECTRON 0.51099895069e6

/* Convolution method for the wake potential. */
enum { OR_CONV_FFT = 0, OR_CONV_DIRECT_LD = 1 };

typedef struct or_state or_state;

/* Number of OpenMP threads used by the particle loops (1 = serial order). */
void or_set_threads(int32_t nthreads);
int32_t or_get_threads(void);

/* ---- per-step restatements (all in place on host arrays) ---- */
double or_compute_global_std(const double* x, int64_t n);     /* src/utils.jl:569-606 */
double or_compute_std(const double* x, int64_t n);            /* src/utils.jl:531-544 */
double or_calc_rf_factor(double freq_rf, double beta);        /* src/utils.jl:484-491 */
int64_t or_next_power_of_two(int64_t n);                      /* src/utils.jl:119-122 */
double or_delta(double x, double sigma);                      /* src/utils.jl:58-66 */
double or_wake_function(double c, const hj_wake* w);          /* src/wakefield.jl:115-118 */
void or_rf_kick(double voltage, double sin_phis, double rf_factor, double phi_s,
                const double* z, double* dE, int64_t n);      /* src/rf_kick.jl:84-87 */
void or_quantum_excitation(double E0, double radius, double sigma_E0,
                           const double* draws, double* dE, int64_t n);  /* src/quantum_excitation.jl:58-71 */
void or_synchrotron_radiation(double E0, double radius, double* dE, int64_t n);  /* src/synchrotron_radiation.jl:44-56 */
void or_drift_update_eta(double E0, double mass, double alpha_c, int64_t harmonic,
                         double phi_s, double freq_rf, const double* dE, double* z,
                         int64_t n);                          /* src/evolution.jl:300-304, :331-344 */
int32_t or_apply_phase_advance(double E0, double mass, double alpha_c, int64_t harmonic,
                               double phi_s, double freq_rf, const double* dE, double* z,
                               int64_t n);                    /* src/evolution.jl:143-167 */
void or_histogram(const double* z, int64_t n, const hj_grid* g, int64_t* counts);  /* src/utils.jl:351-401 */
/* pot[nbins] from counts: MPI branch of src/wakefield.jl:186-327. */
void or_wake_potential(const int64_t* counts, const hj_grid* g, const hj_wake* w,
                       double current, int32_t conv_mode, double* pot);
/* dE -= lerp(pot, z) (src/wakefield.jl:22-105, :342-344). */
void or_interp_kick(const double* z, double* dE, int64_t n, const hj_grid* g,
                    const double* pot);
/* current = particle_factor/E0/(2 pi radius) * sigma_z / (eta0 sigma_E0^2)
 * (src/evolution.jl:373-386); population > 0 replaces particle_factor. */
double or_wake_current(int64_t n_global, double E0, double mass, double alpha_c,
                       double radius, double sigma_z, double sigma_E0_initial,
                       double population);
/* Grid with correctly rounded edges/centers (same construction as hj_make_grid). */
int32_t or_make_grid(double sigma_z0, double half_width_sigmas, int64_t nbins,
                     double* centers, hj_grid* out);
/* Oracle's own standard normals: splitmix64 counter hash of (seed, turn,
 * particle) + Box-Muller.  Independent of the GPU's Philox stream. */
void or_gaussian(uint64_t seed, int64_t turn, int64_t n, double* out);

/* ---- whole turn loop ---- */
/*
 * Create a tracking state over caller-owned host arrays z/dE (n each).
 * Computes sigma_E0_initial / sigma_z0_initial (src/evolution.jl:247-249,
 * compute_global_std) and the bin grid (grid == NULL: or_make_grid on
 * sigma_z0_initial; otherwise copied).  rng: draws == NULL in or_turn uses
 * or_gaussian(seed, turn, ...).
 */
or_state* or_create(double* z, double* dE, int64_t n, const hj_params* p,
                    const hj_wake* w, int64_t nbins, const hj_grid* grid,
                    uint64_t seed, int32_t conv_mode);
/* One full turn of src/evolution.jl:295-456 (RF, QE, SR, drift, wake, E0
 * update).  draws: n normals for this turn or NULL. Returns 0 or an HJ_ERR. */
int32_t or_turn(or_state* s, const double* draws);
/* Final spreads and E0 (src/evolution.jl:458-470). */
void or_result(const or_state* s, hj_result* out);
/* Diagnostics of the last turn. */
double or_last_sigma_z(const or_state* s);
double or_last_current(const or_state* s);
double or_last_mean(const or_state* s);
double or_E0(const or_state* s);
int64_t or_nbins(const or_state* s);
const double* or_centers(const or_state* s);
const int64_t* or_last_counts(const or_state* s);
const double* or_last_potential(const or_state* s);
double or_grid_edge_first(const or_state* s);
double or_grid_edge_last(const or_state* s);
double or_grid_edge_step(const or_state* s);
void or_destroy(or_state* s);

/* Convenience: create, n_turns turns (draws: n_turns*n turn-major or NULL),
 * result, destroy.  Mirrors longitudinal_evolve! end to end. */
int32_t or_evolve(double* z, double* dE, int64_t n, const hj_params* p, const hj_wake* w,
                  int64_t nbins, const hj_grid* grid, const double* draws, uint64_t seed,
                  int32_t conv_mode, hj_result* out);

/* Reference-mode wake constants (src/evolution.jl:276-280). */
void or_wake_reference(const hj_params* p, hj_wake* out);

#ifdef __cplusplus
}
#endif
#endif
