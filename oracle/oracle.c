/*
 * oracle.c -- CPU restatement of HaissinskiJulia's longitudinal_evolve! turn
 * loop (MPI branch at any rank count, which is the branch that runs with the
 * wakefield on).  TEST INFRASTRUCTURE ONLY: the checker for tests/, smoke()
 * and the CPU-baseline leg of bench.py.  Never part of the product path.
 *
 * Parity: UNPINNED against the reference itself (Julia is not installed and
 * the reference ships no golden vectors for this path).  Each step is
 * written as the reference source states it, operation for operation, and
 * compiled without floating-point contraction (-ffp-contract=off) so every
 * rounding happens where the Julia source puts it.
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int32_t g_threads = 1;

void or_set_threads(int32_t nthreads) { g_threads = nthreads < 1 ? 1 : nthreads; }
int32_t or_get_threads(void) { return g_threads; }

/* 2*pi and pi as Julia's Float64 conversions of the Irrational constants. */
static const double TWO_PI = 6.283185307179586;
static const double PI_D = 3.141592653589793;

/* ------------------------------------------------------------------ stats */

/* compute_global_std, src/utils.jl:569-606: single pass sums, biased
 * variance E[x^2]-E[x]^2 scaled by n/(n-1). */
double or_compute_global_std(const double* x, int64_t n) {
  double s = 0.0, s2 = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double v = x[i];
    s += v;
    s2 += v * v;
  }
  if (n <= 1) return 0.0;
  double nd = (double)n;
  double mean = s / nd;
  double var = (s2 / nd) - (mean * mean);
  double svar = var * nd / (double)(n - 1);
  if (!(svar > 0.0)) svar = (svar != svar) ? svar : 0.0; /* max(0, v) keeping NaN */
  return sqrt(svar);
}

/* compute_std, src/utils.jl:531-544: two-pass sample std. */
double or_compute_std(const double* x, int64_t n) {
  if (n <= 1) return 0.0;
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += x[i];
  double mu = s / (double)n;
  double ss = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double d = x[i] - mu;
    ss += d * d;
  }
  double var = ss / (double)(n - 1);
  return sqrt(var > 0.0 ? var : 0.0);
}

/* calc_rf_factor, src/utils.jl:484-491. */
double or_calc_rf_factor(double freq_rf, double beta) {
  if (beta <= 0.0) return INFINITY;
  return freq_rf * TWO_PI / (beta * OR_SPEED_LIGHT);
}

/* next_power_of_two, src/utils.jl:119-122 (2^ceil(log2 n), n <= 0 -> 1). */
int64_t or_next_power_of_two(int64_t n) {
  if (n <= 0) return 1;
  int64_t p = 1;
  while (p < n) p <<= 1;
  return p;
}

/* delta, src/utils.jl:58-66. */
double or_delta(double x, double sigma) {
  double inv = 1.0 / (sqrt(TWO_PI) * sigma);
  double f = -0.5 / (sigma * sigma);
  return inv * exp(x * x * f);
}

/* calculate_wake_function, src/wakefield.jl:115-118 (sin_coef = 0 there). */
double or_wake_function(double c, const hj_wake* w) {
  if (c > 0.0) return 0.0;
  double inv_ctau = 1.0 / w->ctau;
  double osc = cos(w->wake_sqrt * c);
  if (w->sin_coef != 0.0) osc = osc + w->sin_coef * sin(w->wake_sqrt * c);
  return w->wake_factor * exp(c * inv_ctau) * osc;
}

/* ------------------------------------------------------------------ steps */

/* rf_kick!, src/rf_kick.jl:84-87. */
void or_rf_kick(double voltage, double sin_phis, double rf_factor, double phi_s,
                const double* z, double* dE, int64_t n) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double phi = -z[i] * rf_factor + phi_s;
    dE[i] += voltage * (sin(phi) - sin_phis);
  }
}

/* quantum_excitation!, src/quantum_excitation.jl:58-71 (randn! replaced by draws). */
void or_quantum_excitation(double E0, double radius, double sigma_E0, const double* draws,
                           double* dE, int64_t n) {
  double t = E0 / 1e9;
  double dU = 4 * 8.85e-5 * (t * t * t) / radius;
  double om = 1 - dU;
  double excitation = sqrt(1 - om * om) * sigma_E0;
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; ++i) dE[i] += excitation * draws[i];
}

/* synchrotron_radiation!, src/synchrotron_radiation.jl:44-56. */
void or_synchrotron_radiation(double E0, double radius, double* dE, int64_t n) {
  double t = E0 / 1e9;
  double dU = 4 * 8.85e-5 * (t * t * t) / radius;
  double damping = 1 - dU;
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; ++i) dE[i] *= damping;
}

typedef struct turn_scalars {
  double gamma0, beta0, eta0, sin_phis, rf_factor;
} turn_scalars;

/* Per-turn scalars, src/evolution.jl:300-304. */
static turn_scalars scalars_of(double E0, double mass, double alpha_c, double phi_s,
                               double freq_rf) {
  turn_scalars t;
  t.gamma0 = E0 / mass;
  double b2 = 1.0 - 1.0 / (t.gamma0 * t.gamma0);
  t.beta0 = sqrt(b2 > 0.0 ? b2 : 0.0);
  t.eta0 = alpha_c - (1.0 / (t.gamma0 * t.gamma0));
  t.sin_phis = sin(phi_s);
  t.rf_factor = or_calc_rf_factor(freq_rf, t.beta0);
  return t;
}

/* Energy-dependent slip factor drift, src/evolution.jl:331-344. */
void or_drift_update_eta(double E0, double mass, double alpha_c, int64_t harmonic,
                         double phi_s, double freq_rf, const double* dE, double* z,
                         int64_t n) {
  turn_scalars t = scalars_of(E0, mass, alpha_c, phi_s, freq_rf);
  double two_pi_h = TWO_PI * (double)harmonic;
  double b2E0 = t.beta0 * t.beta0 * E0;
  double k = t.rf_factor;
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double dgam = dE[i] / mass;
    double gp = t.gamma0 + dgam;
    double eta = alpha_c - 1.0 / (gp * gp);
    double coeff = (two_pi_h * eta / b2E0);
    double phi = -(z[i] * k - phi_s);
    phi += coeff * dE[i];
    z[i] = (-phi + phi_s) / k;
  }
}

/* apply_phase_advance!, src/evolution.jl:143-167.  Returns 1 when skipped. */
int32_t or_apply_phase_advance(double E0, double mass, double alpha_c, int64_t harmonic,
                               double phi_s, double freq_rf, const double* dE, double* z,
                               int64_t n) {
  turn_scalars t = scalars_of(E0, mass, alpha_c, phi_s, freq_rf);
  if (n == 0) return 0;
  if (t.beta0 <= 0 || E0 == 0 || t.rf_factor == 0) return 1;
  double coeff = (TWO_PI * (double)harmonic * t.eta0 / (t.beta0 * t.beta0 * E0));
  double k = t.rf_factor;
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double phi = -(z[i] * k - phi_s);
    phi += coeff * dE[i];
    z[i] = (-phi + phi_s) / k;
  }
  return 0;
}

/* calculate_local_histogram!, src/utils.jl:351-401. */
void or_histogram(const double* z, int64_t n, const hj_grid* g, int64_t* counts) {
  int64_t B = g->nbins;
  memset(counts, 0, sizeof(int64_t) * (size_t)B);
  if (n == 0) return;
  double e0 = g->edge_first, eN = g->edge_last;
  double inv = 1.0 / g->edge_step;
  if (g_threads <= 1) {
    for (int64_t i = 0; i < n; ++i) {
      double x = z[i];
      int in_range = (x >= e0) & (x <= eN);
      double u = floor((x - e0) * inv);
      int64_t j;
      if (u != u) j = 1;                         /* NaN: out of range anyway */
      else if (u < 0.0) j = 1;
      else if (u >= (double)B) j = B;
      else j = (int64_t)u + 1;
      if (j < 1) j = 1;
      if (j > B) j = B;
      counts[j - 1] += in_range;
    }
    return;
  }
#pragma omp parallel num_threads(g_threads)
  {
    int64_t* loc = (int64_t*)calloc((size_t)B, sizeof(int64_t));
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      double x = z[i];
      int in_range = (x >= e0) & (x <= eN);
      double u = floor((x - e0) * inv);
      int64_t j;
      if (u != u) j = 1;
      else if (u < 0.0) j = 1;
      else if (u >= (double)B) j = B;
      else j = (int64_t)u + 1;
      loc[j - 1] += in_range;
    }
#pragma omp critical
    for (int64_t b = 0; b < B; ++b) counts[b] += loc[b];
    free(loc);
  }
}

/* ------------------------------------------------------------------ FFT */

typedef struct cplx { double re, im; } cplx;

/* Iterative radix-2 complex FFT of size P (power of two), in place.
 * sign = -1 forward, +1 inverse (unnormalised).  Twiddles are computed in
 * long double and rounded once. */
static void fft_radix2(cplx* a, int64_t P, int sign) {
  for (int64_t i = 1, j = 0; i < P; ++i) {
    int64_t bit = P >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) { cplx t = a[i]; a[i] = a[j]; a[j] = t; }
  }
  cplx* tw = (cplx*)malloc(sizeof(cplx) * (size_t)(P / 2 > 0 ? P / 2 : 1));
  const long double PI_L = 3.141592653589793238462643383279502884L;
  for (int64_t k = 0; k < P / 2; ++k) {
    long double ang = (long double)sign * 2.0L * PI_L * (long double)k / (long double)P;
    tw[k].re = (double)cosl(ang);
    tw[k].im = (double)sinl(ang);
  }
  for (int64_t len = 2; len <= P; len <<= 1) {
    int64_t half = len >> 1, stride = P / len;
    for (int64_t i = 0; i < P; i += len) {
      for (int64_t j = 0; j < half; ++j) {
        cplx w = tw[j * stride];
        cplx u = a[i + j], v = a[i + j + half];
        cplx t = {v.re * w.re - v.im * w.im, v.re * w.im + v.im * w.re};
        a[i + j].re = u.re + t.re;
        a[i + j].im = u.im + t.im;
        a[i + j + half].re = u.re - t.re;
        a[i + j + half].im = u.im - t.im;
      }
    }
  }
  free(tw);
}

/* Wake potential at the bin centers: MPI branch of apply_wakefield_inplace!,
 * src/wakefield.jl:186-327. */
void or_wake_potential(const int64_t* counts, const hj_grid* g, const hj_wake* w,
                       double current, int32_t conv_mode, double* pot) {
  int64_t B = g->nbins;
  int64_t P = or_next_power_of_two(B * 2);
  int64_t ntot = 0;
  for (int64_t i = 0; i < B; ++i) ntot += counts[i];
  if (ntot == 0) { /* src/wakefield.jl:305-311: no IFFT, zero potential */
    for (int64_t i = 0; i < B; ++i) pot[i] = 0.0;
    return;
  }
  double inv_n = 1.0 / (double)ntot;                          /* :207 */
  double* Wt = (double*)malloc(sizeof(double) * (size_t)B);
  double* gl = (double*)malloc(sizeof(double) * (size_t)B);
  for (int64_t i = 0; i < B; ++i) {
    Wt[i] = or_wake_function(g->centers[i], w);               /* :194-196 */
    double normalized = (double)counts[i] * inv_n;            /* :209-211 */
    double lam = or_delta(g->centers[i], w->delta_std);       /* :219-221 */
    gl[i] = lam * normalized;                                 /* :238 */
  }
  if (conv_mode == OR_CONV_DIRECT_LD) {
    /* Ground truth: causal truncated linear convolution in long double,
     * pot[i] = current * sum_{j<=i} W[j] g[i-j]. */
    for (int64_t i = 0; i < B; ++i) {
      long double acc = 0.0L;
      for (int64_t j = 0; j <= i; ++j) acc += (long double)Wt[j] * (long double)gl[i - j];
      pot[i] = (double)((long double)current * acc);
    }
  } else {
    cplx* fW = (cplx*)calloc((size_t)P, sizeof(cplx));
    cplx* fL = (cplx*)calloc((size_t)P, sizeof(cplx));
    for (int64_t i = 0; i < B; ++i) { fW[i].re = Wt[i]; fL[i].re = gl[i]; }  /* :234-239 */
    fft_radix2(fW, P, -1);                                    /* :242-243 */
    fft_radix2(fL, P, -1);
    for (int64_t i = 0; i < P; ++i) {                         /* :286-288 */
      cplx a = fW[i], b = fL[i];
      cplx c = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
      fW[i].re = c.re * current;
      fW[i].im = c.im * current;
    }
    fft_radix2(fW, P, +1);                                    /* :307, normalised ifft */
    double invP = 1.0 / (double)P;
    for (int64_t i = 0; i < B; ++i) pot[i] = fW[i].re * invP; /* :315-319 */
    free(fW);
    free(fL);
  }
  free(Wt);
  free(gl);
}

/* zero_alloc_interpolation! + kick, src/wakefield.jl:22-105, :342-344. */
void or_interp_kick(const double* z, double* dE, int64_t n, const hj_grid* g,
                    const double* pot) {
  int64_t B = g->nbins;
  if (B <= 1) {
    double v = (B == 1) ? pot[0] : 0.0;
    for (int64_t i = 0; i < n; ++i) dE[i] -= v;
    return;
  }
  double c1 = g->centers[0], cB = g->centers[B - 1];
  double step = (cB - c1) / (double)(B - 1);
  double inv = 1.0 / step;
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double pos = z[i];
    double cl = pos > cB ? cB : (pos < c1 ? c1 : pos);
    double u = (cl - c1) * inv;
    double fl = floor(u);
    int64_t idx = (int64_t)fl + 1;
    if (idx < 1) idx = 1;
    if (idx > B - 1) idx = B - 1;
    double wgt = u - fl;
    double p = pot[idx - 1] * (1.0 - wgt) + pot[idx] * wgt;
    dE[i] -= p;
  }
}

/* Wake "current", src/evolution.jl:373-386. */
double or_wake_current(int64_t n_global, double E0, double mass, double alpha_c,
                       double radius, double sigma_z, double sigma_E0_initial,
                       double population) {
  double g0 = E0 / mass;
  double eta0 = alpha_c - (1.0 / (g0 * g0));
  double pf;
  if (population > 0.0) {
    pf = population;
  } else {
    double l10 = log10((double)n_global);
    int64_t fl = l10 >= 0 ? (int64_t)floor(l10) : (int64_t)ceil(l10 - 1);
    int64_t pw = fl < 10 ? fl : 10;
    if (pw < -10) pw = -10;
    double den = pow(10.0, (double)pw);
    if (den == 0) den = 1.0;
    pf = (1e11 / den) * (double)n_global;
  }
  return pf / E0 / (TWO_PI * radius) * sigma_z / (eta0 * (sigma_E0_initial * sigma_E0_initial));
}

/* ------------------------------------------------------------------ grid */

int32_t or_make_grid(double sigma_z0, double half_width_sigmas, int64_t nbins,
                     double* centers, hj_grid* out) {
  if (nbins <= 0) return HJ_ERR_NBINS;
  double w = half_width_sigmas * sigma_z0;                   /* src/evolution.jl:270 */
  if (w < 1e-9) w = 1e-6;                                    /* :272 */
  __float128 W = (__float128)w, Bq = (__float128)nbins;
  for (int64_t k = 0; k < nbins; ++k)
    centers[k] = (double)(W * (__float128)(2 * k + 1 - nbins) / Bq);
  out->nbins = nbins;
  out->edge_first = -w;
  out->edge_last = w;
  out->edge_step = (double)((W * 2) / Bq);
  out->centers = centers;
  return HJ_OK;
}

/* ------------------------------------------------------------------ RNG */

static inline uint64_t mix64(uint64_t x) {
  /* SplitMix64 (Steele, Lea & Flood, OOPSLA 2014) output function. */
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

void or_gaussian(uint64_t seed, int64_t turn, int64_t n, double* out) {
  uint64_t ks = mix64(seed ^ mix64((uint64_t)turn * 0xD1B54A32D192ED03ULL));
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int64_t j = 0; j < (n + 1) / 2; ++j) {
    uint64_t a = mix64(ks ^ mix64((uint64_t)j));
    uint64_t b = mix64(a);
    double u1 = ((double)(a >> 11) + 0.5) * 0x1.0p-53;
    double u2 = ((double)(b >> 11) + 0.5) * 0x1.0p-53;
    double r = sqrt(-2.0 * log(u1));
    double th = TWO_PI * u2;
    out[2 * j] = r * cos(th);
    if (2 * j + 1 < n) out[2 * j + 1] = r * sin(th);
  }
}

/* ------------------------------------------------------------------ loop */

struct or_state {
  hj_params p;
  hj_wake w;
  int64_t n;
  double* z;
  double* dE;
  double E0;
  double sigma_E0_initial, sigma_z0_initial;
  hj_grid grid;
  double* centers;
  int64_t* counts;
  double* pot;
  double* dE_init;
  double* draws_buf;
  uint64_t seed;
  int32_t conv_mode;
  int64_t turn;
  double last_sigma_z, last_current, last_mean;
};

void or_wake_reference(const hj_params* p, hj_wake* out) {
  double kp = 3e1, Z0 = 120 * PI_D, ctau = 4e-3;              /* src/evolution.jl:276 */
  out->wake_factor = Z0 * OR_SPEED_LIGHT / (PI_D * p->pipe_radius);   /* :279 */
  double a = 2 * kp / p->pipe_radius;
  out->wake_sqrt = sqrt(a > 0 ? a : 0);                      /* :280 */
  out->ctau = ctau;
  out->sin_coef = 0.0;
  out->population = 0.0;
  out->half_width_sigmas = 7.5;
  out->delta_std = 0.15;
}

or_state* or_create(double* z, double* dE, int64_t n, const hj_params* p,
                    const hj_wake* w, int64_t nbins, const hj_grid* grid,
                    uint64_t seed, int32_t conv_mode) {
  or_state* s = (or_state*)calloc(1, sizeof(or_state));
  s->p = *p;
  if (w) s->w = *w; else or_wake_reference(p, &s->w);
  s->n = n;
  s->z = z;
  s->dE = dE;
  s->E0 = p->E0;
  s->seed = seed;
  s->conv_mode = conv_mode;
  s->sigma_E0_initial = or_compute_global_std(dE, n);         /* src/evolution.jl:248 */
  s->sigma_z0_initial = or_compute_global_std(z, n);          /* :249 */
  if (p->use_wakefield) {
    int64_t B = grid ? grid->nbins : nbins;
    if (B <= 0) { free(s); return NULL; }
    s->centers = (double*)malloc(sizeof(double) * (size_t)B);
    if (grid) {
      memcpy(s->centers, grid->centers, sizeof(double) * (size_t)B);
      s->grid = *grid;
      s->grid.centers = s->centers;
    } else {
      or_make_grid(s->sigma_z0_initial, s->w.half_width_sigmas, B, s->centers, &s->grid);
    }
    s->counts = (int64_t*)calloc((size_t)B, sizeof(int64_t));
    s->pot = (double*)calloc((size_t)B, sizeof(double));
  }
  s->dE_init = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  s->draws_buf = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  return s;
}

int32_t or_turn(or_state* s, const double* draws) {
  const hj_params* p = &s->p;
  int64_t n = s->n;
  s->turn += 1;
  turn_scalars t = scalars_of(s->E0, p->mass, p->alpha_c, p->phi_s, p->freq_rf);  /* :300-304 */
  if (p->update_E0 && n > 0) memcpy(s->dE_init, s->dE, sizeof(double) * (size_t)n);  /* :307-309 */
  if (n > 0) or_rf_kick(p->voltage, t.sin_phis, t.rf_factor, p->phi_s, s->z, s->dE, n);  /* :313 */
  if (p->use_excitation && n > 0) {                                                  /* :318-320 */
    const double* r = draws;
    if (!r) { or_gaussian(s->seed, s->turn, n, s->draws_buf); r = s->draws_buf; }
    or_quantum_excitation(s->E0, p->radius, s->sigma_E0_initial, r, s->dE, n);
  }
  if (p->SR_damping && n > 0) or_synchrotron_radiation(s->E0, p->radius, s->dE, n);  /* :323-325 */
  if (n > 0) {                                                                       /* :329-348 */
    if (p->update_eta)
      or_drift_update_eta(s->E0, p->mass, p->alpha_c, p->harmonic, p->phi_s, p->freq_rf,
                          s->dE, s->z, n);
    else
      or_apply_phase_advance(s->E0, p->mass, p->alpha_c, p->harmonic, p->phi_s,
                             p->freq_rf, s->dE, s->z, n);
  }
  if (p->use_wakefield) {                                                            /* :351-398 */
    if (n == 0) return HJ_ERR_EMPTY;
    double sz = or_compute_global_std(s->z, n);                                      /* :357 */
    double cur = or_wake_current(n, s->E0, p->mass, p->alpha_c, p->radius, sz,
                                 s->sigma_E0_initial, s->w.population);
    s->last_sigma_z = sz;
    s->last_current = cur;
    or_histogram(s->z, n, &s->grid, s->counts);                                      /* wakefield.jl:175 */
    or_wake_potential(s->counts, &s->grid, &s->w, cur, s->conv_mode, s->pot);
    or_interp_kick(s->z, s->dE, n, &s->grid, s->pot);                                /* :331-344 */
  }
  if (p->update_E0) {                                                                /* :401-451 */
    double sum = 0.0;
    for (int64_t i = 0; i < n; ++i) sum += (s->dE[i] - s->dE_init[i]);               /* :408-411 */
    double mean = sum / (double)n;                                                   /* :426 */
    s->E0 = s->E0 + mean;                                                            /* :429 */
    s->last_mean = mean;
    if (n > 0) {
#pragma omp parallel for num_threads(g_threads) schedule(static)
      for (int64_t i = 0; i < n; ++i) s->dE[i] -= mean;                              /* :434 */
    }
  }
  return HJ_OK;
}

void or_result(const or_state* s, hj_result* out) {
  out->sigma_E = or_compute_global_std(s->dE, s->n);          /* src/evolution.jl:462 */
  out->sigma_z = or_compute_global_std(s->z, s->n);           /* :463 */
  out->E0 = s->E0;
  out->sigma_E0_initial = s->sigma_E0_initial;
  out->sigma_z0_initial = s->sigma_z0_initial;
  double sz = 0.0, se = 0.0;
  for (int64_t i = 0; i < s->n; ++i) { sz += s->z[i]; se += s->dE[i]; }
  out->mean_z = s->n > 0 ? sz / (double)s->n : 0.0;
  out->mean_dE = s->n > 0 ? se / (double)s->n : 0.0;
  out->turns = s->turn;
}

double or_last_sigma_z(const or_state* s) { return s->last_sigma_z; }
double or_last_current(const or_state* s) { return s->last_current; }
double or_last_mean(const or_state* s) { return s->last_mean; }
double or_E0(const or_state* s) { return s->E0; }
int64_t or_nbins(const or_state* s) { return s->grid.nbins; }
const double* or_centers(const or_state* s) { return s->centers; }
const int64_t* or_last_counts(const or_state* s) { return s->counts; }
const double* or_last_potential(const or_state* s) { return s->pot; }
double or_grid_edge_first(const or_state* s) { return s->grid.edge_first; }
double or_grid_edge_last(const or_state* s) { return s->grid.edge_last; }
double or_grid_edge_step(const or_state* s) { return s->grid.edge_step; }

void or_destroy(or_state* s) {
  if (!s) return;
  free(s->centers);
  free(s->counts);
  free(s->pot);
  free(s->dE_init);
  free(s->draws_buf);
  free(s);
}

int32_t or_evolve(double* z, double* dE, int64_t n, const hj_params* p, const hj_wake* w,
                  int64_t nbins, const hj_grid* grid, const double* draws, uint64_t seed,
                  int32_t conv_mode, hj_result* out) {
  if (p->use_wakefield && (grid ? grid->nbins : nbins) <= 0) return HJ_ERR_NBINS;
  or_state* s = or_create(z, dE, n, p, w, nbins, grid, seed, conv_mode);
  if (!s) return HJ_ERR_ARG;
  if (p->use_wakefield && (s->w.ctau <= 0 || p->pipe_radius <= 0)) {
    or_destroy(s);
    return HJ_ERR_WAKE_PARAM;
  }
  for (int64_t t = 0; t < p->n_turns; ++t) {
    int32_t rc = or_turn(s, draws ? draws + t * n : NULL);
    if (rc) { or_destroy(s); return rc; }
  }
  or_result(s, out);
  or_destroy(s);
  return HJ_OK;
}
