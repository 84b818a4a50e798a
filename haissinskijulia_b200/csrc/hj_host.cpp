// hj_host.cpp -- host-side set-up of a run: bin grid, wake and smoothing
// tables, FFT twiddles.  Compiled by the host C++ compiler with
// -ffp-contract=off so every rounding happens where the reference source
// puts it (these tables are constant over a run and computed once).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/haissinski_gpu.h"
#include "hj_host.h"

namespace {
const double kTwoPi = 6.283185307179586;    // Float64(2π)
const double kPi = 3.141592653589793;       // Float64(π)
const double kSpeedLight = 299792458.0;     // src/constants.jl:5
}  // namespace

extern "C" hj_status hj_wake_reference(const hj_params* p, hj_wake* out) {
  if (!p || !out) return HJ_ERR_ARG;
  const double kp = 3e1, Z0 = 120 * kPi, ctau = 4e-3;        // src/evolution.jl:276
  out->wake_factor = Z0 * kSpeedLight / (kPi * p->pipe_radius);  // :279
  const double a = 2 * kp / p->pipe_radius;
  out->wake_sqrt = std::sqrt(a > 0 ? a : 0.0);              // :280
  out->ctau = ctau;
  out->sin_coef = 0.0;
  out->population = 0.0;
  out->half_width_sigmas = 7.5;                              // :270
  out->delta_std = 0.15;                                     // src/wakefield.jl:204
  return HJ_OK;
}

extern "C" hj_status hj_wake_resonator(double Rs, double Q, double fr, double population,
                                       double half_width_sigmas, hj_wake* out) {
  if (!out || !(Rs > 0) || !(Q > 0.5) || !(fr > 0) || !(half_width_sigmas > 0))
    return HJ_ERR_ARG;
  // Broadband resonator wake W(τ) = 2αRs e^{-ατ}(cos ω̄τ - (α/ω̄) sin ω̄τ),
  // α = ω_r/2Q, ω̄ = sqrt(ω_r² - α²), written in the reference's variable
  // c = -cτ (c <= 0 behind the source).
  const double wr = kTwoPi * fr;
  const double alpha = wr / (2.0 * Q);
  const double wbar = std::sqrt(wr * wr - alpha * alpha);
  out->wake_factor = 2.0 * alpha * Rs;
  out->wake_sqrt = wbar / kSpeedLight;
  out->ctau = kSpeedLight / alpha;
  // cos(s c) with c = -cτ is even; sin(ω̄τ) = -sin(s c), so the -(α/ω̄) sin
  // term becomes +(α/ω̄) sin(s c).
  out->sin_coef = alpha / wbar;
  out->population = population;
  out->half_width_sigmas = half_width_sigmas;
  out->delta_std = 0.15;
  return HJ_OK;
}

namespace {
// The correctly rounded w·m/B (|m| < 2^53 / |w| headroom, B > 0) in double
// arithmetic: w·m = ph + pl exactly (fma), q0 = ph/B with its exact
// remainder, then the correction.  Returns false when the exact value lies
// within 2^-30 of a half-gap of the candidate (a rounding boundary); the
// caller then takes the quad-precision quotient, which such rare cases need.
bool rounded_ratio(double w, int64_t m, int64_t B, double* out) {
  const double md = (double)m, Bd = (double)B;
  const double ph = w * md;
  const double pl = std::fma(w, md, -ph);
  const double q0 = ph / Bd;
  const double r = std::fma(-q0, Bd, ph);            // exact: ph - q0·B
  const double e = (r + pl) / Bd;                    // x - q0, relative error ~2^-52
  const double q = q0 + e;
  const double d = e - (q - q0);                     // x - q (q - q0 exact)
  const double gap = d >= 0.0 ? std::nextafter(q, INFINITY) - q
                              : q - std::nextafter(q, -INFINITY);
  if (!(std::fabs(d) < 0.5 * gap * (1.0 - 0x1p-30))) return false;
  *out = q;
  return true;
}
}  // namespace

extern "C" hj_status hj_make_grid(double sigma_z0, double half_width_sigmas, int64_t nbins,
                                  double* centers, hj_grid* out) {
  if (!centers || !out) return HJ_ERR_ARG;
  if (nbins <= 0) return HJ_ERR_NBINS;
  double w = half_width_sigmas * sigma_z0;                   // src/evolution.jl:270
  if (w < 1e-9) w = 1e-6;                                    // :272
  // Julia's range(-w, w, length=B+1) and its midpoints hold the correctly
  // rounded values of w(2k-B)/B and w(2k+1-B)/B.
  const __float128 W = (__float128)w, Bq = (__float128)nbins;
  for (int64_t k = 0; k < nbins; ++k) {
    const int64_t m = 2 * k + 1 - nbins;
    double c;
    if (!rounded_ratio(w, m, nbins, &c)) c = (double)(W * (__float128)m / Bq);
    centers[k] = c;
  }
  out->nbins = nbins;
  out->edge_first = -w;
  out->edge_last = w;
  out->edge_step = (double)((W * 2) / Bq);
  out->centers = centers;
  return HJ_OK;
}

namespace hj {

// calculate_wake_function, src/wakefield.jl:115-118.
double host_wake_function(double c, const hj_wake& w) {
  if (c > 0.0) return 0.0;
  const double inv_ctau = 1.0 / w.ctau;
  double osc = std::cos(w.wake_sqrt * c);
  if (w.sin_coef != 0.0) osc = osc + w.sin_coef * std::sin(w.wake_sqrt * c);
  return w.wake_factor * std::exp(c * inv_ctau) * osc;
}

// delta, src/utils.jl:58-66.
double host_delta(double x, double sigma) {
  const double inv = 1.0 / (std::sqrt(kTwoPi) * sigma);
  const double f = -0.5 / (sigma * sigma);
  return inv * std::exp(x * x * f);
}

void host_wake_tables(const double* centers, int64_t B, const hj_wake& w, double* W,
                      double* lam) {
  for (int64_t i = 0; i < B; ++i) {
    W[i] = host_wake_function(centers[i], w);
    lam[i] = host_delta(centers[i], w.delta_std);
  }
}

// tw[k] = exp(-2πi k/P) in long double, rounded once.
// RF kick table of the fused pass: (V sin θm, V cos θm), θm = ϕs - 2π m / M,
// m = 0..M-1, in extended precision and rounded once.
// The extended-precision (sin θm, cos θm) of a phase are kept per (ϕs, M):
// bunches of a voltage scan share ϕs.
void host_rf_table(double V, double phi_s, int64_t M, double* tab_interleaved) {
  static std::mutex mu;
  static std::map<std::pair<uint64_t, int64_t>, std::vector<long double>> cache;
  uint64_t bits;
  std::memcpy(&bits, &phi_s, sizeof(bits));
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find({bits, M});
  if (it == cache.end()) {
    if (cache.size() >= 64) cache.clear();
    const long double kPiL = 3.141592653589793238462643383279502884L;
    std::vector<long double> sc(2 * (size_t)M);
    for (int64_t m = 0; m < M; ++m) {
      const long double a = (long double)phi_s - 2.0L * kPiL * (long double)m / (long double)M;
      sc[2 * m] = sinl(a);
      sc[2 * m + 1] = cosl(a);
    }
    it = cache.insert({{bits, M}, std::move(sc)}).first;
  }
  const std::vector<long double>& sc = it->second;
  for (int64_t m = 0; m < M; ++m) {
    tab_interleaved[2 * m] = (double)((long double)V * sc[2 * m]);
    tab_interleaved[2 * m + 1] = (double)((long double)V * sc[2 * m + 1]);
  }
}

// exp(-2πik/P), k = 0..P-1, interleaved (re, im), in extended precision and
// rounded once.  Tables are computed once per length and reused (a batch
// admits many bunches with the same bin count).
void host_twiddles(int64_t P, double* tw_interleaved) {
  static std::mutex mu;
  static std::map<int64_t, std::vector<double>> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(P);
  if (it == cache.end()) {
    std::vector<double> t(2 * (size_t)P);
    const long double kPiL = 3.141592653589793238462643383279502884L;
    for (int64_t k = 0; k < P; ++k) {
      const long double a = -2.0L * kPiL * (long double)k / (long double)P;
      t[2 * k] = (double)cosl(a);
      t[2 * k + 1] = (double)sinl(a);
    }
    it = cache.emplace(P, std::move(t)).first;
  }
  std::memcpy(tw_interleaved, it->second.data(), sizeof(double) * 2 * (size_t)P);
}

void host_normal_tables(NormalTables* t) {
  const long double kPiL = 3.141592653589793238462643383279502884L;
  const int n = kZigLayers;
  auto f = [](long double x) { return expl(-0.5L * x * x); };
  // area of the base layer: the rectangle [0, r) x [0, f(r)) and the tail
  auto area = [&](long double r) {
    return r * f(r) + sqrtl(kPiL / 2.0L) * erfcl(r / sqrtl(2.0L));
  };
  // Builds X_0 .. X_{n-1} from r; returns f(X_{n-1}) + v / X_{n-1} - 1, which
  // is 0 when layer n - 1 ends exactly at the top f = 1, positive when r is
  // too small (the layers are too tall and reach the top early).
  auto top = [&](long double r, long double* X) -> long double {
    const long double v = area(r);
    long double x = r;
    if (X) {
      X[0] = v / f(r);
      X[1] = r;
    }
    for (int i = 1; i < n - 1; ++i) {
      const long double y = f(x) + v / x;
      if (y >= 1.0L) return 1.0L;
      x = sqrtl(-2.0L * logl(y));
      if (X) X[i + 1] = x;
    }
    return f(x) + v / x - 1.0L;
  };
  long double lo = 3.0L, hi = 6.0L;
  for (int it = 0; it < 200; ++it) {
    const long double mid = 0.5L * (lo + hi);
    if (top(mid, nullptr) > 0.0L) lo = mid; else hi = mid;
  }
  std::vector<long double> X(n + 1, 0.0L);
  top(hi, X.data());
  X[n] = 0.0L;
  for (int i = 0; i < n; ++i) {
    t->xd[i][0] = (double)X[i];
    const long double K = ceill(ldexpl(X[i + 1] / X[i], 52));   // < 2^52: X_{i+1} < X_i
    t->xd[i][1] = (double)(1.0L + ldexpl(K, -52));              // exact in double
  }
  for (int i = 0; i <= n; ++i) t->f[i] = (double)f(X[i]);
  t->r = (double)X[1];
  t->v = (double)area(hi);
}

}  // namespace hj
