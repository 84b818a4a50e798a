// hj_device.cuh -- device-side building blocks shared by the tracking kernels.
//
// Per-turn scalars follow src/evolution.jl:300-304 and the step functions
// src/rf_kick.jl:84-87, src/quantum_excitation.jl:58-71,
// src/synchrotron_radiation.jl:44-56 of the reference.  The random numbers
// are Philox-4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11), one counter per pair of particles, turned into
// Float64 normals by a 2048-layer ziggurat (Marsaglia and Tsang, 2000).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/haissinski_gpu.h"
#include "hj_host.h"

namespace hj {

constexpr double kSpeedLight = 299792458.0;   // src/constants.jl:5
constexpr double kTwoPi = 6.283185307179586;  // Float64(2π)

// Scalars of one turn, all derived from the reference energy E0 of that
// turn (src/evolution.jl:300-304, src/quantum_excitation.jl:58-60,
// src/synchrotron_radiation.jl:44-45, drift coefficients :336-338).
struct TurnScalars {
  double E0;
  double gamma0;
  double beta0;
  double eta0;
  double sin_phis;
  double cos_phis;
  double k;           // rf_factor = 2π f_rf / (β0 c)
  double inv_k;
  double excitation;  // sqrt(1-(1-∂U/∂E)^2) σ_E0_initial
  double damping;     // 1 - ∂U/∂E
  double inv_b2E0;    // 1 / (β0² E0)
  double coeff0;      // 2π h η0 / (β0² E0)  (constant-η drift)
  double Kz;          // 2π h / (β0² E0 k): drift z -= Kz η_i ΔE
  double coeff0z;     // coeff0 / k
  int32_t drift_ok;   // apply_phase_advance! runs (β0 > 0, E0 != 0, k != 0)
  int32_t _pad;
};

// Device-resident state carried from one turn to the next.  The particle
// pass of turn t reads `cur` (scalars of turn t) and owes turn t-1's wake
// kick and E0 re-centring when `pending` is set.
struct TurnState {
  TurnScalars cur;
  double pending_mean;   // mean ΔE of the previous turn, still to subtract
  int32_t pending;       // 1: previous turn's kick + re-centring not yet applied
  int32_t status;        // sticky HJ_ERR_* bits raised on the device
  int64_t turn;          // 1-based index of the turn the next pass runs
  double last_sigma_z;   // σ_z used for the wake current of the last turn
  double last_current;   // wake current of the last turn
  double last_mean;      // E0 change of the last turn
  double last_sum_kick;  // Σ_i lerp(pot, z_i) of the last turn
  double last_n_in;      // particles inside the bin range, last turn
  int64_t turns_left;    // turns still to run (batches); a plain bunch never runs out
  double last_mean_z;    // mean z after the last turn's drift (centres the pass's
                         // shared-memory window of the kick table)
};

__host__ __device__ inline TurnScalars make_turn_scalars(double E0, const hj_params& p,
                                                         double sigma_E0_initial) {
  TurnScalars s;
  s.E0 = E0;
  s.gamma0 = E0 / p.mass;
  double b2 = 1.0 - 1.0 / (s.gamma0 * s.gamma0);
  s.beta0 = sqrt(b2 > 0.0 ? b2 : 0.0);
  s.eta0 = p.alpha_c - (1.0 / (s.gamma0 * s.gamma0));
  s.sin_phis = sin(p.phi_s);
  s.cos_phis = cos(p.phi_s);
  s.k = (s.beta0 <= 0.0) ? (1.0 / 0.0) : p.freq_rf * kTwoPi / (s.beta0 * kSpeedLight);
  s.inv_k = 1.0 / s.k;
  double t = E0 / 1e9;
  double dU = 4 * 8.85e-5 * (t * t * t) / p.radius;
  double om = 1 - dU;
  s.excitation = sqrt(1 - om * om) * sigma_E0_initial;
  s.damping = 1 - dU;
  double b2E0 = s.beta0 * s.beta0 * E0;
  s.inv_b2E0 = 1.0 / b2E0;
  s.coeff0 = (kTwoPi * (double)p.harmonic * s.eta0 / b2E0);
  s.Kz = kTwoPi * (double)p.harmonic * s.inv_b2E0 * s.inv_k;
  s.coeff0z = s.coeff0 * s.inv_k;
  s.drift_ok = !(s.beta0 <= 0 || E0 == 0 || s.k == 0);
  s._pad = 0;
  return s;
}

// compute_global_std from single-pass sums (src/utils.jl:593-605).
__host__ __device__ inline double global_std_of_sums(double s, double s2, int64_t n) {
  if (n <= 1) return 0.0;
  const double nd = (double)n;
  const double mean = s / nd;
  const double var = (s2 / nd) - (mean * mean);
  double v = var * nd / (double)(n - 1);
  if (!(v > 0.0)) v = (v != v) ? v : 0.0;
  return sqrt(v);
}

// ------------------------------------------------------------------ Philox

// Philox-4x32-10 (Salmon, Moraes, Dror & Shaw, SC'11): multipliers
// 0xD2511F53 and 0xCD9E8D57, Weyl key increments 0x9E3779B9 and 0xBB67AE85
// (the published constants); a 128-bit counter and a 64-bit key.
constexpr uint32_t kPhiloxM0 = 0xD2511F53u, kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u, kPhiloxW1 = 0xBB67AE85u;

// Round keys of a 64-bit key: rk[r] = k0 + r·W0, rk[10 + r] = k1 + r·W1.
struct PhiloxKeys {
  uint32_t rk[20];
};

__host__ __device__ inline PhiloxKeys philox_keys(uint64_t key) {
  PhiloxKeys k;
  for (int r = 0; r < 10; ++r) {
    k.rk[r] = (uint32_t)key + (uint32_t)r * kPhiloxW0;
    k.rk[10 + r] = (uint32_t)(key >> 32) + (uint32_t)r * kPhiloxW1;
  }
  return k;
}

__host__ __device__ inline void philox4x32_10(uint32_t (&c)[4], const PhiloxKeys& k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#if defined(__CUDA_ARCH__)
    const uint32_t hi0 = __umulhi(kPhiloxM0, c[0]), lo0 = kPhiloxM0 * c[0];
    const uint32_t hi1 = __umulhi(kPhiloxM1, c[2]), lo1 = kPhiloxM1 * c[2];
#else
    const uint64_t p0 = (uint64_t)kPhiloxM0 * c[0], p1 = (uint64_t)kPhiloxM1 * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    const uint32_t n0 = hi1 ^ c[1] ^ k.rk[r], n2 = hi0 ^ c[3] ^ k.rk[10 + r];
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
  }
}

// ------------------------------------------------------------ normals

// Float64 standard normals by the 2048-layer ziggurat of NormalTables
// (hj_host.h; Marsaglia and Tsang, J. Stat. Softw. 5(8), 2000), the algorithm
// family of Julia's randn.  One normal takes 64 random bits (hi:lo): layer
// i = hi >> 21, sign = bit 20 of hi, and a 52-bit fraction m = (hi mod 2^20):lo,
// U = m 2^-52.  The candidate is x = U X_i.
//
// Fast path (about 99.8 % of draws): 1 + m 2^-52 < D_i, i.e. x < X_{i+1},
// where the candidate lies under the curve at any height of the layer; x is
// returned at once: one table row and one FMA, exact to one rounding.
//
// Slow path (zig_slow): the tail of layer 0 beyond r, or the wedge of layer
// i >= 1 between x = X_{i+1} and X_i, needs more random bits.  They come from
// the retry draws of the particle: Philox-4x32-10 under the same key with the
// counter (p mod 2^32, p >> 32, turn mod 2^32, (turn >> 32) | (2a - 1 + h) << 24)
// for attempt a = 1, 2, ... and the particle's half h of its pair, so every
// normal is a fixed function of (seed, particle, turn) whichever thread, and
// in whichever order, computes it (turns below 2^56).
//   wedge: y = f(X_i) + u (f(X_{i+1}) - f(X_i)) with u from words 0-1; accept
//     x when y < exp(-x²/2), else take a new (layer, sign, fraction) from
//     words 2-3 and test it again from the start;
//   tail: u1, u2 in (0, 1) from words 0-1 and 2-3, a = -ln(u1) / r,
//     b = -ln(u2); accept r + a when 2b > a² (Marsaglia's tail method),
//     else the next attempt.
// The loop stops after 127 attempts (each rejects with probability below
// 1/2, so it never gets there) with the last candidate.

// The fast path: true and x = ±U X_i when the draw (hi:lo) is accepted; x is
// the candidate either way.  zt: the table's (X_i, D_i) rows (shared or
// global memory).
__device__ __forceinline__ bool zig_fast(uint32_t hi, uint32_t lo,
                                         const double2* __restrict__ zt, double& x) {
  const double2 t = zt[hi >> 21];
  const double d = __hiloint2double(0x3FF00000 | (int)(hi & 0xFFFFFu), (int)lo);  // 1 + U
  const double xs = __hiloint2double(__double2hiint(t.x) ^ (int)((hi << 11) & 0x80000000u),
                                     __double2loint(t.x));                          // ±X_i
  x = fma(d, xs, -xs);                                                          // ±U X_i
  return d < t.y;
}

// The 52-bit fraction (hi mod 2^20):lo as an exact double.
__device__ __forceinline__ double zig_fraction(uint32_t hi, uint32_t lo) {
  return (double)(((unsigned long long)(hi & 0xFFFFFu) << 32) | lo);
}

// The slow path for the normal of particle 2p + h at `turn` under `seed`
// whose first draw (hi:lo) failed the fast test.  Out of line, with scalar
// arguments only: the hot loops that may call it keep their registers.
static __device__ __noinline__ double zig_slow(uint64_t seed, int64_t turn, int64_t p, int h,
                                               uint32_t hi, uint32_t lo,
                                               const NormalTables* __restrict__ t) {
  const PhiloxKeys keys = philox_keys(seed);
  int i = (int)(hi >> 21);
  bool neg = (hi >> 20) & 1u;
  double d = __hiloint2double(0x3FF00000 | (int)(hi & 0xFFFFFu), (int)lo);
  const double r = __ldg(&t->r);
  double x = 0.0;
  for (int a = 1; a <= 127; ++a) {
    uint32_t c[4] = {(uint32_t)p, (uint32_t)((uint64_t)p >> 32), (uint32_t)turn,
                     (uint32_t)((uint64_t)turn >> 32) | ((uint32_t)(2 * a - 1 + h) << 24)};
    philox4x32_10(c, keys);
    if (i == 0) {   // tail beyond r
      const double u1 = __dmul_rn(__dadd_rn(zig_fraction(c[1], c[0]), 0.5), 0x1p-52);
      const double u2 = __dmul_rn(__dadd_rn(zig_fraction(c[3], c[2]), 0.5), 0x1p-52);
      const double ta = __ddiv_rn(-log(u1), r);
      const double tb = -log(u2);
      x = __dadd_rn(r, ta);
      if (__dadd_rn(tb, tb) > __dmul_rn(ta, ta)) break;
      continue;
    }
    x = __dmul_rn(__dsub_rn(d, 1.0), __ldg(&t->xd[i][0]));   // in [X_{i+1}, X_i)
    const double fi = __ldg(&t->f[i]), fi1 = __ldg(&t->f[i + 1]);
    const double u = __dmul_rn(zig_fraction(c[1], c[0]), 0x1p-52);
    const double y = __dadd_rn(fi, __dmul_rn(u, __dsub_rn(fi1, fi)));
    if (y < exp(__dmul_rn(__dmul_rn(x, x), -0.5))) break;
    // rejected: a new draw from words 2-3, tested from the start
    i = (int)(c[3] >> 21);
    neg = (c[3] >> 20) & 1u;
    d = __hiloint2double(0x3FF00000 | (int)(c[3] & 0xFFFFFu), (int)c[2]);
    x = __dmul_rn(__dsub_rn(d, 1.0), __ldg(&t->xd[i][0]));
    if (d < __ldg(&t->xd[i][1])) break;
  }
  return neg ? -x : x;
}

// Single-precision Box-Muller transform of words 0 and 1 (the opt-in fast
// normals of the fused pass): u1 = (x0 + 1/2) 2^-32, θ = 2π ((x1 + 1/2)
// 2^-32 - 1/2), on the special-function unit (__logf, __sincosf), widened to
// double.  24-bit uniforms: |normal| <= 6.0 (the tails beyond are cut),
// relative resolution about 1e-7.
__device__ __forceinline__ void box_muller_f32(uint32_t x0, uint32_t x1, double out[2]) {
  const float kScale = 2.3283064365386963e-10f;         // 2^-32
  const float u1 = fmaf((float)x0, kScale, 0.5f * kScale);
  const float th = 6.2831853071795865f * fmaf((float)x1, kScale, -0.5f);
  const float m2l = fmaxf(-2.0f * __logf(u1), 1e-30f);
  const float rad = m2l * rsqrtf(m2l);
  float sn, cs;
  __sincosf(th, &sn, &cs);
  out[0] = (double)(rad * cs);
  out[1] = (double)(rad * sn);
}

// philox_normals2_rk with the single-precision transform of words 0 and 1.
__device__ __forceinline__ void philox_normals2_fast(const PhiloxKeys& keys, int64_t turn,
                                                     int64_t p, double out[2]) {
  uint32_t c[4] = {(uint32_t)p, (uint32_t)((uint64_t)p >> 32), (uint32_t)turn,
                   (uint32_t)((uint64_t)turn >> 32)};
  philox4x32_10(c, keys);
  box_muller_f32(c[0], c[1], out);
}

// Two standard normals for particles 2p and 2p+1 at `turn` under `seed`
// (keys: its round keys): Philox-4x32-10 of the counter (p mod 2^32, p >> 32,
// turn mod 2^32, turn >> 32); words 1:0 make the first normal and 3:2 the
// second, each by the ziggurat (fast path, else zig_slow).  zt: the table's
// (X_i, D_i) rows (shared or global memory); t: the whole table (global).
// Every (seed, pair, turn) has its own counter and key, so distinct seeds,
// pairs and turns never share a draw.
__device__ __forceinline__ void philox_normals2_rk(uint64_t seed, const PhiloxKeys& keys,
                                                   int64_t turn, int64_t p,
                                                   const NormalTables* __restrict__ t,
                                                   const double2* __restrict__ zt,
                                                   double out[2]) {
  uint32_t c[4] = {(uint32_t)p, (uint32_t)((uint64_t)p >> 32), (uint32_t)turn,
                   (uint32_t)((uint64_t)turn >> 32)};
  philox4x32_10(c, keys);
  if (!zig_fast(c[1], c[0], zt, out[0])) out[0] = zig_slow(seed, turn, p, 0, c[1], c[0], t);
  if (!zig_fast(c[3], c[2], zt, out[1])) out[1] = zig_slow(seed, turn, p, 1, c[3], c[2], t);
}

}  // namespace hj
