// hj_device.cuh -- device-side building blocks shared by the tracking kernels.
//
// Per-turn scalars follow src/evolution.jl:300-304 and the step functions
// src/rf_kick.jl:84-87, src/quantum_excitation.jl:58-71,
// src/synchrotron_radiation.jl:44-56 of the reference.  The random numbers
// are Philox-4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11), one counter per pair of particles, turned into
// Float64 normals by a double-precision Box-Muller transform.
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

// Double-precision Box-Muller transform of the four Philox words of a
// particle pair, with its logarithm and its sine and cosine evaluated from
// two 128-row tables (NormalTables, hj_host.h):
//   u1 = (2a + 1) 2^-53 with a the top 52 bits of (x1:x0), so u1 lies in
//     [2^-53, 1 - 2^-53] exactly; ln u1 by the table-driven method of
//     P. T. P. Tang (ACM TOMS 16(4), 1990): u1 = 2^e m, m in [1, 2),
//     ln m = -ln r_j + log1p(m r_j - 1) with r_j ≈ 1/(1 + (j + 1/2)/128) for
//     the top seven bits j of m (|m r_j - 1| < 2^-8), log1p by its Taylor
//     series through t^6 (truncation below 2e-18), e ln 2 with a two-part ln 2;
//   θ = 2π w, w in [0, 1) the top 52 bits of (x3:x2): θ = θ_k + t with
//     θ_k = 2π (k + 1/2)/128 for the top seven bits k of w, |t| <= π/128, sin t
//     and cos t - 1 by their Taylor series through t^7 and t^8 (truncation
//     below 1e-20), then angle addition with the tabulated sin θ_k, cos θ_k;
//   r = sqrt(-2 ln u1) (at most 8.57: the tails are cut only there), and the
//   normals r cos θ, r sin θ.
// About 36 FP64 operations per pair.
__device__ __forceinline__ void box_muller_f64(const uint32_t (&x)[4],
                                               const NormalTables* __restrict__ t,
                                               const double2* __restrict__ lr,
                                               const double2* __restrict__ sc, double out[2]) {
  // u1 = d - (1 - 2^-53), d = 1 + a 2^-52 in [1, 2): exact (Sterbenz)
  const double d = __hiloint2double(0x3FF00000 | (int)(x[1] >> 12),
                                    (int)((x[1] << 20) | (x[0] >> 12)));
  const double u1 = d - 0x1.fffffffffffffp-1;
  const int hi = __double2hiint(u1);
  const int e = (hi >> 20) - 1023;
  const int j = (hi >> 13) & 127;
  const double m = __hiloint2double((hi & 0x000FFFFF) | 0x3FF00000, __double2loint(u1));
  const double2 rj = lr[j];
  const double tt = fma(m, rj.x, -1.0);
  double q = -1.0 / 6.0;                               // log1p(t) = t q(t)
  q = fma(q, tt, 0.2);
  q = fma(q, tt, -0.25);
  q = fma(q, tt, 1.0 / 3.0);
  q = fma(q, tt, -0.5);
  q = fma(q, tt, 1.0);
  const double ed = (double)e;
  const double ln_u1 = fma(ed, t->ln2_hi, rj.y) + fma(ed, t->ln2_lo, tt * q);
  const double r = sqrt(-2.0 * ln_u1);
  // θ = 2π (w - (k + 1/2)/128) + θ_k, w = d2 - 1, d2 = 1 + b 2^-52; the
  // sector's centre 1 + (2k + 1)/256 is built from its bits
  const int h2 = (int)(0x3FF00000 | (x[3] >> 12));
  const double d2 = __hiloint2double(h2, (int)((x[3] << 20) | (x[2] >> 12)));
  const int k = (h2 >> 13) & 127;
  const double ck = __hiloint2double(0x3FF00000 | ((2 * k + 1) << 12), 0);
  const double xs = d2 - ck;                           // exact, |xs| <= 2^-8
  const double ang = fma(xs, t->twopi_hi, xs * t->twopi_lo);
  const double a2 = ang * ang;
  double ps = -1.9841269841269841e-04;                 // -1/7!
  ps = fma(ps, a2, 8.3333333333333333e-03);            // 1/5!
  ps = fma(ps, a2, -1.6666666666666667e-01);           // -1/3!
  const double sn = fma(ang * a2, ps, ang);
  double pc = 2.4801587301587302e-05;                  // 1/8!
  pc = fma(pc, a2, -1.3888888888888889e-03);           // -1/6!
  pc = fma(pc, a2, 4.1666666666666667e-02);            // 1/4!
  pc = fma(pc, a2, -0.5);
  const double cm1 = a2 * pc;
  const double2 skc = sc[k];
  const double sin_th = fma(skc.y, sn, fma(skc.x, cm1, skc.x));
  const double cos_th = fma(-skc.x, sn, fma(skc.y, cm1, skc.y));
  out[0] = r * cos_th;
  out[1] = r * sin_th;
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

// Two standard normals for particles 2p and 2p+1 at `turn` under the round
// keys of a seed: Philox-4x32-10 of the counter (p mod 2^32, p >> 32,
// turn mod 2^32, turn >> 32), then box_muller_f64.  lr, sc: the
// transform's logarithm and angle tables (shared or global memory).  Every
// (seed, pair, turn) has its own counter and key, so distinct seeds, pairs
// and turns never share a draw.
__device__ __forceinline__ void philox_normals2_rk(const PhiloxKeys& keys, int64_t turn,
                                                   int64_t p, const NormalTables* __restrict__ t,
                                                   const double2* __restrict__ lr,
                                                   const double2* __restrict__ sc,
                                                   double out[2]) {
  uint32_t c[4] = {(uint32_t)p, (uint32_t)((uint64_t)p >> 32), (uint32_t)turn,
                   (uint32_t)((uint64_t)turn >> 32)};
  philox4x32_10(c, keys);
  box_muller_f64(c, t, lr, sc, out);
}

}  // namespace hj
