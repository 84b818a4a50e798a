// hj_device.cuh -- device-side building blocks shared by the tracking kernels.
//
// Per-turn scalars follow src/evolution.jl:300-304 and the step functions
// src/rf_kick.jl:84-87, src/quantum_excitation.jl:58-71,
// src/synchrotron_radiation.jl:44-56 of the reference.  The random numbers
// are Philox-2x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11), one counter per pair of particles, turned into
// normals by the Box-Muller transform.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/haissinski_gpu.h"

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

// Philox-2x32 with 10 rounds: multiplier 0xD256D193, Weyl key increment
// 0x9E3779B9 (the published constants).
__host__ __device__ inline void philox2x32_10(uint32_t& c0, uint32_t& c1, uint32_t k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#if defined(__CUDA_ARCH__)
    const uint32_t hi = __umulhi(0xD256D193u, c0), lo = 0xD256D193u * c0;
#else
    const uint64_t pr = (uint64_t)0xD256D193u * c0;
    const uint32_t hi = (uint32_t)(pr >> 32), lo = (uint32_t)pr;
#endif
    c0 = hi ^ k ^ c1;
    c1 = lo;
    k += 0x9E3779B9u;
  }
}

// Philox-2x32-10 with its round keys given: rk[r] = key + r·0x9E3779B9.
__device__ __forceinline__ void philox2x32_10_rk(uint32_t& c0, uint32_t& c1,
                                                 const uint32_t (&rk)[10]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi = __umulhi(0xD256D193u, c0), lo = 0xD256D193u * c0;
    c0 = hi ^ rk[r] ^ c1;
    c1 = lo;
  }
}

// Box-Muller transform of one Philox output pair (see philox_normals2).
__device__ __forceinline__ void box_muller2(uint32_t x0, uint32_t x1, double out[2]) {
  const float kScale = 2.3283064365386963e-10f;  // 2^-32
  const float u1 = fmaf((float)x0, kScale, 0.5f * kScale);
  const float th = 6.2831853071795865f * fmaf((float)x1, kScale, -0.5f);
  const float m2l = fmaxf(-2.0f * __logf(u1), 1e-30f);
  const float rad = m2l * rsqrtf(m2l);                        // sqrt without a slow path
  float sn, cs;
  __sincosf(th, &sn, &cs);
  out[0] = (double)(rad * cs);
  out[1] = (double)(rad * sn);
}

// philox_normals2 with the round keys of (seed ^ seed >> 32) precomputed.
__device__ __forceinline__ void philox_normals2_rk(const uint32_t (&rk)[10], int64_t turn,
                                                   int64_t p, double out[2]) {
  uint32_t c0 = (uint32_t)p;
  uint32_t c1 = ((uint32_t)turn & 0xFFFFFFu) | ((uint32_t)((uint64_t)p >> 32) << 24);
  philox2x32_10_rk(c0, c1, rk);
  box_muller2(c0, c1, out);
}

// Two standard normals for particles 2p and 2p+1 at `turn`: Philox-2x32-10
// with key = (seed ^ seed >> 32) folded to 32 bits and counter
// (p mod 2^32, (turn mod 2^24) | (p >> 32) << 24), then the Box-Muller
// transform of its two uniforms u in (0,1): r = sqrt(-2 ln u1),
// θ = 2π (u2 - 1/2).  The transform runs in single precision on the
// special-function unit (__logf, __sincosf: absolute error below 2^-21 on
// these ranges); the normals are widened to double before they scale the
// Float64 kick, and their statistics are unaffected at the 1e-6 level.
__device__ __forceinline__ void philox_normals2(uint64_t seed, int64_t turn, int64_t p,
                                                double out[2]) {
  uint32_t c0 = (uint32_t)p;
  uint32_t c1 = ((uint32_t)turn & 0xFFFFFFu) | ((uint32_t)((uint64_t)p >> 32) << 24);
  philox2x32_10(c0, c1, (uint32_t)(seed ^ (seed >> 32)));
  box_muller2(c0, c1, out);
}

}  // namespace hj
