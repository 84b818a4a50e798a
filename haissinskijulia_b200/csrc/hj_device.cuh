// hj_device.cuh -- device-side building blocks shared by the tracking kernels.
//
// Per-turn scalars follow src/evolution.jl:300-304 and the step functions
// src/rf_kick.jl:84-87, src/quantum_excitation.jl:58-71,
// src/synchrotron_radiation.jl:44-56 of the reference.  The random numbers
// are Philox-4x32-10 (Salmon, Moraes, Dror & Shaw, "Parallel random numbers:
// as easy as 1, 2, 3", SC'11) turned into normals by the Box-Muller
// transform.
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
  s.drift_ok = !(s.beta0 <= 0 || E0 == 0 || s.k == 0);
  s._pad = 0;
  return s;
}

// ------------------------------------------------------------------ Philox

struct U32x4 {
  uint32_t x, y, z, w;
};

// Philox-4x32 with 10 rounds: multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key
// increments 0x9E3779B9 / 0xBB67AE85 (the published constants).
__host__ __device__ inline U32x4 philox4x32_10(U32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#if defined(__CUDA_ARCH__)
    uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    U32x4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// Four standard normals for particles 4q..4q+3 at `turn`: counter
// (q_lo, q_hi, turn_lo, turn_hi), key (seed_lo, seed_hi); Box-Muller on
// (x,y) and (z,w) with uniforms u in (0,1): r = sqrt(-2 ln u1),
// θ = 2π (u2 - 1/2) in (-π, π).  The transform runs in single precision on the
// special-function unit (__logf, __sincosf: absolute error below 2^-21 on
// these ranges), and the normals are widened to double before they scale the
// Float64 kick; the statistical quality of the variates is unaffected at the
// 1e-6 level.
__device__ __forceinline__ void philox_normals4(uint64_t seed, int64_t turn, int64_t q,
                                                double out[4]) {
  U32x4 c{(uint32_t)q, (uint32_t)((uint64_t)q >> 32), (uint32_t)turn,
          (uint32_t)((uint64_t)turn >> 32)};
  U32x4 r = philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const float kScale = 2.3283064365386963e-10f;  // 2^-32
  const float kTwoPiF = 6.2831853071795865f;
  const float u1 = fmaf((float)r.x, kScale, 0.5f * kScale);
  const float u3 = fmaf((float)r.z, kScale, 0.5f * kScale);
  const float ta = kTwoPiF * fmaf((float)r.y, kScale, -0.5f);
  const float tb = kTwoPiF * fmaf((float)r.w, kScale, -0.5f);
  const float ra = sqrtf(-2.0f * __logf(u1));
  const float rb = sqrtf(-2.0f * __logf(u3));
  float sa, ca, sb, cb;
  __sincosf(ta, &sa, &ca);
  __sincosf(tb, &sb, &cb);
  out[0] = (double)(ra * ca);
  out[1] = (double)(ra * sa);
  out[2] = (double)(rb * cb);
  out[3] = (double)(rb * sb);
}

}  // namespace hj
