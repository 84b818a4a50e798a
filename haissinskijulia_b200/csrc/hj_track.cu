// hj_track.cu -- particle-side kernels of the tracking loop (sm_100a, FP64).
//
// One fused pass per turn replaces the reference's chain of per-particle
// loops in longitudinal_evolve! (src/evolution.jl:307-451):
//   [previous turn]  wake kick  dE -= lerp(pot, z)      src/wakefield.jl:22-105, :342-344
//                    E0 re-centring  dE -= mean         src/evolution.jl:434
//   [this turn]      RF kick                            src/rf_kick.jl:84-87
//                    quantum excitation                 src/quantum_excitation.jl:58-71
//                    SR damping                         src/synchrotron_radiation.jl:44-56
//                    drift (phase advance)              src/evolution.jl:331-344 / :143-167
//                    histogram of z                     src/utils.jl:384-398
//                    Σz, Σz² (σ_z, src/utils.jl:576-580), Σ(ΔE - ΔE_start) (src/evolution.jl:408-411)
//                    CIC deposit of the interpolation weights, so that the bins step
//                    can form Σ_i lerp(pot, z_i) = Σ_k H[k] pot[k] for the E0 update
//                    without another pass over the particles.
// z is unchanged between the drift of turn t and the wake kick of turn t, so
// the kick is applied at the start of the next pass from the same z.
//
// Each thread owns four consecutive particles and moves them with one
// 32-byte load/store per array (ld.global.v4.f64), so a warp touches 1 KB of
// contiguous HBM per array per iteration; the next quad is loaded while the
// current one is computed.  Histograms are privatised in shared memory per
// block and written out as per-block partials, merged by k_hist_reduce.
//
// Per-particle arithmetic of the fused pass (the single-step kernels further
// down keep the reference's exact operation order instead):
//   * RF kick: V(sin(ϕs - x) - sin ϕs) = V sin ϕs (cos x - 1) - V cos ϕs sin x with
//     x = z k, sin x and cos x - 1 from their Taylor series through x^15 and
//     x^16 when |x| <= 0.5 (truncation error < 3e-20); the general sin() path
//     otherwise.  This avoids the cancellation of sin(ϕ) - sin ϕs.
//   * 1/γ² of the drift: rcp.approx.ftz.f64 refined by two Newton steps
//     (relative error at double rounding level).
//   * reciprocals of k, mass and β0²E0 are precomputed per turn.
#include "hj_internal.h"

namespace hj {
namespace {

// Run- and turn-constants of the fused pass.
struct FusedConst {
  double Vs, Vc;            // V sin ϕs, V cos ϕs
  double V, phi_s, sin_phis;
  double k, inv_k;
  double excitation, damping;
  double gamma0, inv_mass, alpha_c, K;   // K = 2π h / (β0² E0)
  double coeff0;            // K η0 (constant-η drift)
  int drift_ok, update_eta, sr;
};

// Constants of the single-step phase-advance kernel (reference operation order).
struct StepConst {
  double phi_s, k, inv_k, gamma0, inv_mass, alpha_c, two_pi_h, inv_b2E0, coeff0;
  int drift_ok, update_eta;
};

struct GridConst {
  int B;
  double e0, eN, inv_e, c1, cB, inv_c;
};

__device__ __forceinline__ int cic_hi(int B) { return B >= 2 ? B - 2 : 0; }

// Packed CIC accumulator V = count·2^44 + Σ w·2^24 per cell (a block
// deposits at most kMaxBlockParticles particles per turn, so neither field
// overflows).  In shared memory V lives as two 32-bit words: 64-bit shared
// atomics are several times slower than 32-bit ones on this GPU, so a deposit
// adds q = w·2^24 to the low word with an atomic that returns the old value,
// and 2^12 (one count) plus the carry out of the low word to the high word.
// Every carry is counted exactly once, so the final words are exact.
constexpr int kCicWeightBits = 24;
constexpr int kCicSumBits = 44;
constexpr unsigned long long kCicSumMask = (1ull << kCicSumBits) - 1ull;

__device__ __forceinline__ void ld4(const double* p, double v[4]) {
  asm("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
      : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
      : "l"(p));
}

__device__ __forceinline__ void st4(double* p, const double v[4]) {
  asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]),
               "d"(v[2]), "d"(v[3])
               : "memory");
}

__device__ __forceinline__ double rcp_approx(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  return r;
}

// Interpolation cell of z on the bin centers (src/wakefield.jl:64-78), 0-based:
// idx = clamp(floor(u), 0, B-2), w = u - floor(u), u = (clamp(z,c1,cB)-c1)/Δc.
// floor() is a round-down conversion to int (exact: u is within [0, B-1]).
// The deposit of turn t and the kick applied in turn t+1 call this with the
// same z, so they agree exactly.
__device__ __forceinline__ void cic_cell(double z, const GridConst& g, int& idx, double& w) {
  const double cl = fmin(fmax(z, g.c1), g.cB);
  const double u = __dmul_rn(__dsub_rn(cl, g.c1), g.inv_c);
  const int i = __double2int_rd(u);
  w = __dsub_rn(u, (double)i);
  idx = min(max(i, 0), cic_hi(g.B));
}

// Kick of the fused pass: lerp from the (pot[k], pot[k+1] - pot[k]) table.
__device__ __forceinline__ double wake_kick(double z, const GridConst& g,
                                            const double2* __restrict__ potd) {
  int idx;
  double w;
  cic_cell(z, g, idx, w);
  const double2 pd = __ldg(potd + idx);
  return fma(w, pd.y, pd.x);
}

// Kick of the single-step kernel in the reference's form v1 (1 - w) + v2 w
// (src/wakefield.jl:94-102).
__device__ __forceinline__ double wake_kick_ref(double z, const GridConst& g,
                                                const double* __restrict__ pot) {
  if (g.B < 2) return __ldg(pot);
  int idx;
  double w;
  cic_cell(z, g, idx, w);
  return __dadd_rn(__dmul_rn(__ldg(pot + idx), __dsub_rn(1.0, w)),
                   __dmul_rn(__ldg(pot + idx + 1), w));
}

// Histogram bin of z (src/utils.jl:387-397), 0-based: clamp(floor((z-e0)/Δe), 0, B-1),
// with (z - e0) and the product rounded exactly as the reference rounds them.
__device__ __forceinline__ int ngp_bin(double z, const GridConst& g, bool& in) {
  in = (z >= g.e0) & (z <= g.eN);
  const int j = __double2int_rd(__dmul_rn(__dsub_rn(z, g.e0), g.inv_e));
  return min(max(j, 0), g.B - 1);
}

// V(sin(ϕs - x) - sin ϕs) for |x| > 0.5, as the reference forms it.
__device__ __noinline__ double rf_kick_general(double z, double k, double phi_s,
                                               double sin_phis, double V) {
  return V * (sin(fma(-z, k, phi_s)) - sin_phis);
}

// V(sin(ϕs - x) - sin ϕs), x = z k, by angle addition and Taylor series.
__device__ __forceinline__ double rf_kick_term(double z, const FusedConst& c) {
  const double x = z * c.k;
  if (!(fabs(x) <= 0.5)) return rf_kick_general(z, c.k, c.phi_s, c.sin_phis, c.V);
  const double t = x * x;
  // sin x = x + x^3 P(t): coefficients (-1)^n / (2n+1)!, n = 1..7
  double p = -7.647163731819816e-13;          // -1/15!
  p = fma(t, p, 1.6059043836821613e-10);      // +1/13!
  p = fma(t, p, -2.505210838544172e-08);      // -1/11!
  p = fma(t, p, 2.7557319223985893e-06);      // +1/9!
  p = fma(t, p, -1.984126984126984e-04);      // -1/7!
  p = fma(t, p, 8.333333333333333e-03);       // +1/5!
  p = fma(t, p, -1.6666666666666666e-01);     // -1/3!
  const double sn = fma(t * x, p, x);
  // cos x - 1 = t Q(t): coefficients (-1)^n / (2n)!, n = 1..8
  double q = 4.779477332387385e-14;           // +1/16!
  q = fma(t, q, -1.1470745597729725e-11);     // -1/14!
  q = fma(t, q, 2.08767569878681e-09);        // +1/12!
  q = fma(t, q, -2.755731922398589e-07);      // -1/10!
  q = fma(t, q, 2.48015873015873e-05);        // +1/8!
  q = fma(t, q, -1.388888888888889e-03);      // -1/6!
  q = fma(t, q, 4.1666666666666664e-02);      // +1/4!
  q = fma(t, q, -0.5);                        // -1/2!
  const double cm1 = t * q;
  return fma(c.Vs, cm1, -c.Vc * sn);
}

// RF kick, QE, SR and drift of one particle for one turn (fused-pass arithmetic).
__device__ __forceinline__ void turn_particle(double& z, double& e, double r, bool qe,
                                              const FusedConst& c) {
  e = e + rf_kick_term(z, c);
  if (qe) e = fma(c.excitation, r, e);
  if (c.sr) e = e * c.damping;
  double coeff;
  if (c.update_eta) {
    const double gp = fma(e, c.inv_mass, c.gamma0);   // γ0 + ΔE/m
    const double g2 = gp * gp;
    double ri = rcp_approx(g2);
    ri = fma(ri, fma(-g2, ri, 1.0), ri);
    ri = fma(ri, fma(-g2, ri, 1.0), ri);
    coeff = c.K * (c.alpha_c - ri);                    // 2π h η_i / (β0² E0)
  } else {
    if (!c.drift_ok) return;                           // apply_phase_advance! skip
    coeff = c.coeff0;
  }
  double ph = fma(-z, c.k, c.phi_s);                   // ϕ = -(z k - ϕs)
  ph = fma(coeff, e, ph);
  z = (c.phi_s - ph) * c.inv_k;                        // z = (-ϕ + ϕs)/k
}

template <bool WAKE>
__device__ __forceinline__ void pass_particle(double& z, double& e, double r, bool qe,
                                              const FusedConst& c, const GridConst& g,
                                              bool pending, bool upd_E0, double pmean,
                                              const double2* __restrict__ potd, double& acc_z,
                                              double& acc_z2, double& acc_d, uint32_t& n_in,
                                              uint32_t* s_cnt, uint32_t* s_lo, uint32_t* s_hi) {
  if (pending) {
    if (WAKE) e = e - wake_kick(z, g, potd);
    if (upd_E0) e = e - pmean;
  }
  const double e_start = e;
  turn_particle(z, e, r, qe, c);
  if (upd_E0) acc_d += e - e_start;
  if (WAKE) {
    acc_z += z;
    acc_z2 = fma(z, z, acc_z2);
    bool in;
    const int j = ngp_bin(z, g, in);
    if (in) {
      atomicAdd(&s_cnt[j], 1u);
      ++n_in;
    }
    int idx;
    double w;
    cic_cell(z, g, idx, w);
    const uint32_t q = __double2uint_rn(w * 16777216.0);
    const uint32_t old = atomicAdd(&s_lo[idx], q);
    atomicAdd(&s_hi[idx], (1u << (kCicSumBits - 32)) + (old + q < old ? 1u : 0u));
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-order block reduction of four accumulators into out[0..3] (thread 0).
template <int THREADS>
__device__ __forceinline__ void block_sum4(double a0, double a1, double a2, double a3,
                                           double* out) {
  __shared__ double red[THREADS / 32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  a0 = warp_sum(a0);
  a1 = warp_sum(a1);
  a2 = warp_sum(a2);
  a3 = warp_sum(a3);
  if (lane == 0) {
    red[warp][0] = a0;
    red[warp][1] = a1;
    red[warp][2] = a2;
    red[warp][3] = a3;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][threadIdx.x];
    out[threadIdx.x] = s;
  }
}

// Particle loads/stores of PPT = 2 or 4 consecutive particles.
template <int PPT>
__device__ __forceinline__ void ldp(const double* p, double v[PPT]) {
  if (PPT == 4) {
    asm("ld.global.v4.f64 {%0,%1,%2,%3}, [%4];"
        : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
        : "l"(p));
  } else {
    asm("ld.global.v2.f64 {%0,%1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "l"(p));
  }
}

template <int PPT>
__device__ __forceinline__ void stp(double* p, const double v[PPT]) {
  if (PPT == 4) {
    asm volatile("st.global.v4.f64 [%0], {%1,%2,%3,%4};" ::"l"(p), "d"(v[0]), "d"(v[1]),
                 "d"(v[2]), "d"(v[3])
                 : "memory");
  } else {
    asm volatile("st.global.v2.f64 [%0], {%1,%2};" ::"l"(p), "d"(v[0]), "d"(v[1]) : "memory");
  }
}

// Normals of particles PPT*g .. PPT*g+PPT-1 (the Philox quad of particle i is
// i/4, its lane i%4; a pair uses half of its quad).
template <int PPT>
__device__ __forceinline__ void group_normals(uint64_t seed, int64_t turn, int64_t g,
                                              double r[PPT]) {
  double q4[4];
  philox_normals4(seed, turn, PPT == 4 ? g : (g >> 1), q4);
  if (PPT == 4) {
#pragma unroll
    for (int j = 0; j < 4; ++j) r[j] = q4[j];
  } else {
    const int h = (int)(g & 1) * 2;
    r[0] = q4[h];
    r[1] = q4[h + 1];
  }
}

// One turn over the bunch.  PPT particles per thread per iteration (4 with the
// next group prefetched in registers, or 2 with twice the threads per SM).
template <bool WAKE, int QE, int PPT, int THREADS>
__global__ void __launch_bounds__(THREADS, 1) k_track_pass(PassArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem_raw);
  uint32_t* s_lo = s_cnt + (WAKE ? a.B : 0);
  uint32_t* s_hi = s_lo + (WAKE ? a.B : 0);

  TurnState* ts = a.ts;
  const TurnScalars sc = ts->cur;
  const bool pending = ts->pending != 0;
  const double pmean = ts->pending_mean;
  const int64_t turn = ts->turn;
  const bool upd_E0 = a.update_E0 != 0;

  FusedConst c;
  c.V = a.V;
  c.phi_s = a.phi_s;
  c.sin_phis = sc.sin_phis;
  c.Vs = a.V * sc.sin_phis;
  c.Vc = a.V * sc.cos_phis;
  c.k = sc.k;
  c.inv_k = sc.inv_k;
  c.excitation = sc.excitation;
  c.damping = sc.damping;
  c.gamma0 = sc.gamma0;
  c.inv_mass = a.inv_mass;
  c.alpha_c = a.alpha_c;
  c.K = a.two_pi_h * sc.inv_b2E0;
  c.coeff0 = sc.coeff0;
  c.drift_ok = sc.drift_ok;
  c.update_eta = a.update_eta;
  c.sr = a.sr;
  GridConst g{a.B, a.e0, a.eN, a.inv_estep, a.c1, a.cB, a.inv_cstep};

  const double* drow = nullptr;
  if (QE == QE_DRAWS) {
    int64_t row = turn - a.draws_first_turn;
    if (row >= 0 && row < a.draws_turns) {
      drow = a.draws + row * a.n;
    } else if (blockIdx.x == 0 && threadIdx.x == 0) {
      atomicOr(&ts->status, 1 << HJ_ERR_ARG);
    }
  }

  if (WAKE) {
    for (int i = threadIdx.x; i < a.B; i += THREADS) {
      s_cnt[i] = 0u;
      s_lo[i] = 0u;
      s_hi[i] = 0u;
    }
    // zero the merged histograms k_hist_reduce accumulates into this turn
    const int gstride = gridDim.x * THREADS;
    for (int i = blockIdx.x * THREADS + threadIdx.x; i < 3 * a.B; i += gstride)
      a.hist_out[i] = 0ull;
    __syncthreads();
  }

  double acc_z = 0.0, acc_z2 = 0.0, acc_d = 0.0;
  uint32_t n_in = 0;
  const double2* __restrict__ potd = a.potd;
  const int64_t ng = a.n / PPT;
  const int64_t stride = (int64_t)gridDim.x * THREADS;
  int64_t q = (int64_t)blockIdx.x * THREADS + threadIdx.x;
  constexpr bool kPrefetch = (PPT == 4);
  double zn[PPT], en[PPT];
  if (kPrefetch && q < ng) {
    ldp<PPT>(a.z + PPT * q, zn);
    ldp<PPT>(a.dE + PPT * q, en);
  }
  for (; q < ng; q += stride) {
    double zz[PPT], ee[PPT], rr[PPT];
    if (kPrefetch) {
#pragma unroll
      for (int j = 0; j < PPT; ++j) {
        zz[j] = zn[j];
        ee[j] = en[j];
      }
      const int64_t qn = q + stride;
      if (qn < ng) {  // the next group streams in while this one is computed
        ldp<PPT>(a.z + PPT * qn, zn);
        ldp<PPT>(a.dE + PPT * qn, en);
      }
    } else {
      ldp<PPT>(a.z + PPT * q, zz);
      ldp<PPT>(a.dE + PPT * q, ee);
    }
#pragma unroll
    for (int j = 0; j < PPT; ++j) rr[j] = 0.0;
    if (QE == QE_PHILOX) {
      group_normals<PPT>(a.seed, turn, q, rr);
    } else if (QE == QE_DRAWS) {
      if (drow) {
#pragma unroll
        for (int j = 0; j < PPT; ++j) rr[j] = __ldg(drow + PPT * q + j);
      }
    }
#pragma unroll
    for (int j = 0; j < PPT; ++j)
      pass_particle<WAKE>(zz[j], ee[j], rr[j], QE != QE_OFF, c, g, pending, upd_E0, pmean,
                          potd, acc_z, acc_z2, acc_d, n_in, s_cnt, s_lo, s_hi);
    stp<PPT>(a.z + PPT * q, zz);
    stp<PPT>(a.dE + PPT * q, ee);
  }
  // Tail of n % PPT particles: the first threads of block 0, scalar.
  if (blockIdx.x == 0 && threadIdx.x < (int)(a.n % PPT)) {
    const int64_t i = ng * PPT + threadIdx.x;
    double rr4[4] = {0.0, 0.0, 0.0, 0.0};
    if (QE == QE_PHILOX) philox_normals4(a.seed, turn, i >> 2, rr4);
    double r = rr4[i & 3];
    if (QE == QE_DRAWS && drow) r = __ldg(drow + i);
    double z = a.z[i], e = a.dE[i];
    pass_particle<WAKE>(z, e, r, QE != QE_OFF, c, g, pending, upd_E0, pmean, potd, acc_z,
                        acc_z2, acc_d, n_in, s_cnt, s_lo, s_hi);
    a.z[i] = z;
    a.dE[i] = e;
  }

  block_sum4<THREADS>(acc_z, acc_z2, acc_d, (double)n_in,
                      a.part_sum + (size_t)blockIdx.x * kNumSums);

  if (WAKE) {
    __syncthreads();
    uint32_t* pc = a.part_cnt + (size_t)blockIdx.x * a.B;
    unsigned long long* pq = a.part_cic + (size_t)blockIdx.x * a.B;
    for (int i = threadIdx.x; i < a.B; i += THREADS) {
      pc[i] = s_cnt[i];
      pq[i] = ((unsigned long long)s_hi[i] << 32) | s_lo[i];
    }
  }
}

// Merge of the per-block histograms.  Grid (bins/256, G): block column g sums
// the partials of blocks g, g+G, ... and adds them to the merged arrays with
// integer atomics (exact, so the result does not depend on their order).
// out layout (u64): counts[B] | CIC counts[B] | CIC Σw·2^24 [B].
__global__ void k_hist_reduce(const uint32_t* __restrict__ part_cnt,
                              const unsigned long long* __restrict__ part_cic, int nblk, int B,
                              unsigned long long* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  unsigned long long sc = 0ull, sn = 0ull, sw = 0ull;
  for (int k = blockIdx.y; k < nblk; k += gridDim.y) {
    sc += __ldg(part_cnt + (size_t)k * B + b);
    if (part_cic) {
      const unsigned long long v = __ldg(part_cic + (size_t)k * B + b);
      sn += v >> kCicSumBits;
      sw += v & kCicSumMask;
    }
  }
  if (sc) atomicAdd(out + b, sc);
  if (part_cic) {
    if (sn) atomicAdd(out + B + b, sn);
    if (sw) atomicAdd(out + 2 * B + b, sw);
  }
}

// Pending kick + re-centring (optional), copy-out (optional) and the moments
// [Σz, Σz², ΣdE, ΣdE²] per block.
__global__ void __launch_bounds__(kTrackThreads) k_flush(FlushArgs a) {
  const bool apply = a.apply && a.ts && a.ts->pending;
  const double pmean = apply ? a.ts->pending_mean : 0.0;
  GridConst g{a.B, 0.0, 0.0, 0.0, a.c1, a.cB, a.inv_cstep};
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
    double z = a.z[i], e = a.dE[i];
    if (apply) {
      if (a.use_wake) e = e - wake_kick(z, g, a.potd);
      if (a.update_E0) e = __dsub_rn(e, pmean);
    }
    if (a.z_out) a.z_out[i] = z;
    if (a.dE_out) a.dE_out[i] = e;
    s0 += z;
    s1 = fma(z, z, s1);
    s2 += e;
    s3 = fma(e, e, s3);
  }
  block_sum4<kTrackThreads>(s0, s1, s2, s3, a.part + (size_t)blockIdx.x * 4);
}

// NGP histogram only (hj_histogram, hj_apply_wakefield).
__global__ void __launch_bounds__(kTrackThreads) k_histogram(const double* __restrict__ z,
                                                            int64_t n, GridConst g,
                                                            uint32_t* __restrict__ part_cnt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* s_cnt = reinterpret_cast<uint32_t*>(smem_raw);
  for (int i = threadIdx.x; i < g.B; i += blockDim.x) s_cnt[i] = 0u;
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    bool in;
    int j = ngp_bin(__ldg(z + i), g, in);
    if (in) atomicAdd(&s_cnt[j], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < g.B; i += blockDim.x)
    part_cnt[(size_t)blockIdx.x * g.B + i] = s_cnt[i];
}

__global__ void k_interp_kick(const double* __restrict__ z, double* __restrict__ dE, int64_t n,
                              const double* __restrict__ pot, GridConst g) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    dE[i] = __dsub_rn(dE[i], wake_kick_ref(__ldg(z + i), g, pot));
}

__global__ void k_rf_kick(double V, double sin_phis, double k, double phi_s,
                          const double* __restrict__ z, double* __restrict__ dE, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double phi = __dadd_rn(__dmul_rn(-__ldg(z + i), k), phi_s);
    dE[i] = __dadd_rn(dE[i], __dmul_rn(V, __dsub_rn(sin(phi), sin_phis)));
  }
}

__global__ void k_qe(double excitation, const double* __restrict__ draws, uint64_t seed,
                     int64_t turn, double* __restrict__ dE, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nq = (n + 3) >> 2;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += stride) {
    double rr[4];
    if (!draws) philox_normals4(seed, turn, q, rr);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int64_t i = 4 * q + j;
      if (i < n) {
        double r = draws ? __ldg(draws + i) : rr[j];
        dE[i] = __dadd_rn(dE[i], __dmul_rn(excitation, r));
      }
    }
  }
}

__global__ void k_sr(double damping, double* __restrict__ dE, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    dE[i] = __dmul_rn(dE[i], damping);
}

__global__ void k_phase_advance(StepConst c, const double* __restrict__ dE,
                                double* __restrict__ z, int64_t n) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double zi = z[i], e = __ldg(dE + i);
    // Drift only: RF/QE/SR disabled by zero voltage/flags in `c`.
    if (c.update_eta) {
      double dg = __dmul_rn(e, c.inv_mass);
      double gp = __dadd_rn(c.gamma0, dg);
      double eta = __dsub_rn(c.alpha_c, 1.0 / __dmul_rn(gp, gp));
      double coeff = __dmul_rn(__dmul_rn(c.two_pi_h, eta), c.inv_b2E0);
      double ph = -__dsub_rn(__dmul_rn(zi, c.k), c.phi_s);
      ph = __dadd_rn(ph, __dmul_rn(coeff, e));
      zi = __dmul_rn(__dadd_rn(-ph, c.phi_s), c.inv_k);
    } else if (c.drift_ok) {
      double ph = -__dsub_rn(__dmul_rn(zi, c.k), c.phi_s);
      ph = __dadd_rn(ph, __dmul_rn(c.coeff0, e));
      zi = __dmul_rn(__dadd_rn(-ph, c.phi_s), c.inv_k);
    }
    z[i] = zi;
  }
}

__global__ void k_gaussian(uint64_t seed, int64_t turn, int64_t n, double* __restrict__ out) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t nq = (n + 3) >> 2;
  for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < nq; q += stride) {
    double rr[4];
    philox_normals4(seed, turn, q, rr);
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (4 * q + j < n) out[4 * q + j] = rr[j];
  }
}

int elementwise_grid(int64_t n) {
  int64_t g = (n + 255) / 256;
  if (g < 1) g = 1;
  if (g > 148 * 16) g = 148 * 16;
  return (int)g;
}

}  // namespace

// Raise a kernel's dynamic shared-memory limit to what the device allows
// beside the kernel's own static shared memory.
cudaError_t allow_dynamic_smem(const void* fn, int max_smem_optin) {
  cudaFuncAttributes attr{};
  cudaError_t e = cudaFuncGetAttributes(&attr, fn);
  if (e != cudaSuccess) return e;
  const int dyn = max_smem_optin - (int)attr.sharedSizeBytes;
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn > 0 ? dyn : 0);
}

namespace {
template <bool W, int Q>
const void* pass_fn_wq(int cfg) {
  switch (cfg) {
    case 0: return (const void*)k_track_pass<W, Q, 4, 512>;
    case 1: return (const void*)k_track_pass<W, Q, 2, 1024>;
    default: return (const void*)k_track_pass<W, Q, 2, 512>;
  }
}

template <bool W>
const void* pass_fn_w(int qe, int cfg) {
  switch (qe) {
    case QE_PHILOX: return pass_fn_wq<W, QE_PHILOX>(cfg);
    case QE_DRAWS: return pass_fn_wq<W, QE_DRAWS>(cfg);
    default: return pass_fn_wq<W, QE_OFF>(cfg);
  }
}

const void* pass_fn(int wake, int qe, int cfg) {
  return wake ? pass_fn_w<true>(qe, cfg) : pass_fn_w<false>(qe, cfg);
}
}  // namespace

int pass_cfg_threads(int cfg) { return cfg == 1 ? 1024 : 512; }
int pass_cfg_ppt(int cfg) { return cfg == 0 ? 4 : 2; }

cudaError_t prepare_track_kernels(int max_smem) {
  for (int w = 0; w < 2; ++w)
    for (int q = 0; q < 3; ++q)
      for (int c = 0; c < kNumPassCfgs; ++c) {
        cudaError_t e = allow_dynamic_smem(pass_fn(w, q, c), max_smem);
        if (e != cudaSuccess) return e;
      }
  return allow_dynamic_smem((const void*)k_histogram, max_smem);
}

size_t track_smem_bytes(int B, int use_wake) {
  return use_wake ? (size_t)B * (sizeof(unsigned long long) + sizeof(uint32_t)) : 0;
}

int track_blocks_per_sm(int B, int qe_mode, int use_wake, int cfg) {
  const size_t smem = track_smem_bytes(B, use_wake);
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, pass_fn(use_wake, qe_mode, cfg),
                                                    pass_cfg_threads(cfg), smem) != cudaSuccess)
    bps = 1;
  return bps < 1 ? 1 : bps;
}

// Blocks of the particle pass: enough to fill the GPU, but each block should
// own at least ~2 bins' worth of histogram traffic per particle it moves.
int track_grid_size(int64_t n, int B, int num_sms, int blocks_per_sm, int cfg) {
  int64_t per_block = (int64_t)pass_cfg_ppt(cfg) * pass_cfg_threads(cfg);
  if (per_block < 2 * (int64_t)B) per_block = 2 * (int64_t)B;
  int64_t g = (n + per_block - 1) / per_block;
  int64_t cap = (int64_t)num_sms * blocks_per_sm;
  if (g > cap) g = cap;
  // the packed CIC counter holds at most kMaxBlockParticles per block and turn
  const int64_t need = (n + kMaxBlockParticles - 1) / kMaxBlockParticles;
  if (g < need) g = need;
  if (g < 1) g = 1;
  return (int)g;
}

cudaError_t launch_track_pass(const PassArgs& a, int grid, cudaStream_t st) {
  const size_t smem = track_smem_bytes(a.B, a.use_wake);
  void* args[] = {const_cast<PassArgs*>(&a)};
  return cudaLaunchKernel(pass_fn(a.use_wake, a.qe_mode, a.cfg), dim3(grid),
                          dim3(pass_cfg_threads(a.cfg)), args, smem, st);
}

cudaError_t launch_hist_reduce(const uint32_t* part_cnt, const unsigned long long* part_cic,
                               int nblk, int B, unsigned long long* out, bool zero_first,
                               cudaStream_t st) {
  if (zero_first) {
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long) * (part_cic ? 3 : 1) * B, st);
    if (e != cudaSuccess) return e;
  }
  const int G = nblk < 16 ? nblk : 16;
  dim3 grid((B + 255) / 256, G > 0 ? G : 1);
  k_hist_reduce<<<grid, 256, 0, st>>>(part_cnt, part_cic, nblk, B, out);
  return cudaGetLastError();
}

cudaError_t launch_flush(const FlushArgs& a, int grid, cudaStream_t st) {
  k_flush<<<grid, kTrackThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_histogram_only(const double* z, int64_t n, int B, double e0, double eN,
                                  double inv_estep, uint32_t* part_cnt, int grid,
                                  cudaStream_t st) {
  GridConst g{B, e0, eN, inv_estep, 0.0, 0.0, 0.0};
  size_t smem = (size_t)B * sizeof(uint32_t);
  k_histogram<<<grid, kTrackThreads, smem, st>>>(z, n, g, part_cnt);
  return cudaGetLastError();
}

cudaError_t launch_interp_kick(const double* z, double* dE, int64_t n, const double* pot,
                               int B, double c1, double cB, double inv_cstep,
                               cudaStream_t st) {
  GridConst g{B, 0.0, 0.0, 0.0, c1, cB, inv_cstep};
  k_interp_kick<<<elementwise_grid(n), 256, 0, st>>>(z, dE, n, pot, g);
  return cudaGetLastError();
}

cudaError_t launch_rf_kick(double V, double sin_phis, double k, double phi_s,
                           const double* z, double* dE, int64_t n, cudaStream_t st) {
  k_rf_kick<<<elementwise_grid(n), 256, 0, st>>>(V, sin_phis, k, phi_s, z, dE, n);
  return cudaGetLastError();
}

cudaError_t launch_qe(double excitation, const double* draws, uint64_t seed, int64_t turn,
                      double* dE, int64_t n, cudaStream_t st) {
  k_qe<<<elementwise_grid((n + 3) / 4), 256, 0, st>>>(excitation, draws, seed, turn, dE, n);
  return cudaGetLastError();
}

cudaError_t launch_sr(double damping, double* dE, int64_t n, cudaStream_t st) {
  k_sr<<<elementwise_grid(n), 256, 0, st>>>(damping, dE, n);
  return cudaGetLastError();
}

cudaError_t launch_phase_advance(int update_eta, TurnScalars s, double inv_mass,
                                 double alpha_c, double two_pi_h, double phi_s,
                                 const double* dE, double* z, int64_t n, cudaStream_t st) {
  StepConst c{};
  c.phi_s = phi_s;
  c.k = s.k;
  c.inv_k = s.inv_k;
  c.gamma0 = s.gamma0;
  c.inv_mass = inv_mass;
  c.alpha_c = alpha_c;
  c.two_pi_h = two_pi_h;
  c.inv_b2E0 = s.inv_b2E0;
  c.coeff0 = s.coeff0;
  c.drift_ok = s.drift_ok;
  c.update_eta = update_eta;
  k_phase_advance<<<elementwise_grid(n), 256, 0, st>>>(c, dE, z, n);
  return cudaGetLastError();
}

cudaError_t launch_gaussian(uint64_t seed, int64_t turn, int64_t n, double* out,
                            cudaStream_t st) {
  k_gaussian<<<elementwise_grid((n + 3) / 4), 256, 0, st>>>(seed, turn, n, out);
  return cudaGetLastError();
}

}  // namespace hj
