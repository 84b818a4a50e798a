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
//   * RF kick: V(sin(ϕs - x) - sin ϕs) with x = z k = m h + t, h = 2π/128,
//     |t| <= π/128, and sin(ϕs - x) = sin θm cos t - cos θm sin t with
//     θm = ϕs - m h from a 128-entry shared-memory table (computed in
//     extended precision on the host) and sin t, cos t - 1 from their Taylor
//     series through t^7 and t^6.  For m = 0 the kick is V sin ϕs (cos t - 1)
//     - V cos ϕs sin t, free of the cancellation in sin(ϕ) - sin ϕs.  No branches.
//   * Philox-4x32 round keys are precomputed on the host (kernel parameters);
//     the Float64 normals come from a 2048-layer ziggurat whose (X_i, D_i)
//     rows sit in shared memory; the ~0.23 % of particles whose draw needs the
//     slow path are finished later, 32 at a time (finish_deferred).
//   * 1/γ² of the drift: rcp.approx.ftz.f64 refined by one Newton step
//     (relative error ~1e-14 on a term 5e-5 of η, i.e. ~1e-18 on η).
//   * drift: z' = z - (2π h / (β0² E0 k)) η_i ΔE, the reference's
//     z' = (ϕs - (ϕs - z k + coeff ΔE)) / k without its cancellation against
//     ϕs (the two agree to the reference's own rounding, ~1e-14 of z).
//   * floor() and round-to-nearest as integers use the 1.5·2^52 addition
//     (directed-rounding add for floor), the integer read from the low word.
//   * clamps are compare-and-select (Julia clamp semantics, NaN stays NaN).
//   * reciprocals of mass and β0²E0 and the RF coefficients V sin ϕs,
//     V cos ϕs are precomputed.
//   * switches that are off act through neutral values (a zero kick table
//     and mean before the first turn, damping 1 without SR, r = 0 without
//     QE), all exact, so the pass has no per-particle branches on them.
#include <algorithm>
#include <memory>

#include "hj_host.h"
#include "hj_internal.h"

namespace hj {
namespace {

// The normal generator's tables (NormalTables) in global memory, filled once
// per device when the kernels are prepared; the fused pass stages them into
// shared memory, the other kernels read them through the cache.
__device__ NormalTables g_normal;

__device__ __forceinline__ void philox_normals2(uint64_t seed, int64_t turn, int64_t p,
                                                double out[2]) {
  philox_normals2_rk(seed, philox_keys(seed), turn, p, &g_normal,
                     reinterpret_cast<const double2*>(g_normal.xd), out);
}

// Run- and turn-constants of the fused pass.
struct FusedConst {
  double Vs;                // V sin ϕs
  double rf_inv_h, rf_h_hi, rf_h_lo;   // RF table step h = 2π/128: 1/h, h (two words)
  double k;
  double excitation, damping;
  double gamma0, inv_mass, alpha_c, Kz;  // Kz = 2π h / (β0² E0 k)
  double coeff0z;           // Kz η0 (constant-η drift)
  int drift_ok, update_eta;
};

// Constants of the single-step phase-advance kernel (reference operation order).
struct StepConst {
  double phi_s, k, inv_k, gamma0, inv_mass, alpha_c, two_pi_h, inv_b2E0, coeff0;
  int drift_ok, update_eta;
};

struct GridConst {
  int B;
  double e0, eN, inv_e, c1, cB, inv_c;
  double v_off;   // 1/2 - e0/Δe: v = z/Δe + v_off is the cell coordinate of the kick table
};

// 1/2 - e0/Δe, rounded the same way by every kernel that forms cell coordinates.
__device__ __forceinline__ double kick_offset(double e0, double inv_e) {
  return __dsub_rn(0.5, __dmul_rn(e0, inv_e));
}

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

constexpr double kMagic = 6755399441055744.0;   // 1.5·2^52: unit ulp, integer in the low word

// Julia's clamp(x, lo, hi) by compare-and-select (NaN stays NaN).
__device__ __forceinline__ double clamp_sel(double x, double lo, double hi) {
  x = (x < lo) ? lo : x;
  return (x > hi) ? hi : x;
}

// Interpolation cell of z on the bin centers (src/wakefield.jl:64-78), 0-based:
// idx = clamp(floor(u), 0, B-2), w = u - floor(u), u = (clamp(z,c1,cB)-c1)/Δc.
// floor(u) = (u + 1.5·2^52 rounded down) - 1.5·2^52, exact for 0 <= u < 2^51.
// The deposit of turn t and the kick applied in turn t+1 call this with the
// same z, so they agree exactly.
__device__ __forceinline__ void cic_cell(double z, const GridConst& g, int& idx, double& w) {
  const double cl = clamp_sel(z, g.c1, g.cB);
  const double u = __dmul_rn(__dsub_rn(cl, g.c1), g.inv_c);
  const double fm = __dadd_rd(u, kMagic);
  w = __dsub_rn(u, __dsub_rn(fm, kMagic));
  idx = min(max(__double2loint(fm), 0), cic_hi(g.B));
}

// Cell of the kick table (B + 1 cells): v = z/Δe + 1/2 - e0/Δe (one FMA),
// j = floor(v) clamped to [0, B], w = v - floor(v).  Cell j >= 1 is the
// reference's interpolation cell j-1 between centres c[j-1] and c[j]
// (src/wakefield.jl:64-78); cells 0 and B hold the flat ends pot[0] and pot[B-1]
// that the reference's clamp of z to [c1, cB] gives, so out-of-range particles need
// no clamp of z.  v agrees with the reference's (z - c1)/Δc to ~1e-15 of the bin
// count, so the kick agrees to that fraction of a bin-to-bin potential step.
// floor(v): the low word of (v + 1.5·2^52 rounded down) when the high word is
// 0x43380000 (0 <= v < 2^32); other high words mean v < 0 (cell 0) or v >= 2^32,
// +inf and NaN (cell B) -- every z lands in a valid cell.
__device__ __forceinline__ void kick_cell(double z, const GridConst& g, int& j, double& w) {
  const double v = fma(z, g.inv_e, g.v_off);
  const double fm = __dadd_rd(v, kMagic);
  w = __dsub_rn(v, __dsub_rn(fm, kMagic));
  const int t = __double2hiint(fm) - 0x43380000;
  const unsigned lo = (unsigned)__double2loint(fm);
  j = (t == 0) ? (int)min(lo, (unsigned)g.B) : (t > 0 ? g.B : 0);
}

__device__ __forceinline__ double2 ld_table(const double2* p) {
  double2 v;
  asm("ld.global.nc.L1::evict_last.v2.f64 {%0,%1}, [%2];" : "=d"(v.x), "=d"(v.y) : "l"(p));
  return v;
}

// The pass's shared-memory windows, both starting at cell w0 (centred on the
// cell of the last turn's mean z).
// * Kick table: s_win[i] = pot_left[w0 + i] (the left value, .x, of table
//   cell w0 + i) for i < lim + 1, where the cells j with w0 <= j < w0 + lim
//   are "hot": their left value and their right neighbour's left value are
//   both in the window.  For cells 1..B-2 the step of the global table is
//   pot[j] - pot[j-1] = pot_left[j+1] - pot_left[j], and for cell 0 it is
//   pot[0] - pot[0] = 0, so a hot cell's (left value, step) from the window
//   is bit-identical to its global entry.  Cells B-1 and B (whose step or
//   value the bins step sets differently) are never hot.
// * Histograms: bins and cells w0 .. w0 + h - 1 have their per-block
//   counters in shared memory.  A deposit outside goes to the bunch's spill
//   histograms in global memory (u64, laid out as the merged ones: counts [B]
//   | cell counts [B+1] | cell Σw·2^24 [B+1]), which the merge folds in and
//   clears; h = B + 1 (w0 = 0) where all cells fit.
struct PassWindow {
  const double* s_win;
  int w0;
  unsigned lim;
  unsigned h;
  unsigned inner;   // max(h, 1) - 1: cells w0 + 1 .. w0 + inner have their bin inside too
};

// Table entry and weight of the kick of z (issued early: the gather's latency
// overlaps the RF and QE arithmetic of the pass).  Hot cells read the
// shared-memory window, the others the kick table in global memory.
struct KickFetch {
  double p0, d, w;
};
__device__ __forceinline__ KickFetch kick_fetch(double z, const GridConst& g,
                                                const PassWindow& kw,
                                                const double2* __restrict__ potd) {
  int j;
  KickFetch f;
  kick_cell(z, g, j, f.w);
  const unsigned r = (unsigned)(j - kw.w0);
  if (r < kw.lim) {
    const double lo = kw.s_win[r], hi = kw.s_win[r + 1];
    f.p0 = lo;
    f.d = __dsub_rn(hi, lo);
  } else {
    const double2 t = ld_table(potd + j);
    f.p0 = t.x;
    f.d = t.y;
  }
  return f;
}

// Kick of the fused pass: lerp from the kick table, cell j holding
// (pot at its left centre, pot step to its right centre), zero step in cells 0 and B.
__device__ __forceinline__ double wake_kick(double z, const GridConst& g,
                                            const double2* __restrict__ potd) {
  int j;
  double w;
  kick_cell(z, g, j, w);
  const double2 pd = ld_table(potd + j);
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
// Only in-range particles are counted, and for them 0 <= u <= B.
__device__ __forceinline__ int ngp_bin(double z, const GridConst& g, bool& in) {
  in = (z >= g.e0) & (z <= g.eN);
  const double u = __dmul_rn(__dsub_rn(z, g.e0), g.inv_e);
  return min(max(__double2loint(__dadd_rd(u, kMagic)), 0), g.B - 1);
}

// Bits of 1/2 - 2^-30 and the span up to 1/2 + 2^-30 (positive doubles order
// as their bit patterns).
constexpr long long kHalfLoBits = 0x3FDFFFFFFF000000ll;
constexpr unsigned long long kHalfSpanBits = 0x3FE0000000800000ull - 0x3FDFFFFFFF000000ull;

// Kick-table cell of z (as kick_cell) and, from the same coordinate, the
// histogram bin of src/utils.jl:387-397.  v - 1/2 = z/Δe + 1/2 - e0/Δe - 1/2
// lies within ~4 B 2^-53 (below 1e-11 for B <= 2^20) of the reference's
// u = RN(RN(z - e0)/Δe), so for |w - 1/2| >= 2^-30 the bin floor(u) is
// floor(v) - 1 + [w >= 1/2] and z is in range iff that bin is in [0, B-1];
// within 2^-30 of a bin edge (at 1e8 particles about one particle in five
// turns) ngp_bin evaluates the reference's own rounding.  The tests on w run
// on its bits, so the bin costs no floating-point work.
__device__ __forceinline__ void cell_and_bin(double z, const GridConst& g, int& j, double& w,
                                             int& nb, bool& in) {
  const double v = fma(z, g.inv_e, g.v_off);
  const double fm = __dadd_rd(v, kMagic);
  w = __dsub_rn(v, __dsub_rn(fm, kMagic));
  const int t = __double2hiint(fm) - 0x43380000;
  const unsigned lo = (unsigned)__double2loint(fm);
  j = (t == 0) ? (int)min(lo, (unsigned)g.B) : (t > 0 ? g.B : 0);
  const unsigned long long near_edge =
      (unsigned long long)(__double_as_longlong(w) - kHalfLoBits);
  if (near_edge <= kHalfSpanBits) {
    nb = ngp_bin(z, g, in);
  } else {
    const int jb = (int)lo - 1 + (__double2hiint(w) >= 0x3FE00000 ? 1 : 0);
    in = (t == 0) & (jb >= 0) & (jb < g.B);
    nb = jb;
  }
}

// Reference-form bin for the single-step histogram kernel (any z).
__device__ __forceinline__ int ngp_bin_any(double z, const GridConst& g, bool& in) {
  in = (z >= g.e0) & (z <= g.eN);
  const int j = __double2int_rd(__dmul_rn(__dsub_rn(z, g.e0), g.inv_e));
  return min(max(j, 0), g.B - 1);
}

// V(sin(ϕs - x) - sin ϕs), x = z k (see the header comment): x = m h + t with
// m = rint(x/h) from the 1.5·2^52 addition, h = 2π/128, t by Cody-Waite with
// a two-word h (|t| <= π/128), and rot = (V sin θm, V cos θm), θm = ϕs - m h,
// from the shared-memory table (entry m mod 128).  sin t and cos t - 1 are
// their Taylor series through t^7 and t^6 (truncation below 1e-20); the kick
// V sin θm (cos t - 1) - V cos θm sin t + (V sin θm - V sin ϕs) is, for m = 0,
// free of the cancellation in sin(ϕ) - sin ϕs.  No branches.
// EXACT: every operation rounds where it is written (no contraction), so
// that a second evaluation anywhere reproduces the result bit for bit (the
// Float64-normals pass needs that to take a provisional turn back).
template <bool EXACT>
__device__ __forceinline__ double rf_term(double z, const FusedConst& c,
                                          const double2* __restrict__ s_rf) {
  if (EXACT) {
    const double x = __dmul_rn(z, c.k);
    const double y = fma(x, c.rf_inv_h, kMagic);
    const double md = __dsub_rn(y, kMagic);
    double t = fma(-md, c.rf_h_hi, x);
    t = fma(-md, c.rf_h_lo, t);
    const double2 rot = s_rf[__double2loint(y) & (kRfTableSize - 1)];
    const double t2 = __dmul_rn(t, t);
    double p = fma(t2, -1.984126984126984e-04, 8.333333333333333e-03);   // -1/7!, 1/5!
    p = fma(t2, p, -1.6666666666666666e-01);                               // -1/3!
    const double sn = fma(__dmul_rn(t, t2), p, t);
    double q = fma(t2, -1.388888888888889e-03, 4.1666666666666664e-02);  // -1/6!, 1/4!
    q = fma(t2, q, -0.5);
    const double cm1 = __dmul_rn(t2, q);
    return __dadd_rn(fma(rot.x, cm1, __dmul_rn(-rot.y, sn)), __dsub_rn(rot.x, c.Vs));
  }
  const double x = z * c.k;
  const double y = fma(x, c.rf_inv_h, kMagic);
  const double md = y - kMagic;
  double t = fma(-md, c.rf_h_hi, x);
  t = fma(-md, c.rf_h_lo, t);
  const double2 rot = s_rf[__double2loint(y) & (kRfTableSize - 1)];
  const double t2 = t * t;
  double p = fma(t2, -1.984126984126984e-04, 8.333333333333333e-03);
  p = fma(t2, p, -1.6666666666666666e-01);
  const double sn = fma(t * t2, p, t);
  double q = fma(t2, -1.388888888888889e-03, 4.1666666666666664e-02);
  q = fma(t2, q, -0.5);
  const double cm1 = t2 * q;
  return fma(rot.x, cm1, -rot.y * sn) + (rot.x - c.Vs);
}

// One particle for one turn, given its wake kick (lerp of the previous turn's
// potential; 0 without the wake) and its RF kick increment rf_term(z), both
// formed from the z this pass starts from: previous turn's kick and E0
// re-centring (zero table / zero mean when nothing is pending), RF kick, QE,
// SR, drift.  Without update_η the drift coefficient is the constant-η one
// (zero when apply_phase_advance! would skip the advance).  The moments and
// deposits of the new z follow in deposit_group.
template <bool WAKE, bool EXACT = false>
__device__ __forceinline__ void particle_turn(double& z, double& e, double r, double kick,
                                              double rf, const FusedConst& c, double pmean,
                                              double& acc_d) {
  if (EXACT) {   // every operation rounds where it is written (see rf_term)
    if (WAKE) e = __dsub_rn(e, kick);
    e = __dsub_rn(e, pmean);
    const double e_start = e;
    e = __dadd_rn(e, rf);
    e = fma(c.excitation, r, e);
    e = __dmul_rn(e, c.damping);
    const double gp = fma(e, c.inv_mass, c.gamma0);
    const double g2 = __dmul_rn(gp, gp);
    double ri = rcp_approx(g2);
    ri = fma(ri, fma(-g2, ri, 1.0), ri);
    const double coeff = c.update_eta ? __dmul_rn(c.Kz, __dsub_rn(c.alpha_c, ri)) : c.coeff0z;
    z = fma(-coeff, e, z);
    acc_d += __dsub_rn(e, e_start);
    return;
  }
  if (WAKE) e = e - kick;
  e = e - pmean;
  const double e_start = e;
  e = e + rf;
  e = fma(c.excitation, r, e);                         // r = 0 without QE
  e = e * c.damping;                                   // damping = 1 without SR
  const double gp = fma(e, c.inv_mass, c.gamma0);     // γ0 + ΔE/m
  const double g2 = gp * gp;
  double ri = rcp_approx(g2);
  ri = fma(ri, fma(-g2, ri, 1.0), ri);
  const double coeff = c.update_eta ? c.Kz * (c.alpha_c - ri) : c.coeff0z;
  z = fma(-coeff, e, z);
  acc_d += e - e_start;
}

// Moments and deposits of K particles' new z: Σz, Σz², the NGP count and, in
// the kick-table cell the next pass reads for this z, the cell count and
// Σ w·2^24.  The shared atomics of all K particles are issued before any of
// their returned values is used, so their latencies overlap.  s_ngp, s_lo and
// s_hi are the shared arrays offset by the window's start (w0 even, so that
// bin b is at word b >> 1, half b & 1, of the 16-bit pairs): bin b's counter
// is s_ngp[b] (s_ngp[b >> 1]), cell c's words s_lo[c], s_hi[c], for b and c
// in the window.  An in-range particle's bin is its cell or the one below, so
// a cell in (w0, w0 + h) puts both in the window: when all K are there the
// deposits run unchecked, else each is checked and spilled when outside.
// Without WIN the window holds every cell and nothing is checked.
template <int K, bool N32, bool WIN>
__device__ __forceinline__ void deposit_group(const double (&z)[K], const GridConst& g,
                                              const PassWindow& hw, double& acc_z,
                                              double& acc_z2, int32_t& n_in, uint32_t* s_ngp,
                                              uint32_t* s_lo, uint32_t* s_hi,
                                              unsigned long long* __restrict__ spill) {
  int nb[K], cj[K];
  bool nin[K];
  uint32_t cq[K];
  bool inner = true;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    acc_z += z[k];
    acc_z2 = fma(z[k], z[k], acc_z2);
    double w;
    cell_and_bin(z[k], g, cj[k], w, nb[k], nin[k]);
    n_in += nin[k] ? 1 : 0;
    // w·2^24 rounded to nearest (at most 2^24; a NaN z lands in cell B with
    // any q and is flagged by the moments)
    cq[k] = min((uint32_t)__double2loint(fma(w, 16777216.0, kMagic)), 16777216u);
    if (WIN) inner &= (uint32_t)(cj[k] - hw.w0 - 1) < hw.inner;
  }
  uint32_t ong[K], olo[K];
  if (inner) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      ong[k] = 0u;
      if (nin[k]) {
        if (N32) {
          atomicAdd(&s_ngp[nb[k]], 1u);   // one 32-bit counter per bin, no return value used
        } else {
          ong[k] = atomicAdd(&s_ngp[nb[k] >> 1], 1u << ((nb[k] & 1) << 4));
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) olo[k] = atomicAdd(&s_lo[cj[k]], cq[k]);
#pragma unroll
    for (int k = 0; k < K; ++k)
      atomicAdd(&s_hi[cj[k]], (1u << (kCicSumBits - 32)) + (olo[k] + cq[k] < olo[k] ? 1u : 0u));
  } else {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      ong[k] = 0u;
      if (nin[k]) {
        if ((uint32_t)(nb[k] - hw.w0) < hw.h) {
          if (N32) atomicAdd(&s_ngp[nb[k]], 1u);
          else ong[k] = atomicAdd(&s_ngp[nb[k] >> 1], 1u << ((nb[k] & 1) << 4));
        } else {
          atomicAdd(spill + nb[k], 1ull);
          nin[k] = false;                 // no 16-bit counter to check below
        }
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if ((uint32_t)(cj[k] - hw.w0) < hw.h) {
        olo[k] = atomicAdd(&s_lo[cj[k]], cq[k]);
        atomicAdd(&s_hi[cj[k]], (1u << (kCicSumBits - 32)) + (olo[k] + cq[k] < olo[k] ? 1u : 0u));
      } else {
        atomicAdd(spill + g.B + cj[k], 1ull);
        atomicAdd(spill + 2 * g.B + 1 + cj[k], (unsigned long long)cq[k]);
      }
    }
  }
  if (!N32) {
    // 16-bit counters, two bins per word: the increment that takes a counter
    // to 2^15 moves 2^15 counts to the spill counts (the counter has another
    // 2^15 - 1 increments of room before the move lands)
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const int sh = (nb[k] & 1) << 4;
      if (nin[k] && ((ong[k] >> sh) & 0xFFFFu) == 0x7FFFu) {
        atomicSub(&s_ngp[nb[k] >> 1], 0x8000u << sh);
        atomicAdd(spill + nb[k], 0x8000ull);
      }
    }
  }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Fixed-order block reduction of four accumulators into out[0..3] (thread 0).
// red: shared scratch of THREADS/32 x 4 doubles.
template <int THREADS>
__device__ __forceinline__ void block_sum4(double a0, double a1, double a2, double a3,
                                           double* out, double (*red)[4]) {
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
    asm("ld.global.L1::no_allocate.v4.f64 {%0,%1,%2,%3}, [%4];"
        : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
        : "l"(p));
  } else {
    asm("ld.global.L1::no_allocate.v2.f64 {%0,%1}, [%2];" : "=d"(v[0]), "=d"(v[1]) : "l"(p));
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

// Single-precision normals of the PPT particles of pairs pair0, pair0 + 1
// (the opt-in fast layouts).
template <int PPT>
__device__ __forceinline__ void group_normals_fast(const PhiloxKeys& rk, int64_t turn,
                                                   int64_t pair0, double r[PPT]) {
  philox_normals2_fast(rk, turn, pair0, r);
  if (PPT == 4) philox_normals2_fast(rk, turn, pair0 + 1, r + 2);
}

// Float64 normals of the PPT particles of pairs pair0, pair0 + 1 by the
// ziggurat's fast path: bit j of the result is set where particle j's draw
// was accepted; r[j] holds its normal, or its rejected candidate.
template <int PPT>
__device__ __forceinline__ unsigned group_normals_zig(const PhiloxKeys& rk, int64_t turn,
                                                      int64_t pair0,
                                                      const double2* __restrict__ zt,
                                                      double r[PPT]) {
  unsigned ok = 0u;
#pragma unroll
  for (int h = 0; h < PPT / 2; ++h) {
    const int64_t p = pair0 + h;
    uint32_t c[4] = {(uint32_t)p, (uint32_t)((uint64_t)p >> 32), (uint32_t)turn,
                     (uint32_t)((uint64_t)turn >> 32)};
    philox4x32_10(c, rk);
    ok |= (zig_fast(c[1], c[0], zt, r[2 * h]) ? 1u : 0u) << (2 * h);
    ok |= (zig_fast(c[3], c[2], zt, r[2 * h + 1]) ? 1u : 0u) << (2 * h + 1);
  }
  return ok;
}

// Takes back what deposit_group added for one particle at z: the moments (to
// rounding) and the NGP and cell deposits (exactly: the packed cell word
// loses the 2^44 + q it gained, borrow included; the spill histograms, and
// the spill counts in place of a 16-bit NGP counter, take the negative,
// modulo 2^64).
template <bool N32>
__device__ __forceinline__ void undeposit(double z, const GridConst& g, const PassWindow& hw,
                                          double& acc_z, double& acc_z2, int32_t& n_in,
                                          uint32_t* s_ngp, uint32_t* s_lo, uint32_t* s_hi,
                                          unsigned long long* __restrict__ spill) {
  acc_z = __dsub_rn(acc_z, z);
  acc_z2 = fma(-z, z, acc_z2);
  int cj, nb;
  double w;
  bool nin;
  cell_and_bin(z, g, cj, w, nb, nin);
  if (nin) {
    n_in -= 1;
    if (N32 && (uint32_t)(nb - hw.w0) < hw.h) atomicSub(&s_ngp[nb], 1u);
    else atomicAdd(spill + nb, ~0ull);
  }
  const uint32_t cq = min((uint32_t)__double2loint(fma(w, 16777216.0, kMagic)), 16777216u);
  if ((uint32_t)(cj - hw.w0) < hw.h) {
    const uint32_t old = atomicSub(&s_lo[cj], cq);
    atomicSub(&s_hi[cj], (1u << (kCicSumBits - 32)) + (old < cq ? 1u : 0u));
  } else {
    atomicAdd(spill + g.B + cj, ~0ull);
    atomicAdd(spill + 2 * g.B + 1 + cj, 0ull - (unsigned long long)cq);
  }
}

// One turn over the bunch.  PPT particles per thread per iteration (4 with the
// next group prefetched in registers, or 2 with twice the threads per SM).
// Particle groups (PPT particles each) one block processes: thread t takes
// groups q_begin + t, + q_step, ... below q_end; its partial histograms and
// sums go to slot `part`; the `tail` block also takes the n % PPT last particles.
struct PassRange {
  int64_t q_begin, q_step, q_end;
  int32_t part;
  bool tail;
};

// Shared-memory tables of the pass: RF table [kRfTableSize] | the ziggurat's
// (X_i, D_i) rows [kZigLayers].
constexpr size_t kPassTableBytes = (size_t)(kRfTableSize + kZigLayers) * 16u;

// Finishes particle i, whose draw failed the ziggurat's fast test.  The pass
// turned and deposited it with the rejected candidate (so that its loop needs
// no per-particle masks) but stored it as it was loaded.  That provisional
// turn is evaluated again, bit for bit (particle_turn rounds where written),
// and taken back (undeposit, and its share of the sums); the turn with the
// normal from the ziggurat's slow path is then applied, deposited and stored.
template <bool WAKE, bool N32, bool WIN>
__device__ __forceinline__ void finish_deferred(const PassArgs& a, const FusedConst& c,
                                                const GridConst& g, const PassWindow& kw,
                                                double pmean, int64_t turn, int64_t i,
                                                const double2* s_zt, const double2* s_rf,
                                                uint32_t* s_ngp, uint32_t* s_lo,
                                                uint32_t* s_hi, double& acc_z, double& acc_z2,
                                                double& acc_d, int32_t& n_in) {
  const double z0 = __ldcg(a.z + i), e0 = __ldcg(a.dE + i);
  double kick = 0.0;
  if (WAKE) {
    const KickFetch kf = kick_fetch(z0, g, kw, a.potd);
    kick = fma(kf.w, kf.d, kf.p0);
  }
  const int64_t pr = (i >> 1) + a.pair_offset;
  const int h = (int)(i & 1);
  uint32_t w[4] = {(uint32_t)pr, (uint32_t)((uint64_t)pr >> 32), (uint32_t)turn,
                   (uint32_t)((uint64_t)turn >> 32)};
  philox4x32_10(w, a.philox);
  const uint32_t whi = h ? w[3] : w[1], wlo = h ? w[2] : w[0];
  double xg;
  zig_fast(whi, wlo, s_zt, xg);
  const double rf = rf_term<true>(z0, c, s_rf);
  double zg = z0, eg = e0, dg = 0.0;
  particle_turn<WAKE, true>(zg, eg, xg, kick, rf, c, pmean, dg);
  const double r = zig_slow(a.seed, turn, pr, h, whi, wlo, &g_normal);
  double z1[1] = {z0};
  double e1 = e0, d1 = 0.0;
  particle_turn<WAKE, true>(z1[0], e1, r, kick, rf, c, pmean, d1);
  acc_d = __dadd_rn(__dsub_rn(acc_d, dg), d1);
  if (WAKE) {
    undeposit<N32>(zg, g, kw, acc_z, acc_z2, n_in, s_ngp, s_lo, s_hi, a.hist_spill);
    deposit_group<1, N32, WIN>(z1, g, kw, acc_z, acc_z2, n_in, s_ngp, s_lo, s_hi,
                               a.hist_spill);
  }
  a.z[i] = z1[0];
  a.dE[i] = e1;
}

// Moves the particles whose bit is set in the lanes' `pend` (bit k PPT + j:
// particle j of the group k iterations before `qref`) into the warp's
// staging queue wq (kDeferStage indices in global memory, `staged` of them
// held; each lane's entries after those of the lanes below it, by a prefix
// over the lanes' counts), and finishes them 32 at a time (finish_deferred)
// -- all of them when `last`, else only full waves, the rest staying queued.
// Every lane of the warp must take part.
template <bool WAKE, int PPT, bool N32, bool WIN>
__device__ __forceinline__ void drain_deferred(const PassArgs& a, const FusedConst& c,
                                               const GridConst& g, const PassWindow& kw,
                                               double pmean, int64_t turn, int64_t qref,
                                               int64_t stride, unsigned long long& pend,
                                               int64_t* wq, int& staged, bool last,
                                               const double2* s_zt, const double2* s_rf,
                                               uint32_t* s_ngp, uint32_t* s_lo, uint32_t* s_hi,
                                               double& acc_z, double& acc_z2, double& acc_d,
                                               int32_t& n_in) {
  const int lane = threadIdx.x & 31;
  for (;;) {
    const int cnt = __popcll(pend);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int space = kDeferStage - staged;
    int slot = staged + incl - cnt;
    while (pend && slot < kDeferStage) {
      const int b = __ffsll(pend) - 1;
      wq[slot++] = (int64_t)PPT * (qref - (int64_t)(b / PPT) * stride) + (b % PPT);
      pend &= pend - 1ull;
    }
    staged += min(total, space);
    __syncwarp();
    while (staged >= 32 || (last && staged > 0)) {
      const int n = min(staged, 32);
      staged -= n;
      if (lane < n)
        finish_deferred<WAKE, N32, WIN>(a, c, g, kw, pmean, turn, __ldcg(wq + staged + lane), s_zt,
                                   s_rf, s_ngp, s_lo, s_hi, acc_z, acc_z2, acc_d, n_in);
      __syncwarp();
    }
    if (total <= space) break;
  }
}

template <bool WAKE, int QE, int PPT, int THREADS, bool PREFETCH, bool N32 = false,
          bool WIN = false>
__device__ __forceinline__ void pass_body(const PassArgs& a, const PassRange& rg,
                                          unsigned char* smem_raw) {
  // dynamic shared memory: RF table [128] | the ziggurat's rows [2048] (a.zig) |
  // kick-table window [win] | NGP counters | cell words lo, hi [hot] for the
  // hot window's `hot` bins and cells; NGP counters: (hot+1)/2 words of two
  // 16-bit counters, or hot 32-bit ones (N32)
  const int nc = a.B + 1;                 // kick-table cells
  const int hot = WAKE ? a.hwin : 0;
  const int nw = N32 ? hot : (hot + 1) / 2;
  const int win = WAKE ? a.win : 0;
  double2* s_rf = reinterpret_cast<double2*>(smem_raw);
  double2* s_zt = s_rf + kRfTableSize;
  double* s_win = reinterpret_cast<double*>(
      smem_raw + (a.zig ? kPassTableBytes : kRfTableSize * sizeof(double2)));
  uint32_t* const h_ngp = reinterpret_cast<uint32_t*>(s_win + win);
  uint32_t* const h_lo = h_ngp + nw;
  uint32_t* const h_hi = h_lo + hot;
  for (int i = threadIdx.x; i < kRfTableSize; i += THREADS) s_rf[i] = __ldg(a.rf_table + i);
  if (QE == QE_PHILOX)
    for (int i = threadIdx.x; i < kZigLayers; i += THREADS)
      s_zt[i] = reinterpret_cast<const double2*>(g_normal.xd)[i];

  TurnState* ts = a.ts;
  const TurnScalars sc = ts->cur;
  const double pmean = ts->pending ? ts->pending_mean : 0.0;
  const int64_t turn = ts->turn;

  FusedConst c;
  c.Vs = a.Vs;
  c.rf_inv_h = a.rf_inv_h;
  c.rf_h_hi = a.rf_h_hi;
  c.rf_h_lo = a.rf_h_lo;
  c.k = sc.k;
  c.excitation = sc.excitation;
  c.damping = a.sr ? sc.damping : 1.0;
  c.gamma0 = sc.gamma0;
  c.inv_mass = a.inv_mass;
  c.alpha_c = a.alpha_c;
  c.Kz = sc.Kz;
  c.coeff0z = sc.drift_ok ? sc.coeff0z : 0.0;
  c.drift_ok = sc.drift_ok;
  c.update_eta = a.update_eta;
  GridConst g{a.B, a.e0, a.eN, a.inv_estep, a.c1, a.cB, a.inv_cstep,
              kick_offset(a.e0, a.inv_estep)};

  const double* drow = nullptr;
  if (QE == QE_DRAWS) {
    int64_t row = turn - a.draws_first_turn;
    if (row >= 0 && row < a.draws_turns) {
      drow = a.draws + row * a.n;
    } else if (rg.part == 0 && threadIdx.x == 0) {
      atomicOr(&ts->status, 1 << HJ_ERR_ARG);
    }
  }

  // windows centred on the cell of the last turn's mean z: histogram cells
  // w0 .. w0 + hot - 1 (never beyond cell B) and kick-table entries w0 .. w0 +
  // wv - 1 (wv <= win, never beyond cell B - 1)
  PassWindow kw{s_win, 0, 0u, 0u, 0u};
  if (WAKE) {
    for (int i = threadIdx.x; i < hot; i += THREADS) {
      if (i < nw) h_ngp[i] = 0u;
      h_lo[i] = 0u;
      h_hi[i] = 0u;
    }
    int w0 = 0;
    if (WIN && hot < nc) {   // even, so that the 16-bit pairs keep bin b at word b >> 1
      int jm;
      double wm;
      kick_cell(ts->last_mean_z, g, jm, wm);
      w0 = max(0, min(jm - hot / 2, nc - hot)) & ~1;
    }
    kw.w0 = w0;
    kw.h = (unsigned)hot;
    kw.inner = hot > 0 ? (unsigned)hot - 1u : 0u;
    if (win > 0) {
      const int wv = min(win, a.B - w0);
      for (int i = threadIdx.x; i < wv; i += THREADS) s_win[i] = a.potd[w0 + i].x;
      kw.lim = (unsigned)max(wv - 1, 0);
    }
  }
  __syncthreads();
  // the histograms indexed by absolute bin and cell (valid inside the window)
  uint32_t* const s_ngp = h_ngp - (N32 ? kw.w0 : kw.w0 / 2);
  uint32_t* const s_lo = h_lo - kw.w0;
  uint32_t* const s_hi = h_hi - kw.w0;

  double acc_z = 0.0, acc_z2 = 0.0, acc_d = 0.0;
  int32_t n_in = 0;
  const double2* __restrict__ potd = a.potd;
  const int64_t ng = rg.q_end;
  const int64_t stride = rg.q_step;
  int64_t q = rg.q_begin + threadIdx.x;
  constexpr bool kPrefetch = PREFETCH;
  double zn[PPT], en[PPT];
  if (kPrefetch && q < ng) {
    ldp<PPT>(a.z + PPT * q, zn);
    ldp<PPT>(a.dE + PPT * q, en);
  }
  // With the Float64 normals (QE_PHILOX), a particle whose draw fails the
  // ziggurat's fast test (about 0.23 %) is turned and deposited like the
  // others with its rejected candidate but stored as loaded, and its bit set in
  // its lane's history `pend`; every 16 iterations (and at the end) the warp
  // moves those particles to its staging queue and finishes them 32 at a time
  // (drain_deferred), so that the slow path runs on full warps and this loop
  // carries no per-particle branches.
  constexpr bool kDefer = QE == QE_PHILOX;
  unsigned long long pend = 0ull;
  int it = 0, staged = 0;
  int64_t* wq = kDefer ? a.defer_q + ((int64_t)rg.part * (THREADS / 32) + (threadIdx.x >> 5)) *
                                         kDeferStage
                       : nullptr;
  for (; q < ng; q += stride, ++it) {
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
    KickFetch kf[PPT];
    if (WAKE) {
#pragma unroll
      for (int j = 0; j < PPT; ++j) kf[j] = kick_fetch(zz[j], g, kw, potd);
    }
#pragma unroll
    for (int j = 0; j < PPT; ++j) rr[j] = 0.0;
    unsigned ok = (1u << PPT) - 1u;
    if (QE == QE_PHILOX) {
      ok = group_normals_zig<PPT>(a.philox, turn, (PPT / 2) * q + a.pair_offset, s_zt, rr);
    } else if (QE == QE_PHILOX_FAST) {
      group_normals_fast<PPT>(a.philox, turn, (PPT / 2) * q + a.pair_offset, rr);
    } else if (QE == QE_DRAWS) {
      if (drow) {
#pragma unroll
        for (int j = 0; j < PPT; ++j) rr[j] = __ldg(drow + PPT * q + j);
      }
    }
    double rf[PPT];
#pragma unroll
    for (int j = 0; j < PPT; ++j) rf[j] = rf_term<kDefer>(zz[j], c, s_rf);
    double zs[PPT], es[PPT];               // what is stored
#pragma unroll
    for (int j = 0; j < PPT; ++j) {
      const double z0 = zz[j], e0 = ee[j];
      particle_turn<WAKE, kDefer>(zz[j], ee[j], rr[j],
                                  WAKE ? fma(kf[j].w, kf[j].d, kf[j].p0) : 0.0, rf[j], c, pmean,
                                  acc_d);
      const bool keep = kDefer && !((ok >> j) & 1u);
      zs[j] = keep ? z0 : zz[j];
      es[j] = keep ? e0 : ee[j];
    }
    if (WAKE)
      deposit_group<PPT, N32, WIN>(zz, g, kw, acc_z, acc_z2, n_in, s_ngp, s_lo, s_hi, a.hist_spill);
    stp<PPT>(a.z + PPT * q, zs);
    stp<PPT>(a.dE + PPT * q, es);
    if (kDefer) {
      pend = (pend << PPT) | (unsigned long long)(~ok & ((1u << PPT) - 1u));
      if ((it & 15) == 15 && __activemask() == 0xffffffffu)
        drain_deferred<WAKE, PPT, N32, WIN>(a, c, g, kw, pmean, turn, q, stride, pend, wq, staged,
                                       false, s_zt, s_rf, s_ngp, s_lo, s_hi, acc_z, acc_z2,
                                       acc_d, n_in);
    }
  }
  if (kDefer) {
    __syncwarp();
    staged = __reduce_max_sync(0xffffffffu, (unsigned)staged);
    drain_deferred<WAKE, PPT, N32, WIN>(a, c, g, kw, pmean, turn, q - stride, stride, pend, wq, staged,
                                   true, s_zt, s_rf, s_ngp, s_lo, s_hi, acc_z, acc_z2, acc_d,
                                   n_in);
  }
  // Tail of n % PPT particles: the first threads of the tail block, scalar.
  if (rg.tail && threadIdx.x < (int)(a.n % PPT)) {
    const int64_t i = (a.n / PPT) * PPT + threadIdx.x;
    double r2[2] = {0.0, 0.0};
    if (QE == QE_PHILOX)
      philox_normals2_rk(a.seed, a.philox, turn, (i >> 1) + a.pair_offset, &g_normal, s_zt, r2);
    if (QE == QE_PHILOX_FAST) philox_normals2_fast(a.philox, turn, (i >> 1) + a.pair_offset, r2);
    double r = r2[i & 1];
    if (QE == QE_DRAWS) r = drow ? __ldg(drow + i) : 0.0;
    double z1[1] = {a.z[i]};
    double e = a.dE[i];
    const double kick = WAKE ? wake_kick(z1[0], g, potd) : 0.0;
    particle_turn<WAKE, kDefer>(z1[0], e, r, kick, rf_term<kDefer>(z1[0], c, s_rf), c, pmean,
                               acc_d);
    if (WAKE)
      deposit_group<1, N32, WIN>(z1, g, kw, acc_z, acc_z2, n_in, s_ngp, s_lo, s_hi, a.hist_spill);
    a.z[i] = z1[0];
    a.dE[i] = e;
  }

  __syncthreads();                        // the RF table's space becomes the reduction scratch
  static_assert(THREADS / 32 * 4 * sizeof(double) <= kRfTableSize * sizeof(double2),
                "reduction scratch exceeds the RF table");
  block_sum4<THREADS>(acc_z, acc_z2, acc_d, (double)n_in,
                      a.part_sum + (size_t)rg.part * kNumSums,
                      reinterpret_cast<double(*)[4]>(s_rf));

  if (WAKE) {
    __syncthreads();
    uint32_t* pc = a.part_cnt + (size_t)rg.part * a.B;
    unsigned long long* pq = a.part_cic + (size_t)rg.part * nc;
    for (int i = threadIdx.x; i < nc; i += THREADS) {   // zeros outside the hot window
      const unsigned r = (unsigned)(i - kw.w0);
      const bool in = r < kw.h;
      if (i < a.B)
        pc[i] = !in ? 0u : N32 ? h_ngp[r] : (h_ngp[r >> 1] >> ((r & 1) << 4)) & 0xFFFFu;
      pq[i] = in ? ((unsigned long long)h_hi[r] << 32) | h_lo[r] : 0ull;
    }
  }
}

// One turn over one bunch: block b takes groups b, b + grid, ... (THREADS
// apart) and writes partial slot b; block 0 takes the tail.  WIN: the hot
// window holds fewer than all cells (kPassWindowed).
template <bool WAKE, int QE, int PPT, int THREADS, bool PREFETCH, int MINB = 1, bool N32 = false,
          bool WIN = false>
__global__ void __launch_bounds__(THREADS, MINB) k_track_pass(PassArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  grid_dependency_wait();
  if (WAKE) {  // zero the merged histograms k_hist_reduce accumulates into this turn
    const int gstride = gridDim.x * THREADS;
    for (int i = blockIdx.x * THREADS + threadIdx.x; i < 3 * a.B + 2; i += gstride)
      a.hist_out[i] = 0ull;
  }
  const PassRange rg{(int64_t)blockIdx.x * THREADS, (int64_t)gridDim.x * THREADS, a.n / PPT,
                     (int32_t)blockIdx.x, blockIdx.x == 0};
  pass_body<WAKE, QE, PPT, THREADS, PREFETCH, N32, WIN>(a, rg, smem_raw);
}

// One turn over a batch of bunches.  Chunk c of the chunk table (a
// contiguous run of one bunch's particles) is processed by one block into the
// bunch's partial slot ch.part; chunks of bunches with no turns left are
// skipped.  Without QUEUE, block c takes chunk c (blocks past the table's
// length return at once).  With QUEUE (the turn's counter, zero at launch),
// the blocks are resident -- one per SM slot -- and each takes the next
// chunk index from the counter until the table is exhausted.  Either way a
// chunk's arithmetic and slot do not depend on the block that takes it.  The
// two are separate instantiations: around the inlined pass body the loop of
// the queued form costs about 300 bytes of register spills per thread
// (ptxas, 4 x 512 layout), which the one-chunk form does not pay.
template <bool WAKE, int QE, int PPT, int THREADS, bool PREFETCH, int MINB = 1, bool N32 = false,
          bool QUEUE = false, bool WIN = false>
__global__ void __launch_bounds__(THREADS, MINB)
    k_batch_pass(const PassArgs* __restrict__ bunches, const BatchChunk* __restrict__ chunks,
                 const int32_t* __restrict__ n_chunks, int32_t* queue) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ int s_chunk;
  const int nch = *n_chunks;
  int c = (int)blockIdx.x;
  if (QUEUE) {
    if (threadIdx.x == 0) s_chunk = atomicAdd(queue, 1);
    __syncthreads();
    c = s_chunk;
  }
  while (c < nch) {
    const BatchChunk ch = chunks[c];
    const PassArgs a = bunches[ch.bunch];
    if (a.ts->turns_left > 0) {
      if (WAKE && ch.part == 0) {  // zero the merged histograms k_batch_reduce adds into
        for (int i = threadIdx.x; i < 3 * a.B + 2; i += THREADS) a.hist_out[i] = 0ull;
      }
      const PassRange rg{ch.first / PPT, THREADS, (ch.first + ch.count) / PPT, ch.part,
                         ch.first + ch.count == a.n};
      pass_body<WAKE, QE, PPT, THREADS, PREFETCH, N32, WIN>(a, rg, smem_raw);
    }
    if (!QUEUE) break;
    __syncthreads();                   // the chunk's shared memory is read no more
    if (threadIdx.x == 0) s_chunk = atomicAdd(queue, 1);
    __syncthreads();
    c = s_chunk;
  }
}

// Merge of the per-block histograms.  Grid (bins/256, G): block column g sums
// the partials of blocks g, g+G, ... and adds them to the merged arrays with
// integer atomics (exact, so the result does not depend on their order).
// out layout (u64): counts[B] | cell counts[B+1] | cell Σw·2^24 [B+1].
// spill (optional): the pass's deposits outside its hot window and beyond its
// 16-bit counters, in out's layout (counts only without part_cic); folded in
// and cleared for the next turn.
__global__ void k_hist_reduce(const uint32_t* __restrict__ part_cnt,
                              const unsigned long long* __restrict__ part_cic, int nblk, int B,
                              unsigned long long* __restrict__ out,
                              unsigned long long* __restrict__ spill) {
  grid_dependency_wait();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int nc = B + 1;
  if (b >= (part_cic ? nc : B)) return;
  unsigned long long sc = 0ull, sn = 0ull, sw = 0ull;
  if (spill && blockIdx.y == 0) {
    if (b < B) {
      sc = spill[b];
      if (sc) spill[b] = 0ull;
    }
    if (part_cic) {
      sn = spill[B + b];
      sw = spill[B + nc + b];
      if (sn) spill[B + b] = 0ull;
      if (sw) spill[B + nc + b] = 0ull;
    }
  }
  for (int k = blockIdx.y; k < nblk; k += gridDim.y) {
    if (b < B) sc += __ldg(part_cnt + (size_t)k * B + b);
    if (part_cic) {
      const unsigned long long v = __ldg(part_cic + (size_t)k * nc + b);
      sn += v >> kCicSumBits;
      sw += v & kCicSumMask;
    }
  }
  if (sc) atomicAdd(out + b, sc);
  if (part_cic) {
    if (sn) atomicAdd(out + B + b, sn);
    if (sw) atomicAdd(out + B + nc + b, sw);
  }
}

// Merge of a batch's per-chunk histograms: block (x, i) takes item i of the
// merge table -- partial slots [first, first + count) of one bunch -- sums
// them for 256 cells and adds the sums to the merged arrays (zeroed by the
// bunch's first chunk in the pass) with integer atomics: exact, so neither
// the items' order nor their grouping matters.
__global__ void k_batch_reduce(const PassArgs* __restrict__ bunches,
                               const BatchChunk* __restrict__ items,
                               const int32_t* __restrict__ n_items) {
  if ((int)blockIdx.y >= *n_items) return;
  const BatchChunk it = items[blockIdx.y];
  const PassArgs& a = bunches[it.bunch];
  if (a.ts->turns_left <= 0 || !a.use_wake) return;
  const int B = a.B, nc = B + 1;
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nc) return;
  unsigned long long sc = 0ull, sn = 0ull, sw = 0ull;
  if (it.first == 0) {   // the spill histograms, once per bunch
    unsigned long long* sp = a.hist_spill;
    if (b < B) {
      sc = sp[b];
      if (sc) sp[b] = 0ull;
    }
    sn = sp[B + b];
    sw = sp[B + nc + b];
    if (sn) sp[B + b] = 0ull;
    if (sw) sp[B + nc + b] = 0ull;
  }
  for (int64_t k = it.first; k < it.first + it.count; ++k) {
    if (b < B) sc += __ldg(a.part_cnt + (size_t)k * B + b);
    const unsigned long long v = __ldg(a.part_cic + (size_t)k * nc + b);
    sn += v >> kCicSumBits;
    sw += v & kCicSumMask;
  }
  if (sc) atomicAdd(a.hist_out + b, sc);
  if (sn) atomicAdd(a.hist_out + B + b, sn);
  if (sw) atomicAdd(a.hist_out + B + nc + b, sw);
}

// Pending kick + re-centring (optional), copy-out (optional) and the moments
// [Σz, Σz², ΣdE, ΣdE²] per block.
__global__ void __launch_bounds__(kTrackThreads) k_flush(FlushArgs a) {
  const bool apply = a.apply && a.ts && a.ts->pending;
  const double pmean = apply ? a.ts->pending_mean : 0.0;
  GridConst g{a.B, a.e0, 0.0, a.inv_estep, a.c1, a.cB, a.inv_cstep,
              kick_offset(a.e0, a.inv_estep)};
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
  __shared__ double red[kTrackThreads / 32][4];
  block_sum4<kTrackThreads>(s0, s1, s2, s3, a.part + (size_t)blockIdx.x * 4, red);
}

// One record of a bunch's turn log: [turn, E0, σ_z, σ_E, mean z, mean ΔE, wake
// current, particles in the bins] of the state after the last completed turn
// (moments from k_flush with the pending kick applied), then the B bin
// counts of that turn when `counts` is given.
__global__ void k_log_record(const double* __restrict__ part, int nblk, int64_t n,
                             const TurnState* __restrict__ ts,
                             const unsigned long long* __restrict__ counts, int B,
                             double* __restrict__ rec) {
  if (threadIdx.x == 0) {
    double s[4] = {0.0, 0.0, 0.0, 0.0};
    for (int b = 0; b < nblk; ++b)
      for (int k = 0; k < 4; ++k) s[k] += part[(size_t)b * 4 + k];
    const double nd = n > 0 ? (double)n : 1.0;
    rec[0] = (double)(ts->turn - 1);
    rec[1] = ts->cur.E0;
    rec[2] = global_std_of_sums(s[0], s[1], n);
    rec[3] = global_std_of_sums(s[2], s[3], n);
    rec[4] = s[0] / nd;
    rec[5] = s[2] / nd;
    rec[6] = ts->last_current;
    rec[7] = ts->last_n_in;
  }
  if (counts)
    for (int i = threadIdx.x; i < B; i += blockDim.x) rec[kLogHeader + i] = (double)counts[i];
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
    int j = ngp_bin_any(__ldg(z + i), g, in);
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
  const int64_t np = (n + 1) >> 1;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += stride) {
    double rr[2];
    if (!draws) philox_normals2(seed, turn, p, rr);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const int64_t i = 2 * p + j;
      if (i < n) {
        const double r = draws ? __ldg(draws + i) : rr[j];
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
  const int64_t np = (n + 1) >> 1;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += stride) {
    double rr[2];
    philox_normals2(seed, turn, p, rr);
    out[2 * p] = rr[0];
    if (2 * p + 1 < n) out[2 * p + 1] = rr[1];
  }
}

// Independent Gaussian bunch: particle i gets the Philox pair (i, turn 0) of
// seed ^ kInitTag (turn 0 is never a tracking turn, and the tag keeps the
// stream apart from the quantum-excitation one of the same seed).
constexpr uint64_t kInitTag = 0x6A09E667F3BCC909ull;
__global__ void k_gaussian_bunch(uint64_t seed, int64_t n, double mu_z, double sigma_z,
                                 double mu_E, double sigma_E, double* __restrict__ z,
                                 double* __restrict__ dE) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double rr[2];
    philox_normals2(seed ^ kInitTag, 0, i, rr);
    z[i] = fma(sigma_z, rr[0], mu_z);
    dE[i] = fma(sigma_E, rr[1], mu_E);
  }
}

// ---- generate_particles (src/evolution.jl:42-133) on the device
constexpr uint64_t kSampleTag = 0xBB67AE8584CAA73Bull;   // covariance-estimate sample
constexpr uint64_t kCorrTag = 0x3C6EF372FE94F82Bull;     // the bunch itself

__device__ __forceinline__ double block_sum_1024(double v, double* red) {
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  return s;
}

// Sample covariance (two-pass, divisor S - 1) of S independent draws
// z ~ N(mu_z, sz), E ~ N(mu_E, sE): out = (cov zz, cov EE, cov zE).  One block.
__global__ void __launch_bounds__(1024) k_gen_sample_cov(uint64_t seed, int64_t S, double mu_z, double sz, double mu_E,
                                 double sE, double* __restrict__ out) {
  __shared__ double red[32];
  double a = 0.0, b = 0.0;
  for (int64_t i = threadIdx.x; i < S; i += blockDim.x) {
    double r[2];
    philox_normals2(seed ^ kSampleTag, 0, i, r);
    a += fma(sz, r[0], mu_z);
    b += fma(sE, r[1], mu_E);
  }
  const double mz = block_sum_1024(a, red) / (double)S;
  const double mE = block_sum_1024(b, red) / (double)S;
  double czz = 0.0, cEE = 0.0, czE = 0.0;
  for (int64_t i = threadIdx.x; i < S; i += blockDim.x) {
    double r[2];
    philox_normals2(seed ^ kSampleTag, 0, i, r);
    const double dz = fma(sz, r[0], mu_z) - mz, dEv = fma(sE, r[1], mu_E) - mE;
    czz = fma(dz, dz, czz);
    cEE = fma(dEv, dEv, cEE);
    czE = fma(dz, dEv, czE);
  }
  czz = block_sum_1024(czz, red);
  cEE = block_sum_1024(cEE, red);
  czE = block_sum_1024(czE, red);
  if (threadIdx.x == 0) {
    out[0] = czz / (double)(S - 1);
    out[1] = cEE / (double)(S - 1);
    out[2] = czE / (double)(S - 1);
  }
}

// (z, E) = mu + L eps with L = [[l00, 0], [l10, l11]] (the bunch's MvNormal draw).
__global__ void k_gen_correlated(uint64_t seed, int64_t n, double mu_z, double mu_E, double l00,
                                 double l10, double l11, double* __restrict__ z,
                                 double* __restrict__ dE) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    double r[2];
    philox_normals2(seed ^ kCorrTag, 0, i, r);
    z[i] = fma(l00, r[0], mu_z);
    dE[i] = fma(l11, r[1], fma(l10, r[0], mu_E));
  }
}

// Per-block sums for compute_std (src/utils.jl:531-544): of x (first pass,
// mean = NaN) or of (x - mean)^2 (second pass).
__global__ void k_std_parts(const double* __restrict__ x, int64_t n, double mean, int second,
                            double* __restrict__ part) {
  __shared__ double red[32];
  double s = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double v = x[i];
    if (second) {
      const double d = v - mean;
      s = fma(d, d, s);
    } else {
      s += v;
    }
  }
  s = block_sum_1024(s, red);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// Per-block sums for the Pearson correlation of (x, y): first pass [Σx, Σy];
// second pass [Σ(x-mx)², Σ(y-my)², Σ(x-mx)(y-my)] (Statistics.cor, two-pass).
// part: 3 doubles per block.
__global__ void k_cor_parts(const double* __restrict__ x, const double* __restrict__ y,
                            int64_t n, double mx, double my, int second,
                            double* __restrict__ part) {
  __shared__ double red[32];
  double a = 0.0, b = 0.0, c = 0.0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const double u = x[i], v = y[i];
    if (second) {
      const double du = u - mx, dv = v - my;
      a = fma(du, du, a);
      b = fma(dv, dv, b);
      c = fma(du, dv, c);
    } else {
      a += u;
      b += v;
    }
  }
  a = block_sum_1024(a, red);
  b = block_sum_1024(b, red);
  c = block_sum_1024(c, red);
  if (threadIdx.x == 0) {
    part[3 * (size_t)blockIdx.x] = a;
    part[3 * (size_t)blockIdx.x + 1] = b;
    part[3 * (size_t)blockIdx.x + 2] = c;
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
// cfg: thread layout (bits 0-2) | kPassN32 (32-bit NGP counters) |
// kPassFastNormals | kPassWindowed (range-checked deposits; with the wake only)
template <bool W, int Q, bool N, bool H>
const void* pass_fn_wqnh(int layout) {
  switch (layout) {
    case 0: return (const void*)k_track_pass<W, Q, 4, 512, true, 1, N, H>;
    case 1: return (const void*)k_track_pass<W, Q, 2, 1024, true, 1, N, H>;
    case 2: return (const void*)k_track_pass<W, Q, 2, 768, true, 1, N, H>;
    case 4: return (const void*)k_track_pass<W, Q, 2, 512, true, 2, N, H>;
    case 5: return (const void*)k_track_pass<W, Q, 4, 256, true, 2, N, H>;
    default: return (const void*)k_track_pass<W, Q, 2, 512, false, 1, N, H>;
  }
}

template <bool W, int Q, bool N>
const void* pass_fn_wqn(int cfg) {
  if constexpr (W) {   // without the wake nothing is deposited: one form
    if (cfg & kPassWindowed) return pass_fn_wqnh<W, Q, N, true>(cfg & kPassLayoutMask);
  }
  return pass_fn_wqnh<W, Q, N, false>(cfg & kPassLayoutMask);
}

template <bool W, int Q>
const void* pass_fn_wq(int cfg) {
  if constexpr (W) {
    if (cfg & kPassN32) return pass_fn_wqn<W, Q, true>(cfg);
  }
  return pass_fn_wqn<W, Q, false>(cfg);
}

template <bool W>
const void* pass_fn_w(int qe, int cfg) {
  switch (qe) {
    case QE_PHILOX:
      return (cfg & kPassFastNormals) ? pass_fn_wq<W, QE_PHILOX_FAST>(cfg)
                                      : pass_fn_wq<W, QE_PHILOX>(cfg);
    case QE_DRAWS: return pass_fn_wq<W, QE_DRAWS>(cfg);
    default: return pass_fn_wq<W, QE_OFF>(cfg);
  }
}

const void* pass_fn(int wake, int qe, int cfg) {
  return wake ? pass_fn_w<true>(qe, cfg) : pass_fn_w<false>(qe, cfg);
}

template <bool W, int Q, bool N, bool U, bool H>
const void* batch_fn_wqnuh(int layout) {
  switch (layout) {
    case 0: return (const void*)k_batch_pass<W, Q, 4, 512, true, 1, N, U, H>;
    case 1: return (const void*)k_batch_pass<W, Q, 2, 1024, true, 1, N, U, H>;
    case 2: return (const void*)k_batch_pass<W, Q, 2, 768, true, 1, N, U, H>;
    case 4: return (const void*)k_batch_pass<W, Q, 2, 512, true, 2, N, U, H>;
    case 5: return (const void*)k_batch_pass<W, Q, 4, 256, true, 2, N, U, H>;
    default: return (const void*)k_batch_pass<W, Q, 2, 512, false, 1, N, U, H>;
  }
}

template <bool W, int Q, bool N, bool U>
const void* batch_fn_wqnu(int cfg) {
  if constexpr (W) {
    if (cfg & kPassWindowed) return batch_fn_wqnuh<W, Q, N, U, true>(cfg & kPassLayoutMask);
  }
  return batch_fn_wqnuh<W, Q, N, U, false>(cfg & kPassLayoutMask);
}

template <bool W, int Q, bool U>
const void* batch_fn_wqu(int cfg) {
  if constexpr (W) {
    if (cfg & kPassN32) return batch_fn_wqnu<W, Q, true, U>(cfg);
  }
  return batch_fn_wqnu<W, Q, false, U>(cfg);
}

// Batches draw QE normals on the device or not at all (no host-fed draws).
template <bool W, bool U>
const void* batch_fn_wu(int qe, int cfg) {
  if (qe != QE_PHILOX) return batch_fn_wqu<W, QE_OFF, U>(cfg);
  return (cfg & kPassFastNormals) ? batch_fn_wqu<W, QE_PHILOX_FAST, U>(cfg)
                                  : batch_fn_wqu<W, QE_PHILOX, U>(cfg);
}

// The batched pass for (wake, excitation mode, configuration), one block per
// chunk or resident blocks on a chunk queue.
const void* batch_fn(int wake, int qe, int cfg, bool queue) {
  if (queue) return wake ? batch_fn_wu<true, true>(qe, cfg) : batch_fn_wu<false, true>(qe, cfg);
  return wake ? batch_fn_wu<true, false>(qe, cfg) : batch_fn_wu<false, false>(qe, cfg);
}
}  // namespace

namespace {
// Grids up to this many bins read the kick table from global memory (L1).
constexpr int kWindowMinBins = 4096;


// Dynamic shared memory one block of the pass may take: the device's opt-in
// limit (set when the kernels are prepared), or per block of the layout that
// keeps two blocks on an SM (228 KB per SM, 1 KB reserved per block).
int g_pass_smem_limit = 227 * 1024;

// Static shared memory the pass kernels declare beside the dynamic part (the
// batched pass's chunk index and the reduction's alignment), kept out of the
// dynamic budget.
constexpr size_t kPassStaticSmem = 256;

size_t pass_smem_budget(int cfg) {
  const size_t lim = (size_t)g_pass_smem_limit - kPassStaticSmem;
  return pass_cfg_two_blocks(cfg) ? std::min(lim, (size_t)(113 * 1024)) : lim;
}

// The tables in shared memory: RF, and the ziggurat's rows when the pass draws
// the Float64 normals.
size_t pass_table_bytes(bool zig) {
  return zig ? kPassTableBytes : kRfTableSize * sizeof(double2);
}

}  // namespace

// The pass's hot window for B bins: per cell a pair of cell words (8 bytes),
// an NGP counter (4 bytes, or 2 with 16-bit pairs) and, above kWindowMinBins
// bins, a kick-table entry (8 bytes), as many cells as the shared-memory
// budget leaves beside the tables, at most B + 1 (up to 4096 bins the 64 KB
// kick table stays in L1 beside the histograms: a kick window would only add
// its load to every block, measured no gain).
PassWindows track_windows(int B, int cfg, bool zig) {
  const size_t tables = pass_table_bytes(zig), budget = pass_smem_budget(cfg);
  const bool kick = B > kWindowMinBins;
  const size_t per = 8 + ((cfg & kPassN32) ? 4 : 2) + (kick ? 8 : 0);
  const size_t room = budget > tables + 4 ? budget - tables - 4 : 0;   // 4: an odd 16-bit word
  const size_t hot = std::min(room / per, (size_t)B + 1);
  PassWindows w;
  w.hot = (int)hot;
  w.kick = kick ? (int)std::min(hot, (size_t)B) : 0;
  return w;
}

// Tables, and with the wake the windows: kick-table entries, NGP counters and
// cell words of the hot window.
size_t track_smem_bytes(int B, int use_wake, int cfg, bool zig) {
  if (!use_wake) return pass_table_bytes(zig);
  const PassWindows w = track_windows(B, cfg, zig);
  const size_t nw = (cfg & kPassN32) ? (size_t)w.hot : (size_t)(w.hot + 1) / 2;
  return pass_table_bytes(zig) + (size_t)w.kick * sizeof(double) + nw * sizeof(uint32_t) +
         (size_t)w.hot * 2 * sizeof(uint32_t);
}

namespace {
bool pass_zig(int qe_mode, int cfg) { return qe_mode == QE_PHILOX && !(cfg & kPassFastNormals); }

// The configuration a pass over B bins is launched with: cfg, plus
// kPassWindowed where the hot window holds fewer than all B + 1 cells.
int launch_cfg(int B, int use_wake, int qe_mode, int cfg) {
  if (!use_wake) return cfg;
  const PassWindows w = track_windows(B, cfg, pass_zig(qe_mode, cfg));
  return w.hot < B + 1 ? (cfg | kPassWindowed) : cfg;
}
}  // namespace

cudaError_t prepare_track_kernels(int max_smem) {
  g_pass_smem_limit = max_smem;
  {
    std::unique_ptr<NormalTables> tab(new NormalTables);   // 48 KB: not on the stack
    host_normal_tables(tab.get());
    cudaError_t e = cudaMemcpyToSymbol(g_normal, tab.get(), sizeof(NormalTables));
    if (e != cudaSuccess) return e;
  }
  for (int w = 0; w < 2; ++w)
    for (int q = 0; q < 3; ++q)
      for (int n = 0; n < 2; ++n)
        for (int f = 0; f < 2; ++f)
          for (int h = 0; h < 2; ++h)
            for (int l = 0; l < kNumPassCfgs; ++l) {
              const int c = l | (n ? kPassN32 : 0) | (f ? kPassFastNormals : 0) |
                            (h ? kPassWindowed : 0);
              cudaError_t e = allow_dynamic_smem(pass_fn(w, q, c), max_smem);
              for (int u = 0; u < 2 && e == cudaSuccess && q != QE_DRAWS; ++u)
                e = allow_dynamic_smem(batch_fn(w, q, c, u != 0), max_smem);
              if (e != cudaSuccess) return e;
            }
  return allow_dynamic_smem((const void*)k_histogram, max_smem);
}


int track_blocks_per_sm(int B, int qe_mode, int use_wake, int cfg) {
  const size_t smem = track_smem_bytes(B, use_wake, cfg, pass_zig(qe_mode, cfg));
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &bps, pass_fn(use_wake, qe_mode, launch_cfg(B, use_wake, qe_mode, cfg)),
          pass_cfg_threads(cfg), smem) != cudaSuccess)
    bps = 1;
  return bps < 1 ? 1 : bps;
}

cudaError_t launch_track_pass(const PassArgs& a, int grid, cudaStream_t st) {
  const size_t smem = track_smem_bytes(a.B, a.use_wake, a.cfg, a.zig != 0);
  void* args[] = {const_cast<PassArgs*>(&a)};
  PdlConfig l(dim3(grid), dim3(pass_cfg_threads(a.cfg)), smem, st);
  const int cfg = a.use_wake && a.hwin < a.B + 1 ? (a.cfg | kPassWindowed) : a.cfg;
  return cudaLaunchKernelExC(&l.cfg, pass_fn(a.use_wake, a.qe_mode, cfg), args);
}

cudaError_t launch_batch_pass(const PassArgs* d_bunches, const BatchChunk* d_chunks,
                              const int32_t* d_n_chunks, int max_chunks, int max_B, int wake,
                              int qe, int cfg, int32_t* d_queue, int resident_blocks,
                              cudaStream_t st) {
  const size_t smem = track_smem_bytes(max_B, wake, cfg, pass_zig(qe, cfg));
  void* args[] = {const_cast<PassArgs**>(&d_bunches), const_cast<BatchChunk**>(&d_chunks),
                  const_cast<int32_t**>(&d_n_chunks), &d_queue};
  int grid = max_chunks > 0 ? max_chunks : 1;
  if (d_queue) {
    cudaError_t e = cudaMemsetAsync(d_queue, 0, sizeof(int32_t), st);
    if (e != cudaSuccess) return e;
    grid = std::max(1, std::min(grid, resident_blocks));
  }
  return cudaLaunchKernel(batch_fn(wake, qe, launch_cfg(max_B, wake, qe, cfg), d_queue != nullptr),
                          dim3(grid), dim3(pass_cfg_threads(cfg)), args, smem, st);
}

int batch_blocks_per_sm(int max_B, int qe_mode, int use_wake, int cfg) {
  const size_t smem = track_smem_bytes(max_B, use_wake, cfg, pass_zig(qe_mode, cfg));
  int bps = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
          &bps, batch_fn(use_wake, qe_mode, launch_cfg(max_B, use_wake, qe_mode, cfg), true),
          pass_cfg_threads(cfg), smem) != cudaSuccess)
    bps = 1;
  return bps < 1 ? 1 : bps;
}

// Fixed-order sum of nblk per-block sum vectors into out[kNumSums] (one block).
__global__ void k_sum_parts(const double* __restrict__ part, int nblk, double* __restrict__ out) {
  if (threadIdx.x < kNumSums) {
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[(size_t)b * kNumSums + threadIdx.x];
    out[threadIdx.x] = s;
  }
}

cudaError_t launch_sum_parts(const double* part, int nblk, double* out, cudaStream_t st) {
  k_sum_parts<<<1, 32, 0, st>>>(part, nblk, out);
  return cudaGetLastError();
}

cudaError_t launch_batch_reduce(const PassArgs* d_bunches, const BatchChunk* d_items,
                                const int32_t* d_n_items, int max_items, int max_B,
                                cudaStream_t st) {
  dim3 grid((max_B + 1 + 255) / 256, max_items > 0 ? max_items : 1);
  k_batch_reduce<<<grid, 256, 0, st>>>(d_bunches, d_items, d_n_items);
  return cudaGetLastError();
}

cudaError_t launch_hist_reduce(const uint32_t* part_cnt, const unsigned long long* part_cic,
                               int nblk, int B, unsigned long long* out, bool zero_first,
                               cudaStream_t st, unsigned long long* spill) {
  if (zero_first) {
    cudaError_t e = cudaMemsetAsync(
        out, 0, sizeof(unsigned long long) * (part_cic ? 3 * (size_t)B + 2 : (size_t)B), st);
    if (e != cudaSuccess) return e;
  }
  const int G = nblk < 16 ? nblk : 16;
  dim3 grid((B + 1 + 255) / 256, G > 0 ? G : 1);
  PdlConfig l(grid, dim3(256), 0, st);
  cudaError_t e = cudaLaunchKernelEx(&l.cfg, k_hist_reduce, part_cnt, part_cic, nblk, B, out,
                                     spill);
  if (e != cudaSuccess) return e;
  return cudaGetLastError();
}

cudaError_t launch_log_record(const double* part, int nblk, int64_t n, const TurnState* ts,
                              const unsigned long long* counts, int B, double* rec,
                              cudaStream_t st) {
  k_log_record<<<1, 256, 0, st>>>(part, nblk, n, ts, counts, B, rec);
  return cudaGetLastError();
}

cudaError_t launch_gen_sample_cov(uint64_t seed, int64_t S, double mu_z, double sz, double mu_E,
                                  double sE, double* out, cudaStream_t st) {
  k_gen_sample_cov<<<1, 1024, 0, st>>>(seed, S, mu_z, sz, mu_E, sE, out);
  return cudaGetLastError();
}

cudaError_t launch_gen_correlated(uint64_t seed, int64_t n, double mu_z, double mu_E, double l00,
                                  double l10, double l11, double* z, double* dE,
                                  cudaStream_t st) {
  k_gen_correlated<<<elementwise_grid(n), 256, 0, st>>>(seed, n, mu_z, mu_E, l00, l10, l11, z,
                                                        dE);
  return cudaGetLastError();
}

cudaError_t launch_std_parts(const double* x, int64_t n, double mean, int second, double* part,
                             int grid, cudaStream_t st) {
  k_std_parts<<<grid, 1024, 0, st>>>(x, n, mean, second, part);
  return cudaGetLastError();
}

cudaError_t launch_cor_parts(const double* x, const double* y, int64_t n, double mx, double my,
                             int second, double* part, int grid, cudaStream_t st) {
  k_cor_parts<<<grid, 1024, 0, st>>>(x, y, n, mx, my, second, part);
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
  k_qe<<<elementwise_grid((n + 1) / 2), 256, 0, st>>>(excitation, draws, seed, turn, dE, n);
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
  k_gaussian<<<elementwise_grid((n + 1) / 2), 256, 0, st>>>(seed, turn, n, out);
  return cudaGetLastError();
}

cudaError_t launch_gaussian_bunch(uint64_t seed, int64_t n, double mu_z, double sigma_z,
                                  double mu_E, double sigma_E, double* z, double* dE,
                                  cudaStream_t st) {
  k_gaussian_bunch<<<elementwise_grid(n), 256, 0, st>>>(seed, n, mu_z, sigma_z, mu_E, sigma_E, z,
                                                        dE);
  return cudaGetLastError();
}

}  // namespace hj
