// hj_wake.cu -- per-turn "bins" step: wake potential by FFT convolution and
// the E0 update, in one CTA that keeps the FFT working set in shared memory.
//
// Reference (MPI branch of apply_wakefield_inplace!, src/wakefield.jl:186-327):
//   g[i]   = delta(c_i, 0.15) * counts[i] / Σcounts                 :207-221, :238
//   pot[i] = Re(IFFT_P(FFT_P(W) .* FFT_P(g) * current))[i], i < B,
//            P = next_pow2(2B), zero padded                         :231-243, :286-319
// i.e. the causal, truncated linear convolution pot[i] = current Σ_{j<=i} W[j] g[i-j].
//
// B200 design.  W and g are real and zero beyond B <= M = P/2, so
//   * the length-P real transform is one length-M complex transform of
//     x[n] = g[2n] + i g[2n+1] followed by the usual split into even/odd
//     spectra, and
//   * x is zero for n >= M/2 = H, so the first radix-2 decimation-in-frequency
//     stage of that length-M transform is trivial: X[2m] = FFT_H(x)[m] and
//     X[2m+1] = FFT_H(x[n] w_M^n)[m].
// The inverse needs only outputs n < H, which is again two length-H
// transforms combined with one twiddle.  Each turn therefore runs four
// length-H FFTs in shared memory (H = P/4 = 8192 complex doubles = 128 KB at
// B = 16384), with the length-M spectrum parked in L2-resident global memory
// between them.  FFT(W) is constant over a run and computed once.
//
// The same CTA then forms Σ_i lerp(pot, z_i) = Σ_k H[k] pot[k] from the CIC
// deposit of the particle pass, the mean energy change of the turn
// (src/evolution.jl:401-429), the new E0 and the scalars of the next turn,
// so a turn needs no host round trip.
#include <cooperative_groups.h>

#include "hj_internal.h"

namespace hj {
namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) {
  return make_double2(a.x - b.x, a.y - b.y);
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// ---------------------------------------------------------------- FFT
// Self-sorting (Stockham) FFT of size N = 2^logN in shared memory, natural
// order in and out (Govindaraju et al., "High performance discrete Fourier
// transforms on graphics processors", SC'08): radix-8 passes, then one
// radix-4 or radix-2 pass.  Each thread loads its R points with unit stride
// across threads (conflict-free), applies the twiddles, does the R-point DFT
// in registers, and after a barrier stores them to their self-sorted
// positions in the same buffer.  tw[j] = w_N^j, j < N/2, in shared memory.

// w_N^m, 0 <= m < N, from the half table (w^{m+N/2} = -w^m).
__device__ __forceinline__ double2 twiddle(const double2* tw, int m, int halfN, bool inverse) {
  double2 w = (m < halfN) ? tw[m] : make_double2(-tw[m - halfN].x, -tw[m - halfN].y);
  if (inverse) w.y = -w.y;
  return w;
}

// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ double2 rot_q(double2 a) {
  return INV ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

template <bool INV>
__device__ __forceinline__ void dft2(double2* v) {
  const double2 t = v[0];
  v[0] = cadd(t, v[1]);
  v[1] = csub(t, v[1]);
}

template <bool INV>
__device__ __forceinline__ void dft4(double2* v) {
  const double2 d0 = cadd(v[0], v[2]), d1 = csub(v[0], v[2]);
  const double2 d2 = cadd(v[1], v[3]), d3 = rot_q<INV>(csub(v[1], v[3]));
  v[0] = cadd(d0, d2);
  v[2] = csub(d0, d2);
  v[1] = cadd(d1, d3);
  v[3] = csub(d1, d3);
}

// 8-point DFT: one radix-2 decimation-in-frequency split into two 4-point DFTs.
template <bool INV>
__device__ __forceinline__ void dft8(double2* v) {
  const double r = 0.70710678118654752440;  // 1/sqrt(2)
  double2 a[4], b[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    a[k] = cadd(v[k], v[k + 4]);
    b[k] = csub(v[k], v[k + 4]);
  }
  // b[k] *= w_8^k
  if (!INV) {
    b[1] = make_double2(r * (b[1].x + b[1].y), r * (b[1].y - b[1].x));
    b[3] = make_double2(r * (b[3].y - b[3].x), -r * (b[3].x + b[3].y));
  } else {
    b[1] = make_double2(r * (b[1].x - b[1].y), r * (b[1].x + b[1].y));
    b[3] = make_double2(-r * (b[3].x + b[3].y), r * (b[3].x - b[3].y));
  }
  b[2] = rot_q<INV>(b[2]);
  dft4<INV>(a);
  dft4<INV>(b);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[2 * k] = a[k];
    v[2 * k + 1] = b[k];
  }
}

template <int LR, bool INV>
__device__ __forceinline__ void dftR(double2* v) {
  if (LR == 3) dft8<INV>(v);
  else if (LR == 2) dft4<INV>(v);
  else dft2<INV>(v);
}

constexpr int kMaxFftH = 8192;   // largest shared-memory transform (B = 16384)

// Twiddle tables of a length-H transform in shared memory:
//   tw[j] = w_H^j, j < H/2 (the last, radix-2 or radix-4, pass reads it with
//           unit stride);
//   ct[(Ns-1)/7 + jm] = w_{8 Ns}^jm, jm < Ns, one compact row per radix-8
//           pass (Ns = 1, 8, 64, ...), so that pass also reads unit stride.
// A butterfly's q-th twiddle is w1^q, w1 = w_{Ns R}^jm (a few complex
// multiplications instead of R-1 scattered table reads).
struct FftTables {
  const double2* tw;
  const double2* ct;
};

__device__ __forceinline__ int compact_table_size(int H) { return H / 7 + 2; }

template <int LR, bool INV, int NT, int MAXH>
__device__ __forceinline__ void stockham_pass(double2* s, FftTables t, int N, int Ns) {
  constexpr int R = 1 << LR;
  constexpr int PER = (MAXH / R + NT - 1) / NT;
  const int nb = N >> LR;
  double2 v[PER][R];
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int j = threadIdx.x + u * NT;
    if (j < nb) {
      const int jm = j & (Ns - 1);
#pragma unroll
      for (int q = 0; q < R; ++q) v[u][q] = s[j + q * nb];
      double2 w1 = (LR == 3) ? t.ct[(Ns - 1) / 7 + jm] : t.tw[jm];   // last pass: Ns R = N
      if (INV) w1.y = -w1.y;
      if (LR >= 1) v[u][1] = cmul(v[u][1], w1);
      if (LR >= 2) {
        const double2 w2 = cmul(w1, w1);
        v[u][2] = cmul(v[u][2], w2);
        const double2 w3 = cmul(w2, w1);
        v[u][3] = cmul(v[u][3], w3);
        if (LR == 3) {
          const double2 w4 = cmul(w2, w2);
          v[u][4] = cmul(v[u][4], w4);
          v[u][5] = cmul(v[u][5], cmul(w4, w1));
          v[u][6] = cmul(v[u][6], cmul(w4, w2));
          v[u][7] = cmul(v[u][7], cmul(w4, w3));
        }
      }
      dftR<LR, INV>(v[u]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int j = threadIdx.x + u * NT;
    if (j < nb) {
      const int jm = j & (Ns - 1);
      const int base = ((j - jm) << LR) + jm;
#pragma unroll
      for (int q = 0; q < R; ++q) s[base + q * Ns] = v[u][q];
    }
  }
  __syncthreads();
}

// Length-N (N <= MAXH) transform by NT threads.
template <bool INV, int NT = kBinsThreads, int MAXH = kMaxFftH>
__device__ void smem_fft(double2* s, FftTables t, int N, int logN) {
  int Ns = 1, rem = logN;
  while (rem >= 3) {
    stockham_pass<3, INV, NT, MAXH>(s, t, N, Ns);
    Ns <<= 3;
    rem -= 3;
  }
  if (rem == 2) stockham_pass<2, INV, NT, MAXH>(s, t, N, Ns);
  else if (rem == 1) stockham_pass<1, INV, NT, MAXH>(s, t, N, Ns);
}

// Twiddle tables of a length-N transform into shared memory, w_N^j =
// twP[step j] with step = P/N (4 for the length-H transforms).
__device__ void load_twiddles(double2* tw, double2* ct, int N, const double2* __restrict__ twP,
                              int step = 4) {
  for (int j = threadIdx.x; j < (N >> 1); j += blockDim.x) tw[j] = __ldg(&twP[step * j]);
  for (int Ns = 1; 8 * Ns <= N; Ns <<= 3) {
    const int off = (Ns - 1) / 7, stride = N / (8 * Ns);
    for (int jm = threadIdx.x; jm < Ns; jm += blockDim.x)
      ct[off + jm] = __ldg(&twP[step * jm * stride]);
  }
  __syncthreads();
}

// X[0..M) = FFT_M(x), x[n] = v(2n) + i v(2n+1), v(j) = 0 for j >= L (L <= M):
// X[2m] = FFT_H(x)[m] and X[2m+1] = FFT_H(x[n] w_M^n)[m], since x[n] = 0 for n >= H.
template <typename Vals>
__device__ void forward_packed(const Vals& v, int L, int H, int logH,
                               const double2* __restrict__ twP, double2* s, FftTables tb,
                               double2* Xg) {
#pragma unroll 8
  for (int n = threadIdx.x; n < H; n += kBinsThreads) {
    const int j = 2 * n;
    s[n] = make_double2(j < L ? v(j) : 0.0, j + 1 < L ? v(j + 1) : 0.0);
  }
  __syncthreads();
  smem_fft<false>(s, tb, H, logH);
  for (int m = threadIdx.x; m < H; m += kBinsThreads) Xg[2 * m] = s[m];
  __syncthreads();
#pragma unroll 8
  for (int n = threadIdx.x; n < H; n += kBinsThreads) {
    const int j = 2 * n;
    const double2 a = make_double2(j < L ? v(j) : 0.0, j + 1 < L ? v(j + 1) : 0.0);
    s[n] = cmul(a, __ldg(&twP[2 * n]));  // w_M^n = w_P^{2n}
  }
  __syncthreads();
  smem_fft<false>(s, tb, H, logH);
  for (int m = threadIdx.x; m < H; m += kBinsThreads) Xg[2 * m + 1] = s[m];
  __syncthreads();
}

// Spectrum G[k] (0 <= k <= M) of the real length-P sequence from the packed
// transform X: G = E + w_P^k O, E = (X[k] + conj X[M-k])/2, O = (X[k] - conj X[M-k])/(2i).
__device__ __forceinline__ double2 real_spectrum(const double2* __restrict__ Xg, int k, int M,
                                                 const double2* __restrict__ twP) {
  const double2 xk = Xg[k == M ? 0 : k];
  const double2 xc = cconj(Xg[k == 0 ? 0 : M - k]);
  const double2 E = make_double2(0.5 * (xk.x + xc.x), 0.5 * (xk.y + xc.y));
  const double2 D = make_double2(0.5 * (xk.x - xc.x), 0.5 * (xk.y - xc.y));
  const double2 O = make_double2(D.y, -D.x);
  return cadd(E, cmul(__ldg(&twP[k]), O));
}

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
  return s;  // valid in thread 0
}

// Four block_sum's at once (one pair of barriers): each value is summed in
// block_sum's order, so the results are the same.  Valid in thread 0.
__device__ __forceinline__ void block_sum4(double (&v)[4], double (*red4)[4]) {
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) red4[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red4[w][k];
      v[k] = s;
    }
}

struct WakeVals {
  const double* W;
  __device__ double operator()(int j) const { return W[j]; }
};

struct DensityVals {
  const unsigned long long* cnt;
  const double* lam;
  double inv_n;
  __device__ double operator()(int j) const {
    return lam[j] * ((double)cnt[j] * inv_n);  // src/wakefield.jl:210, :238
  }
};

__global__ void __launch_bounds__(kBinsThreads)
    k_wake_spectrum(const double* __restrict__ W, int B, int P, int M, int H, int logH,
                    const double2* __restrict__ twP, double2* Xg, double2* Wf) {
  extern __shared__ __align__(16) double2 s_fft[];
  double2* s_tw = s_fft + H;
  double2* s_ct = s_tw + H / 2;
  load_twiddles(s_tw, s_ct, H, twP);
  forward_packed(WakeVals{W}, B, H, logH, twP, s_fft, FftTables{s_tw, s_ct}, Xg);
  for (int k = threadIdx.x; k <= M; k += blockDim.x) Wf[k] = real_spectrum(Xg, k, M, twP);
}

// Exact 10^p for 0 <= p <= 22.
__device__ __forceinline__ double pow10_exact(int p) {
  double d = 1.0;
  for (int i = 0; i < p; ++i) d *= 10.0;
  return d;
}

// Wake current of src/evolution.jl:373-386; floor(log10 N) by digit count.
__device__ double wake_current(int64_t n, double E0, const hj_params& p, double sigma_z,
                               double sigma_E0_initial, double population) {
  const double g0 = E0 / p.mass;
  const double eta0 = p.alpha_c - (1.0 / (g0 * g0));
  double pf;
  if (population > 0.0) {
    pf = population;
  } else {
    int digits = 0;
    for (int64_t m = n; m > 0; m /= 10) ++digits;
    int pw = digits - 1;
    if (pw > 10) pw = 10;
    if (pw < -10) pw = -10;
    double den = pw >= 0 ? pow10_exact(pw) : 1.0 / pow10_exact(-pw);
    pf = (1e11 / den) * (double)n;
  }
  return pf / E0 / (kTwoPi * p.radius) * sigma_z / (eta0 * (sigma_E0_initial * sigma_E0_initial));
}

// compute_global_std from sums, src/utils.jl:593-605.
__device__ __forceinline__ double global_std(double s, double s2, int64_t n) {
  if (n <= 1) return 0.0;
  const double nd = (double)n;
  const double mean = s / nd;
  const double var = (s2 / nd) - (mean * mean);
  double sv = var * nd / (double)(n - 1);
  if (!(sv > 0.0)) sv = (sv != sv) ? sv : 0.0;
  return sqrt(sv);
}

// The bins step as a cluster of C = 2 or 4 CTAs; CTA r owns the spectrum
// entries k = r (mod C).  Since x[n] = 0 for n >= H = M/2,
//   X[Cm + r] = FFT_L(y_r)[m],  y_r[n] = Σ_{t<C/2} x[n + tL] w_M^{(n + tL) r},
// L = M/C, so each CTA runs one forward and one inverse length-L FFT in its own
// shared memory.  The partner X[M-k] of a spectrum pair has residue -r: for
// C = 2 it is in the same CTA (each pair is formed in place); for C = 4 CTAs 1
// and 3 read each other's through distributed shared memory.  The inverse
// outputs z[n] = Σ_r w_M^{-nr} ẑ_r[n mod L], n < H, are combined through
// distributed shared memory, a quarter (C = 4) or half (C = 2) per CTA.
template <int NT, int MAXH = kMaxFftH, int C = 2>
__device__ __forceinline__ void bins_body(const BinsArgs& a) {
  static_assert(C == 2 || C == 4 || C == 8, "two, four or eight CTAs per cluster");
  constexpr int kLogC = C == 2 ? 1 : (C == 4 ? 2 : 3);
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  extern __shared__ __align__(16) double2 s_fft[];
  __shared__ double red[NT / 32];
  __shared__ double sh[8];
  __shared__ double s_peer_sum[C];

  // 1. partial sums of the particle pass, fixed block order (both CTAs)
  //    sh[0..3] = Σz, Σz², Σ(ΔE - ΔE_start), particles inside the bin range
  if (!a.conv_only) {
    static_assert(kNumSums == 4, "four partial sums per block");
    __shared__ double red4[NT / 32][4];
    double t[kNumSums] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < a.nblk; b += blockDim.x)
#pragma unroll
      for (int k = 0; k < kNumSums; ++k) t[k] += a.part_sum[(size_t)b * kNumSums + k];
    block_sum4(t, red4);
    if (threadIdx.x == 0)
#pragma unroll
      for (int k = 0; k < kNumSums; ++k) sh[k] = t[k];
  } else {
    double t = 0.0;
    for (int i = threadIdx.x; i < a.B; i += blockDim.x) t += (double)a.cnt[i];
    double v = block_sum(t, red);
    if (threadIdx.x == 0) sh[3] = v;
  }
  TurnState* ts = a.ts;
  if (threadIdx.x == 0) {
    if (a.conv_only) {
      sh[4] = a.conv_current;
      sh[5] = 0.0;
      sh[6] = (a.use_wake && sh[3] > 0.0) ? 1.0 : 0.0;
    } else {
      const double E0 = ts->cur.E0;
      double sigma_z = 0.0, current = 0.0;
      if (a.use_wake) {
        sigma_z = global_std(sh[0], sh[1], a.n);                 // src/evolution.jl:357
        current = wake_current(a.n, E0, a.params, sigma_z, a.sigma_E0_initial, a.population);
      }
      sh[4] = current;
      sh[5] = sigma_z;
      sh[6] = (a.use_wake && sh[3] > 0.0) ? 1.0 : 0.0;          // src/wakefield.jl:305
    }
  }
  __syncthreads();
  const double current = sh[4];
  const bool do_conv = sh[6] != 0.0;
  double sum_kick = 0.0;

  if (a.use_wake) {
    if (do_conv && a.H >= 2 * C) {
      const int H = a.H, M = a.M;
      const int L = M / C, logL = a.logH + 1 - kLogC;
      double2* s = s_fft;
      double2* s_tw = s_fft + L;
      double2* s_ct = s_tw + L / 2;
      const FftTables tb{s_tw, s_ct};
      load_twiddles(s_tw, s_ct, L, a.twP, 2 * C);              // w_L^j = w_P^{2Cj}
      const double inv_n = 1.0 / sh[3];                          // src/wakefield.jl:207
      const DensityVals g{a.cnt, a.lam, inv_n};
      // y_r[n] = Σ_t x[n + tL] w_M^{(n + tL) r}, x[n] = g[2n] + i g[2n+1]
#pragma unroll 8
      for (int n = threadIdx.x; n < L; n += NT) {
        double2 y = make_double2(0.0, 0.0);
#pragma unroll
        for (int t = 0; t < C / 2; ++t) {
          const int nn = n + t * L;
          const int j = 2 * nn;
          const double2 x = make_double2(j < a.B ? g(j) : 0.0, j + 1 < a.B ? g(j + 1) : 0.0);
          const double2 xr = rank ? cmul(x, __ldg(&a.twP[(2 * nn * rank) & (a.P - 1)])) : x;
          if (t == 0) y = xr;
          else y = cadd(y, xr);
        }
        s[n] = y;
      }
      __syncthreads();
      smem_fft<false, NT, MAXH>(s, tb, L, logL);                           // s[m] = X[Cm + rank]
      if constexpr (C >= 4) {
        // spectrum of this residue from X[k] here and X[M-k] in the CTA of
        // residue -rank; Z[k] kept in registers until every CTA has read
        constexpr int PER = (MAXH + NT - 1) / NT;                 // L <= MAXH
        cluster.sync();
        const int pr = (C - rank) % C;
        const double2* sp = cluster.map_shared_rank(s_fft, pr);
        double2 zk[PER];
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const int m = threadIdx.x + u * NT;
          if (m < L) {
            const int k = C * m + rank;
            const int kp = (M - k) & (M - 1);                     // M-k, X[M] = X[0]
            const double2 xk = s[m], xm = sp[(kp - pr) / C];
            const double2 tk = k <= M / 2 ? __ldg(&a.twP[k])
                                          : make_double2(-__ldg(&a.twP[M - k]).x,
                                                         __ldg(&a.twP[M - k]).y);
            const double2 tm = make_double2(-tk.x, tk.y);       // w_P^{M-k}
            double2 E = make_double2(0.5 * (xk.x + xm.x), 0.5 * (xk.y - xm.y));
            double2 D = make_double2(0.5 * (xk.x - xm.x), 0.5 * (xk.y + xm.y));
            const double2 Gk = cadd(E, cmul(tk, make_double2(D.y, -D.x)));
            E = make_double2(0.5 * (xm.x + xk.x), 0.5 * (xm.y - xk.y));
            D = make_double2(0.5 * (xm.x - xk.x), 0.5 * (xm.y + xk.y));
            const double2 Gm = cadd(E, cmul(tm, make_double2(D.y, -D.x)));
            double2 Yk = cmul(Gk, __ldg(&a.Wf[k]));
            double2 Ym = cmul(Gm, __ldg(&a.Wf[M - k]));
            Yk.x *= current;
            Yk.y *= current;
            Ym.x *= current;
            Ym.y *= current;
            const double2 Ez = make_double2(0.5 * (Yk.x + Ym.x), 0.5 * (Yk.y - Ym.y));
            const double2 Dz = make_double2(0.5 * (Yk.x - Ym.x), 0.5 * (Yk.y + Ym.y));
            const double2 Oz = cmul(Dz, cconj(tk));
            zk[u] = make_double2(Ez.x - Oz.y, Ez.y + Oz.x);
          }
        }
        cluster.sync();
#pragma unroll
        for (int u = 0; u < PER; ++u) {
          const int m = threadIdx.x + u * NT;
          if (m < L) s[m] = zk[u];
        }
        __syncthreads();
        smem_fft<true, NT, MAXH>(s, tb, L, logL);                          // unnormalised inverse
        cluster.sync();
        // z[n] = Σ_r conj(w_M^{nr}) ẑ_r[n mod L] / M, n in this CTA's quarter of [0, H)
        const double invM = 1.0 / (double)M;
        const double2* sr[C];
#pragma unroll
        for (int r = 0; r < C; ++r) sr[r] = cluster.map_shared_rank(s_fft, r);
        const int n0 = rank * (H / C), n1 = n0 + H / C;
#pragma unroll 2
        for (int n = n0 + threadIdx.x; n < n1; n += NT) {
          const int nl = n & (L - 1);
          double2 z = sr[0][nl];
#pragma unroll
          for (int r = 1; r < C; ++r)
            z = cadd(z, cmul(sr[r][nl], cconj(__ldg(&a.twP[(2 * n * r) & (a.P - 1)]))));
          const int j = 2 * n;
          if (j < a.B) a.pot[j] = z.x * invM;
          if (j + 1 < a.B) a.pot[j + 1] = z.y * invM;
        }
      } else {
      // spectrum pairs (k, M-k) of this parity, in place
      const int mlast = rank ? H / 2 - 1 : H / 2;
      for (int m = threadIdx.x; m <= mlast; m += NT) {
        const int k = 2 * m + rank;
        const int mp = rank ? H - 1 - m : (m == 0 ? 0 : H - m);  // X[M-k] = s[mp]
        const double2 xk = s[m], xm = s[mp];
        const double2 tk = __ldg(&a.twP[k]);
        const double2 tm = make_double2(-tk.x, tk.y);           // w_P^{M-k}
        double2 E = make_double2(0.5 * (xk.x + xm.x), 0.5 * (xk.y - xm.y));
        double2 D = make_double2(0.5 * (xk.x - xm.x), 0.5 * (xk.y + xm.y));
        const double2 Gk = cadd(E, cmul(tk, make_double2(D.y, -D.x)));
        E = make_double2(0.5 * (xm.x + xk.x), 0.5 * (xm.y - xk.y));
        D = make_double2(0.5 * (xm.x - xk.x), 0.5 * (xm.y + xk.y));
        const double2 Gm = cadd(E, cmul(tm, make_double2(D.y, -D.x)));
        double2 Yk = cmul(Gk, __ldg(&a.Wf[k]));
        double2 Ym = cmul(Gm, __ldg(&a.Wf[M - k]));
        Yk.x *= current;
        Yk.y *= current;
        Ym.x *= current;
        Ym.y *= current;
        double2 Ez = make_double2(0.5 * (Yk.x + Ym.x), 0.5 * (Yk.y - Ym.y));
        double2 Dz = make_double2(0.5 * (Yk.x - Ym.x), 0.5 * (Yk.y + Ym.y));
        double2 Oz = cmul(Dz, cconj(tk));
        const double2 Zk = make_double2(Ez.x - Oz.y, Ez.y + Oz.x);
        if (mp != m && !(rank == 0 && m == 0)) {
          Ez = make_double2(0.5 * (Ym.x + Yk.x), 0.5 * (Ym.y - Yk.y));
          Dz = make_double2(0.5 * (Ym.x - Yk.x), 0.5 * (Ym.y + Yk.y));
          Oz = cmul(Dz, cconj(tm));
          s[mp] = make_double2(Ez.x - Oz.y, Ez.y + Oz.x);
        }
        s[m] = Zk;
      }
      __syncthreads();
      smem_fft<true, NT, MAXH>(s, tb, L, logL);                            // unnormalised inverse
      cluster.sync();
      // z[n] = (zE[n] + conj(w_M^n) zO[n]) / M, pot[2n] = Re z, pot[2n+1] = Im z
      const double2* sE = cluster.map_shared_rank(s_fft, 0);
      const double2* sO = cluster.map_shared_rank(s_fft, 1);
      const double invM = 1.0 / (double)M;
      const int n0 = rank * (H / 2), n1 = n0 + H / 2;
#pragma unroll 4
      for (int n = n0 + threadIdx.x; n < n1; n += NT) {
        const double2 zo = cmul(sO[n], cconj(__ldg(&a.twP[2 * n])));
        const double2 ze = sE[n];
        const int j = 2 * n;
        if (j < a.B) a.pot[j] = (ze.x + zo.x) * invM;
        if (j + 1 < a.B) a.pot[j + 1] = (ze.y + zo.y) * invM;
      }
      }
    } else if (do_conv) {
      // Tiny grids (P < 16): direct causal convolution in CTA 0.
      if (rank == 0 && threadIdx.x == 0) {
        const double inv_n = 1.0 / sh[3];
        for (int i = 0; i < a.B; ++i) {
          double acc = 0.0;
          for (int j = 0; j <= i; ++j)
            acc += a.W[j] * (a.lam[i - j] * ((double)a.cnt[i - j] * inv_n));
          a.pot[i] = acc * current;
        }
      }
    } else {
      for (int i = rank * NT + threadIdx.x; i < a.B; i += C * NT) a.pot[i] = 0.0;
    }
    cluster.sync();   // pot complete; the peer is done reading this CTA's shared memory
    // Kick table of the next pass, B + 1 cells: cell j in 1..B-1 spans centres
    // c[j-1]..c[j] and holds (pot[j-1], pot[j] - pot[j-1]); cells 0 and B are
    // flat: pot[0] below c1, and above cB the value the reference's clamped
    // interpolation takes there, pot[hi] (1 - w) + pot[hi+1] w with u =
    // (cB - c1)/Δc rounded as it rounds it (pot[B-2] when u is exactly B-1,
    // src/wakefield.jl:80-102).  With C[j] particles
    // deposited in cell j and S[j] = Σ w·2^24 over them, the same table gives
    //   Σ_i lerp(pot, z_i) = Σ_j C[j] pot_j + 2^-24 Σ_j S[j] step_j.
    if (a.potd || a.cic) {
      const int nc = a.B + 1;
      const int part = (nc + C - 1) / C;
      const int j1 = min(nc, (rank + 1) * part);
      for (int j = rank * part + threadIdx.x; j < j1; j += blockDim.x) {
        double p0 = a.pot[j > 0 ? j - 1 : 0];
        if (j == a.B && a.B >= 2)
          p0 = __dadd_rn(__dmul_rn(a.pot[a.hi_idx], __dsub_rn(1.0, a.hi_w)),
                         __dmul_rn(a.pot[a.hi_idx + 1], a.hi_w));
        const double d = (j > 0 && j < a.B) ? a.pot[j] - p0 : 0.0;
        if (a.potd) a.potd[j] = make_double2(p0, d);
        if (a.cic) sum_kick += (double)a.cic[j] * p0 + (double)a.cic[nc + j] * 5.9604644775390625e-08 * d;
      }
    }
  }
  sum_kick = block_sum(sum_kick, red);
  if (rank > 0 && threadIdx.x == 0) *cluster.map_shared_rank(&s_peer_sum[rank], 0) = sum_kick;
  cluster.sync();

  // E0 update and next-turn scalars (src/evolution.jl:401-451, :300-304)
  if (rank == 0 && threadIdx.x == 0 && !a.conv_only) {
    for (int r = 1; r < C; ++r) sum_kick += s_peer_sum[r];
    const double E0 = ts->cur.E0;
    double mean = 0.0;
    if (a.params.update_E0) mean = (sh[2] - sum_kick) / (double)a.n;
    const double E0n = E0 + mean;
    ts->pending = 1;
    ts->pending_mean = mean;
    ts->last_sigma_z = sh[5];
    ts->last_current = current;
    ts->last_mean = mean;
    ts->last_sum_kick = sum_kick;
    ts->last_n_in = sh[3];
    ts->last_mean_z = sh[0] / (double)a.n;
    ts->turn = ts->turn + 1;
    ts->turns_left = ts->turns_left - 1;
    ts->cur = make_turn_scalars(E0n, a.params, a.sigma_E0_initial);
    // Flag what the turn actually used: a NaN current with no particle in
    // range never reaches the bunch (src/wakefield.jl:305-311).
    if (!isfinite(mean) || (a.use_wake && !isfinite(sh[5])) || (do_conv && !isfinite(current)))
      ts->status |= (1 << HJ_ERR_NONFINITE);
  }
}

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(kBinsThreads, 1) k_bins(BinsArgs a) {
  grid_dependency_wait();
  bins_body<kBinsThreads>(a);
}

// Four CTAs, length-L = M/4 transforms (at most kMaxFftH / 2), 512 threads
// each: a radix-8 pass of a length-4096 transform has 512 butterflies, and
// the step's many barriers are cheaper with fewer warps (1e5 particles at
// 4096 bins: 27.0 -> 25.7 us per turn against 1024 threads).
constexpr int kBins4MinH = 1024;
constexpr int kBins4Threads = 512;
__global__ void __cluster_dims__(4, 1, 1) __launch_bounds__(kBins4Threads, 1) k_bins4(BinsArgs a) {
  grid_dependency_wait();
  bins_body<kBins4Threads, kMaxFftH / 2, 4>(a);
}

// Eight CTAs, length-L = M/8 transforms, 512 threads each (1e6 particles at
// 16384 bins: 56.5 -> 55.1 us per turn against 1024 threads).
constexpr int kBins8MinH = 4096;
__global__ void __cluster_dims__(8, 1, 1) __launch_bounds__(kBins4Threads, 1) k_bins8(BinsArgs a) {
  grid_dependency_wait();
  bins_body<kBins4Threads, kMaxFftH / 4, 8>(a);
}

// The bins step of a batch: cluster i (CTAs Ci .. Ci + C - 1) runs bunch i;
// slots past the live count and bunches with no turns left return at once
// (the CTAs of a cluster read the same state before any writes it, so they agree).
template <int NT, int MAXH, int MINB, int C = 2>
__global__ void __cluster_dims__(C, 1, 1) __launch_bounds__(NT, MINB)
    k_batch_bins(const BinsArgs* __restrict__ bunches, const int32_t* __restrict__ n_bunches) {
  const int i = (int)(blockIdx.x / C);
  if (i >= *n_bunches) return;
  const BinsArgs& a = bunches[i];
  if (a.ts->turns_left <= 0) return;
  bins_body<NT, MAXH, C>(a);
}

// The batched bins step for H <= 2048 (up to 4096 bins): a radix-8 pass of a
// length-2048 transform has 256 butterflies, so 256 threads per CTA keep every
// pass busy, and four CTAs share an SM -- a batch of bunches runs in a quarter
// of the waves of the 1024-thread kernel.
constexpr int kBatchBinsSmallThreads = 256;
constexpr int kBatchBinsSmallMaxH = 2048;

}  // namespace

cudaError_t prepare_wake_kernels(int max_smem) {
  cudaError_t e = allow_dynamic_smem((const void*)k_bins, max_smem);
  if (e == cudaSuccess) e = allow_dynamic_smem((const void*)k_bins4, max_smem);
  if (e == cudaSuccess) e = allow_dynamic_smem((const void*)k_bins8, max_smem);
  if (e == cudaSuccess)
    e = allow_dynamic_smem((const void*)k_batch_bins<kBinsThreads, kMaxFftH, 1>, max_smem);
  if (e == cudaSuccess)
    e = allow_dynamic_smem((const void*)k_batch_bins<kBinsThreads, kMaxFftH / 2, 1, 4>,
                           max_smem);
  if (e == cudaSuccess)
    e = allow_dynamic_smem(
        (const void*)k_batch_bins<kBatchBinsSmallThreads, kBatchBinsSmallMaxH, 4>, max_smem);
  if (e == cudaSuccess) e = allow_dynamic_smem((const void*)k_wake_spectrum, max_smem);
  return e;
}

// FFT data (H complex) + twiddles (H/2) + compact radix-8 twiddle rows.
size_t bins_smem_bytes(int H) {
  const int h = H < 4 ? 4 : H;
  return (size_t)(h + h / 2 + h / 7 + 2) * sizeof(double2);
}

cudaError_t launch_wake_spectrum(const double* W, int B, int P, int M, int H, int logH,
                                 const double2* twP, double2* Xg, double2* Wf,
                                 cudaStream_t st) {
  size_t smem = bins_smem_bytes(H);
  k_wake_spectrum<<<1, kBinsThreads, smem, st>>>(W, B, P, M, H, logH, twP, Xg, Wf);
  return cudaGetLastError();
}

cudaError_t launch_bins(const BinsArgs& a, cudaStream_t st) {
  if (a.H >= kBins8MinH) {
    PdlConfig l(dim3(8), dim3(kBins4Threads), bins_smem_bytes(a.M / 8), st);
    return cudaLaunchKernelEx(&l.cfg, k_bins8, a);
  }
  if (a.H >= kBins4MinH) {
    PdlConfig l(dim3(4), dim3(kBins4Threads), bins_smem_bytes(a.M / 4), st);
    return cudaLaunchKernelEx(&l.cfg, k_bins4, a);
  }
  PdlConfig l(dim3(2), dim3(kBinsThreads), bins_smem_bytes(a.H), st);
  return cudaLaunchKernelEx(&l.cfg, k_bins, a);
}

// CTAs per bunch of a batch's bins step, fixed when the batch is created so
// that a bunch's arithmetic does not depend on which bunches share it: four
// for large grids when every slot's cluster still fits in one wave, else two.
int batch_bins_ctas(int max_H, int max_bunches, int num_sms) {
  return (max_H >= kBins4MinH && 4 * max_bunches <= num_sms) ? 4 : 2;
}

cudaError_t launch_batch_bins(const BinsArgs* d_bunches, const int32_t* d_n_bunches,
                              int max_bunches, int max_H, int ctas, cudaStream_t st) {
  size_t smem = bins_smem_bytes(max_H);
  const int grid = 2 * (max_bunches > 0 ? max_bunches : 1);
  if (ctas == 4) {
    k_batch_bins<kBinsThreads, kMaxFftH / 2, 1, 4>
        <<<2 * grid, kBinsThreads, bins_smem_bytes(max_H / 2), st>>>(d_bunches, d_n_bunches);
  } else if (max_H <= kBatchBinsSmallMaxH)
    k_batch_bins<kBatchBinsSmallThreads, kBatchBinsSmallMaxH, 4>
        <<<grid, kBatchBinsSmallThreads, smem, st>>>(d_bunches, d_n_bunches);
  else
    k_batch_bins<kBinsThreads, kMaxFftH, 1><<<grid, kBinsThreads, smem, st>>>(d_bunches,
                                                                             d_n_bunches);
  return cudaGetLastError();
}

}  // namespace hj
