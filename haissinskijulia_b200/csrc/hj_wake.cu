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
__device__ __forceinline__ int bitrev(int n, int logH) {
  return (int)(__brev((unsigned)n) >> (32 - logH));
}

// In-place decimation-in-time FFT of size H on shared memory that holds its
// input in bit-reversed order.  tw[j] = exp(-2πi j/H), j < H/2, also in shared
// memory.  Pairs of radix-2 stages are fused into radix-4 passes (each thread
// keeps the four points of two consecutive stages in registers), so a
// length-8192 transform takes 7 passes over shared memory instead of 13.
// inverse uses conjugate twiddles and no normalisation.
__device__ void smem_fft(double2* s, const double2* tw, int H, int logH, bool inverse) {
  int h = 1;
  int stage = 0;
  for (; stage + 2 <= logH; stage += 2, h <<= 2) {
    const int sa = H / (2 * h), sb = H / (4 * h);
    for (int b = threadIdx.x; b < (H >> 2); b += blockDim.x) {
      const int j = b & (h - 1);
      const int i0 = ((b - j) << 2) + j;
      double2 x0 = s[i0], x1 = s[i0 + h], x2 = s[i0 + 2 * h], x3 = s[i0 + 3 * h];
      double2 wa = tw[j * sa], wb = tw[j * sb];
      if (inverse) {
        wa.y = -wa.y;
        wb.y = -wb.y;
      }
      // span h: (x0, x1) and (x2, x3) with w_{2h}^j
      double2 t = cmul(x1, wa);
      x1 = csub(x0, t);
      x0 = cadd(x0, t);
      t = cmul(x3, wa);
      x3 = csub(x2, t);
      x2 = cadd(x2, t);
      // span 2h: (x0, x2) with w_{4h}^j, (x1, x3) with w_{4h}^{j+h} = w_{4h}^j (-i or +i)
      t = cmul(x2, wb);
      s[i0] = cadd(x0, t);
      s[i0 + 2 * h] = csub(x0, t);
      t = cmul(x3, wb);
      t = inverse ? make_double2(-t.y, t.x) : make_double2(t.y, -t.x);
      s[i0 + h] = cadd(x1, t);
      s[i0 + 3 * h] = csub(x1, t);
    }
    __syncthreads();
  }
  if (stage < logH) {  // odd number of stages: final radix-2 pass, span H/2
    for (int b = threadIdx.x; b < (H >> 1); b += blockDim.x) {
      const int j = b & (h - 1);
      const int i0 = ((b - j) << 1) + j;
      double2 w = tw[j * (H / (2 * h))];
      if (inverse) w.y = -w.y;
      const double2 u = s[i0];
      const double2 t = cmul(s[i0 + h], w);
      s[i0] = cadd(u, t);
      s[i0 + h] = csub(u, t);
    }
    __syncthreads();
  }
}

// Twiddles of the length-H transform into shared memory: w_H^j = twP[4j].
__device__ void load_twiddles(double2* tw, int H, const double2* __restrict__ twP) {
  for (int j = threadIdx.x; j < (H >> 1); j += blockDim.x) tw[j] = __ldg(&twP[4 * j]);
  __syncthreads();
}

// X[0..M) = FFT_M(x), x[n] = v(2n) + i v(2n+1), v(j) = 0 for j >= L (L <= M).
template <typename Vals>
__device__ void forward_packed(const Vals& v, int L, int P, int H, int logH,
                               const double2* __restrict__ twP, double2* s, const double2* tw,
                               double2* Xg) {
  for (int n = threadIdx.x; n < H; n += blockDim.x) {
    const int j = 2 * n;
    s[bitrev(n, logH)] = make_double2(j < L ? v(j) : 0.0, j + 1 < L ? v(j + 1) : 0.0);
  }
  __syncthreads();
  smem_fft(s, tw, H, logH, false);
  for (int m = threadIdx.x; m < H; m += blockDim.x) Xg[2 * m] = s[m];
  __syncthreads();
  for (int n = threadIdx.x; n < H; n += blockDim.x) {
    const int j = 2 * n;
    double2 a = make_double2(j < L ? v(j) : 0.0, j + 1 < L ? v(j + 1) : 0.0);
    s[bitrev(n, logH)] = cmul(a, __ldg(&twP[2 * n]));  // w_M^n = w_P^{2n}
  }
  __syncthreads();
  smem_fft(s, tw, H, logH, false);
  for (int m = threadIdx.x; m < H; m += blockDim.x) Xg[2 * m + 1] = s[m];
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

// Packed inverse input Z[k] (0 <= k < M) for the real inverse transform of
// the Hermitian spectrum Y: E' = (Y[k] + conj Y[M-k])/2,
// O' = (Y[k] - conj Y[M-k]) conj(w_P^k)/2, Z = E' + i O'.
__device__ __forceinline__ double2 packed_inverse_input(const double2* __restrict__ Xg,
                                                        const double2* __restrict__ Wf, int k,
                                                        int M, double current,
                                                        const double2* __restrict__ twP) {
  double2 yk = cmul(real_spectrum(Xg, k, M, twP), __ldg(&Wf[k]));
  yk.x *= current;
  yk.y *= current;
  double2 ym = cmul(real_spectrum(Xg, M - k, M, twP), __ldg(&Wf[M - k]));
  ym.x *= current;
  ym.y *= current;
  const double2 yc = cconj(ym);
  const double2 E = make_double2(0.5 * (yk.x + yc.x), 0.5 * (yk.y + yc.y));
  const double2 D = make_double2(0.5 * (yk.x - yc.x), 0.5 * (yk.y - yc.y));
  const double2 O = cmul(D, cconj(__ldg(&twP[k])));
  return make_double2(E.x - O.y, E.y + O.x);
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
  load_twiddles(s_tw, H, twP);
  forward_packed(WakeVals{W}, B, P, H, logH, twP, s_fft, s_tw, Xg);
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

__global__ void __launch_bounds__(kBinsThreads) k_bins(BinsArgs a) {
  extern __shared__ __align__(16) double2 s_fft[];
  __shared__ double red[kBinsThreads / 32];
  __shared__ double sh[8];

  // 1. partial sums of the particle pass, fixed block order
  //    sh[0..3] = Σz, Σz², Σ(ΔE - ΔE_start), particles inside the bin range
  if (!a.conv_only) {
    double t[kNumSums] = {0.0, 0.0, 0.0, 0.0};
    for (int b = threadIdx.x; b < a.nblk; b += blockDim.x)
#pragma unroll
      for (int k = 0; k < kNumSums; ++k) t[k] += a.part_sum[(size_t)b * kNumSums + k];
    for (int k = 0; k < kNumSums; ++k) {
      double v = block_sum(t[k], red);
      if (threadIdx.x == 0) sh[k] = v;
    }
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
    if (!do_conv) {
      for (int i = threadIdx.x; i < a.B; i += blockDim.x) a.pot[i] = 0.0;
    } else {
      const double inv_n = 1.0 / sh[3];                          // src/wakefield.jl:207
      if (a.H >= 4) {
        double2* s_tw = s_fft + a.H;
        load_twiddles(s_tw, a.H, a.twP);
        forward_packed(DensityVals{a.cnt, a.lam, inv_n}, a.B, a.P, a.H, a.logH, a.twP, s_fft,
                       s_tw, a.Xg);
        // inverse, even half -> zE
        for (int m = threadIdx.x; m < a.H; m += blockDim.x)
          s_fft[bitrev(m, a.logH)] = packed_inverse_input(a.Xg, a.Wf, 2 * m, a.M, current, a.twP);
        __syncthreads();
        smem_fft(s_fft, s_tw, a.H, a.logH, true);
        for (int m = threadIdx.x; m < a.H; m += blockDim.x) a.zE[m] = s_fft[m];
        __syncthreads();
        // inverse, odd half, combine, potential and Σ H[k] pot[k]
        for (int m = threadIdx.x; m < a.H; m += blockDim.x)
          s_fft[bitrev(m, a.logH)] =
              packed_inverse_input(a.Xg, a.Wf, 2 * m + 1, a.M, current, a.twP);
        __syncthreads();
        smem_fft(s_fft, s_tw, a.H, a.logH, true);
        const double invM = 1.0 / (double)a.M;
        for (int m = threadIdx.x; m < a.H; m += blockDim.x) {
          const double2 zo = cmul(s_fft[m], cconj(__ldg(&a.twP[2 * m])));
          const double2 ze = a.zE[m];
          const double re = (ze.x + zo.x) * invM, im = (ze.y + zo.y) * invM;
          const int j = 2 * m;
          if (j < a.B) a.pot[j] = re;
          if (j + 1 < a.B) a.pot[j + 1] = im;
        }
      } else {
        // Tiny grids (P < 16): direct causal convolution.
        if (threadIdx.x == 0) {
          for (int i = 0; i < a.B; ++i) {
            double acc = 0.0;
            for (int j = 0; j <= i; ++j)
              acc += a.W[j] * (a.lam[i - j] * ((double)a.cnt[i - j] * inv_n));
            a.pot[i] = acc * current;
          }
        }
      }
      // Σ_i lerp(pot, z_i) from the CIC deposit: with C[k] particles in cell k
      // and S[k] = Σ w·2^24 over them,
      //   Σ_i lerp = Σ_k C[k] pot[k] + 2^-24 Σ_k S[k] (pot[k+1] - pot[k]).
      __syncthreads();
      if (a.cic) {
        const unsigned long long* C = a.cic;
        const unsigned long long* S = a.cic + a.B;
        for (int k = threadIdx.x; k < a.B; k += blockDim.x) {
          double t = (double)C[k] * a.pot[k];
          if (k + 1 < a.B) t += (double)S[k] * 5.9604644775390625e-08 * (a.pot[k + 1] - a.pot[k]);
          sum_kick += t;
        }
      }
    }
  }
  sum_kick = block_sum(sum_kick, red);

  // 4. E0 update and next-turn scalars (src/evolution.jl:401-451, :300-304)
  if (threadIdx.x == 0 && !a.conv_only) {
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
    ts->turn = ts->turn + 1;
    ts->cur = make_turn_scalars(E0n, a.params, a.sigma_E0_initial);
    // Flag what the turn actually used: a NaN current with no particle in
    // range never reaches the bunch (src/wakefield.jl:305-311).
    if (!isfinite(mean) || (a.use_wake && !isfinite(sh[5])) || (do_conv && !isfinite(current)))
      ts->status |= (1 << HJ_ERR_NONFINITE);
  }
}

}  // namespace

cudaError_t prepare_wake_kernels(int max_smem) {
  cudaError_t e = allow_dynamic_smem((const void*)k_bins, max_smem);
  if (e == cudaSuccess) e = allow_dynamic_smem((const void*)k_wake_spectrum, max_smem);
  return e;
}

// FFT data (H complex) + twiddles (H/2 complex).
size_t bins_smem_bytes(int H) {
  const int h = H < 4 ? 4 : H;
  return (size_t)(h + h / 2) * sizeof(double2);
}

cudaError_t launch_wake_spectrum(const double* W, int B, int P, int M, int H, int logH,
                                 const double2* twP, double2* Xg, double2* Wf,
                                 cudaStream_t st) {
  size_t smem = bins_smem_bytes(H);
  k_wake_spectrum<<<1, kBinsThreads, smem, st>>>(W, B, P, M, H, logH, twP, Xg, Wf);
  return cudaGetLastError();
}

cudaError_t launch_bins(const BinsArgs& a, cudaStream_t st) {
  size_t smem = bins_smem_bytes(a.H);
  k_bins<<<1, kBinsThreads, smem, st>>>(a);
  return cudaGetLastError();
}

}  // namespace hj
