// hj_noalloc.cu -- wake potential from device counts with no allocation.
//
// Who needs it: callers that own all of their device memory through another
// allocator (a framework's memory pool, or a fixed arena sized at start-up)
// and must not call cudaMalloc behind its back, and latency-critical loops
// that cannot afford cudaMalloc/cudaFree, which can synchronise the device
// and stall work on other streams.
//
// hj_wake_potential_noalloc computes the same potential as
// hj_wake_potential (the FFT convolution of the bins kernel) on
// caller-provided DEVICE buffers, and keeps every intermediate array in the
// file-scope array g_noalloc_scratch below.  It never calls cudaMalloc,
// cudaFree or any allocating library routine.
//
// Limits and sharing rules:
//   * at most kNoAllocMaxBins = 16384 bins (FFT length 32768); larger grids
//     are rejected with HJ_ERR_TOO_LARGE;
//   * the scratch array (about 1.4 MB) is a static device variable: every
//     GPU that loads this library holds it until the process exits;
//   * all calls on a device share the one array.  Calls whose work overlaps
//     on the GPU (different streams, or different host threads) race on it;
//     serialise them (same stream, or events);
//   * each call overwrites every scratch element it later reads (tables,
//     spectra, FFT work space), so nothing has to start at zero and the
//     previous call's leftovers are never read;
//   * the array's device address is looked up once per device and kept for
//     the life of the process, so the library does not survive a
//     cudaDeviceReset of that device (nor does any of its other state);
//   * the caller's current device is restored before the call returns.
#include <mutex>

#include "hj_state.h"

namespace hj {
namespace {

constexpr int kNoAllocMaxBins = 16384;
constexpr int kNoAllocP = 2 * kNoAllocMaxBins;           // next_pow2(2B) at the limit
constexpr int kNoAllocM = kNoAllocP / 2;
constexpr int kNoAllocH = kNoAllocM / 2;
// Layout in doubles: W[B] | lam[B] | twP[2P] | Wf[2(M+1)] | Xg[2M] | zE[2H],
// each slot sized for the largest grid and rounded to 32 doubles (256 B).
constexpr size_t slot(size_t d) { return (d + 31) / 32 * 32; }
constexpr size_t kOffW = 0;
constexpr size_t kOffLam = kOffW + slot(kNoAllocMaxBins);
constexpr size_t kOffTw = kOffLam + slot(kNoAllocMaxBins);
constexpr size_t kOffWf = kOffTw + slot(2 * (size_t)kNoAllocP);
constexpr size_t kOffXg = kOffWf + slot(2 * ((size_t)kNoAllocM + 1));
constexpr size_t kOffZe = kOffXg + slot(2 * (size_t)kNoAllocM);
constexpr size_t kScratchDoubles = kOffZe + slot(2 * (size_t)kNoAllocH);

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (cudaGetSymbolAddress; the host-side name is only a stand-in).
cudaError_t scratch_address(int device, double** out) {
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[device]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

// Wake table, smoothing weights (from the centres already copied into W)
// and FFT twiddles exp(-2πik/P), all written into the scratch.
__global__ void k_noalloc_tables(double* W, double* lam, double2* twP, int B, int P,
                                 double F, double s, double ctau, double sin_coef,
                                 double delta_std) {
  const int stride = gridDim.x * blockDim.x;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += stride) {
    const double c = W[i];
    // src/utils.jl:58-66
    lam[i] = 1.0 / (sqrt(kTwoPi) * delta_std) * exp(c * c * (-0.5 / (delta_std * delta_std)));
    // src/wakefield.jl:115-118 (+ optional resonator sine term)
    double w = 0.0;
    if (!(c > 0.0)) {
      double osc = cos(s * c);
      if (sin_coef != 0.0) osc = osc + sin_coef * sin(s * c);
      w = F * exp(c * (1.0 / ctau)) * osc;
    }
    W[i] = w;
  }
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < P; k += stride) {
    double sn, cs;
    sincospi(-2.0 * (double)k / (double)P, &sn, &cs);
    twP[k] = make_double2(cs, sn);
  }
}

int ilog2i(int v) {
  int l = 0;
  while ((1 << l) < v) ++l;
  return l;
}

// Puts the caller's current device back when the entry point returns.
struct DeviceRestore {
  int device = -1;
  DeviceRestore() {
    if (cudaGetDevice(&device) != cudaSuccess) device = -1;
  }
  ~DeviceRestore() {
    if (device >= 0) cudaSetDevice(device);
  }
};

}  // namespace
}  // namespace hj

using namespace hj;

extern "C" hj_status hj_wake_potential_noalloc(hj_ctx* ctx, const int64_t* d_counts,
                                               const hj_grid* grid, const hj_wake* wake,
                                               double current, double* d_pot, void* stream) {
  if (!ctx) return HJ_ERR_ARG;
  DeviceRestore restore;
  HJ_TRY(ctx_ok(ctx));                 // the context's device; clears the last error
  HJ_TRY(check_grid(ctx, grid));
  if (!d_counts || !d_pot || !wake)
    return ctx_set_error(ctx, HJ_ERR_ARG, "NULL counts, potential or wake");
  if (grid->nbins > kNoAllocMaxBins)
    return ctx_set_error(ctx, HJ_ERR_TOO_LARGE,
                         "hj_wake_potential_noalloc holds at most 16384 bins in its static "
                         "scratch; use hj_wake_potential for larger grids");
  if (!(wake->ctau > 0)) return ctx_set_error(ctx, HJ_ERR_WAKE_PARAM, "Wake parameter cτ must be positive.");
  const int device = ctx_device(ctx);
  double* base = nullptr;
  cudaError_t se = scratch_address(device, &base);
  if (se != cudaSuccess)
    return ctx_set_error(ctx, HJ_ERR_CUDA, cudaGetErrorString(se));

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int B = (int)grid->nbins;
  int P = 1;
  while (P < 2 * B) P <<= 1;
  const int M = P / 2, H = M / 2;
  const int logH = H >= 1 ? ilog2i(H) : 0;
  double* W = base + kOffW;
  double* lam = base + kOffLam;
  double2* twP = reinterpret_cast<double2*>(base + kOffTw);
  double2* Wf = reinterpret_cast<double2*>(base + kOffWf);
  double2* Xg = reinterpret_cast<double2*>(base + kOffXg);
  double2* zE = reinterpret_cast<double2*>(base + kOffZe);

  // The centres travel into the W slot; the table kernel turns them into W.
  if (cudaMemcpyAsync(W, grid->centers, sizeof(double) * B, cudaMemcpyHostToDevice, st) !=
      cudaSuccess)
    return ctx_set_error(ctx, HJ_ERR_CUDA, "copy of the bin centres failed");
  const int threads = 256;
  const int blocks = (P + threads - 1) / threads;
  k_noalloc_tables<<<blocks, threads, 0, st>>>(W, lam, twP, B, P, wake->wake_factor,
                                               wake->wake_sqrt, wake->ctau, wake->sin_coef,
                                               wake->delta_std);
  if (cudaGetLastError() != cudaSuccess)
    return ctx_set_error(ctx, HJ_ERR_CUDA, "table kernel launch failed");
  if (H >= 4 && launch_wake_spectrum(W, B, P, M, H, logH, twP, Xg, Wf, st) != cudaSuccess)
    return ctx_set_error(ctx, HJ_ERR_CUDA, "spectrum kernel launch failed");
  BinsArgs g{};
  g.use_wake = 1;
  g.B = B;
  g.P = P;
  g.M = M;
  g.H = H;
  g.logH = logH;
  g.cnt = reinterpret_cast<const unsigned long long*>(d_counts);
  g.cic = nullptr;
  g.lam = lam;
  g.Wf = Wf;
  g.twP = twP;
  g.Xg = Xg;
  g.zE = zE;
  g.pot = d_pot;
  g.W = W;
  g.conv_only = 1;
  g.conv_current = current;
  if (launch_bins(g, st) != cudaSuccess)
    return ctx_set_error(ctx, HJ_ERR_CUDA, "convolution kernel launch failed");
  return HJ_OK;
}
