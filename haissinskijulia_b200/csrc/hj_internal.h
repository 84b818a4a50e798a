// hj_internal.h -- launch interface between the C-ABI layer (hj_api.cu) and
// the kernels (hj_track.cu, hj_wake.cu).  Not part of the public ABI.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "hj_device.cuh"
#include "hj_launch.h"

namespace hj {

// The per-turn kernels of a bunch are launched with programmatic stream
// serialisation: each may be scheduled while the previous kernel on the
// stream drains, and starts with grid_dependency_wait(), which returns once
// that kernel has completed and its memory is visible.
__device__ __forceinline__ void grid_dependency_wait() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

struct PdlConfig {
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  PdlConfig(dim3 grid, dim3 block, size_t smem, cudaStream_t st) {
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
};

constexpr int kNumSums = 4;         // per-block partial sums of the particle pass
constexpr int kTrackThreads = 512;  // threads per block of the particle kernels
constexpr int kBinsThreads = 1024;  // threads of the single-CTA bins kernel
constexpr int64_t kMaxBins = 16384; // largest grid the shared-memory FFT holds (P = 32768)
// kMaxBlockParticles, the thread layouts and the pass grid rule: hj_launch.h
constexpr int kRfTableSize = 128;    // entries of the fused pass's RF kick table
constexpr int kLogHeader = 8;       // doubles before the bin counts in a turn-log record

// Quantum-excitation source of the particle pass.
// QE_PHILOX_FAST: the same Philox words turned into normals in single
// precision (the kPassFastNormals layouts).
enum QeMode { QE_OFF = 0, QE_PHILOX = 1, QE_DRAWS = 2, QE_PHILOX_FAST = 3 };

// Arguments of the fused per-turn particle pass (one launch per turn).
struct PassArgs {
  double* z;
  double* dE;
  int64_t n;
  TurnState* ts;
  const double2* potd;     // [B+1] kick table of the previous turn (cell j: pot[j-1], step)
  int32_t win;             // entries of the kick table's left values held in shared memory
  // bin grid
  int32_t B;
  int32_t use_wake;
  double e0, eN, inv_estep;       // histogram (edges)
  double c1, cB, inv_cstep;       // interpolation (centers)
  // physics constants of the run
  double V, phi_s, inv_mass, alpha_c, two_pi_h;
  // RF kick: x = z k = m h + t, h = 2π / kRfTableSize (h_hi + h_lo), and
  // rf_table[m mod kRfTableSize] = (V sin(ϕs - m h), V cos(ϕs - m h)); Vs = V sin ϕs
  const double2* rf_table;
  double rf_inv_h, rf_h_hi, rf_h_lo, Vs;
  PhiloxKeys philox;       // Philox-4x32 round keys of the bunch's seed
  int32_t update_eta, update_E0, sr, qe_mode;
  int32_t cfg;             // thread layout (kNumPassCfgs)
  uint64_t seed;
  const double* draws;     // QE_DRAWS: turns x n, row = turn - draws_first_turn
  int64_t draws_first_turn;
  int64_t draws_turns;
  // per-block outputs
  uint32_t* part_cnt;              // [grid][B]
  unsigned long long* part_cic;    // [grid][B+1] packed cell deposit (count << 44 | Σw·2^24)
  double* part_sum;                // [grid][kNumSums]
  unsigned long long* hist_out;    // [3B+2] merged histograms, zeroed by the pass
  unsigned long long* hist_spill;  // [3B+2] deposits outside the hot window and beyond the
                                   // 16-bit counters (the merged layout), cleared by the merge
  int32_t n_parts;                 // partial slots written per turn (batches)
  int64_t pair_offset;             // Philox pair index of particle 0 (shards of a bunch)
  int64_t* defer_q;                // [partial slots][warps][kDeferStage]: indices of the
                                   // particles whose Float64 normal takes the slow path
  int32_t zig;                     // 1: shared memory holds the ziggurat's rows (the pass
                                   // draws the Float64 normals), 0: the RF table alone
  int32_t hwin;                    // bins and cells of the pass's hot histogram window
};

// One entry of a batch's chunk table: particles [first, first + count) of
// bunch `bunch`, deposited into that bunch's partial slot `part`.  first is a
// multiple of 4, so the 32-byte particle loads stay aligned.
struct BatchChunk {
  int64_t first;
  int64_t count;
  int32_t bunch;
  int32_t part;
};

// Arguments of the per-turn bins step (single CTA).
struct BinsArgs {
  TurnState* ts;
  const double* part_sum;
  int32_t nblk;
  int64_t n;
  hj_params params;
  double sigma_E0_initial;
  double population;
  int32_t use_wake;
  int32_t B, P, M, H, logH;
  const unsigned long long* cnt;   // [B] bin counts
  const unsigned long long* cic;   // [2(B+1)] cell counts | cell Σw·2^24 (NULL: not needed)
  const double* lam;               // [B]
  const double2* Wf;               // [M+1]
  const double2* twP;              // [P]
  double2* Xg;                     // [M]
  double2* zE;                     // [H]
  double* pot;                     // [B]
  double2* potd;                   // [B+1] kick table for the next pass; NULL: not needed
  // the reference's interpolation at z >= cB: pot[hi_idx] (1 - hi_w) + pot[hi_idx+1] hi_w
  int32_t hi_idx;
  double hi_w;
  const double* W;                 // [B] wake table (direct path for tiny grids)
  // standalone convolution (hj_wake_potential): no turn-state update
  int32_t conv_only;
  double conv_current;
};

// Moments of (z, dE) per block: [Σz, Σz², ΣdE, ΣdE²], optionally after
// applying a pending kick/re-centring (flush) and writing the result.
struct FlushArgs {
  double* z;          // state
  double* dE;
  int64_t n;
  const TurnState* ts;
  const double2* potd;
  int32_t B;
  int32_t use_wake, update_E0;
  double c1, cB, inv_cstep;
  double e0, inv_estep;   // kick-table cell coordinate
  int32_t apply;      // 1: apply pending ops
  double* z_out;      // destination (may alias z/dE); NULL -> not written
  double* dE_out;
  double* part;       // [grid][4]
};

// ---- launchers (hj_track.cu) ----
cudaError_t allow_dynamic_smem(const void* fn, int max_smem_optin);
cudaError_t prepare_track_kernels(int max_smem);   // once per device: dynamic smem limits
int track_blocks_per_sm(int B, int qe_mode, int use_wake, int cfg);
// zig: the pass draws the Float64 normals (QE_PHILOX without the fast bit),
// so its shared memory holds the ziggurat's rows.
size_t track_smem_bytes(int B, int use_wake, int cfg, bool zig);
// Shared-memory windows of the fused pass for B bins (with the wake): `hot`
// bins and cells whose per-block histograms are in shared memory (at most
// B + 1), and `kick` kick-table entries (0 up to 4096 bins, else min(hot, B)).
struct PassWindows {
  int32_t hot, kick;
};
PassWindows track_windows(int B, int cfg, bool zig);
cudaError_t launch_track_pass(const PassArgs& a, int grid, cudaStream_t st);
// Batched pass over a chunk table (*d_n_chunks entries live, grid max_chunks)
// and the per-bunch merge of its partials.
cudaError_t launch_batch_pass(const PassArgs* d_bunches, const BatchChunk* d_chunks,
                              const int32_t* d_n_chunks, int max_chunks, int max_B, int wake,
                              int qe, int cfg, int32_t* d_queue, int resident_blocks,
                              cudaStream_t st);
// Blocks of the batched pass that fit on one SM for the batch's largest grid.
int batch_blocks_per_sm(int max_B, int qe_mode, int use_wake, int cfg);
cudaError_t launch_sum_parts(const double* part, int nblk, double* out, cudaStream_t st);
cudaError_t launch_batch_reduce(const PassArgs* d_bunches, const BatchChunk* d_items,
                                const int32_t* d_n_items, int max_items, int max_B,
                                cudaStream_t st);
// out: counts[B] (| cell counts[B+1] | cell Σw·2^24 [B+1] when part_cic != NULL);
// zero_first clears out before the merge (the fused pass clears it itself).
cudaError_t launch_hist_reduce(const uint32_t* part_cnt, const unsigned long long* part_cic,
                               int nblk, int B, unsigned long long* out, bool zero_first,
                               cudaStream_t st, unsigned long long* spill = nullptr);
cudaError_t launch_flush(const FlushArgs& a, int grid, cudaStream_t st);
// generate_particles on the device (covariance sample, correlated bunch, two-pass std)
cudaError_t launch_gen_sample_cov(uint64_t seed, int64_t S, double mu_z, double sz, double mu_E,
                                  double sE, double* out, cudaStream_t st);
cudaError_t launch_gen_correlated(uint64_t seed, int64_t n, double mu_z, double mu_E, double l00,
                                  double l10, double l11, double* z, double* dE, cudaStream_t st);
cudaError_t launch_std_parts(const double* x, int64_t n, double mean, int second, double* part,
                             int grid, cudaStream_t st);
cudaError_t launch_cor_parts(const double* x, const double* y, int64_t n, double mx, double my,
                             int second, double* part, int grid, cudaStream_t st);
cudaError_t launch_log_record(const double* part, int nblk, int64_t n, const TurnState* ts,
                              const unsigned long long* counts, int B, double* rec,
                              cudaStream_t st);
cudaError_t launch_histogram_only(const double* z, int64_t n, int B, double e0, double eN,
                                  double inv_estep, uint32_t* part_cnt, int grid,
                                  cudaStream_t st);
cudaError_t launch_interp_kick(const double* z, double* dE, int64_t n, const double* pot,
                               int B, double c1, double cB, double inv_cstep,
                               cudaStream_t st);
cudaError_t launch_rf_kick(double V, double sin_phis, double k, double phi_s,
                           const double* z, double* dE, int64_t n, cudaStream_t st);
cudaError_t launch_qe(double excitation, const double* draws, uint64_t seed, int64_t turn,
                      double* dE, int64_t n, cudaStream_t st);
cudaError_t launch_sr(double damping, double* dE, int64_t n, cudaStream_t st);
cudaError_t launch_phase_advance(int update_eta, TurnScalars s, double inv_mass,
                                 double alpha_c, double two_pi_h, double phi_s,
                                 const double* dE, double* z, int64_t n, cudaStream_t st);
cudaError_t launch_gaussian(uint64_t seed, int64_t turn, int64_t n, double* out,
                            cudaStream_t st);
cudaError_t launch_gaussian_bunch(uint64_t seed, int64_t n, double mu_z, double sigma_z,
                                  double mu_E, double sigma_E, double* z, double* dE,
                                  cudaStream_t st);

// ---- launchers (hj_wake.cu) ----
cudaError_t prepare_wake_kernels(int max_smem);    // once per device: dynamic smem limits
cudaError_t launch_wake_spectrum(const double* W, int B, int P, int M, int H, int logH,
                                 const double2* twP, double2* Xg, double2* Wf,
                                 cudaStream_t st);
cudaError_t launch_bins(const BinsArgs& a, cudaStream_t st);
int batch_bins_ctas(int max_H, int max_bunches, int num_sms);
cudaError_t launch_batch_bins(const BinsArgs* d_bunches, const int32_t* d_n_bunches,
                              int max_bunches, int max_H, int ctas, cudaStream_t st);
size_t bins_smem_bytes(int H);

// ---- context access for entry points outside hj_api.cu ----
int ctx_device(const hj_ctx* ctx);
hj_status ctx_set_error(hj_ctx* ctx, hj_status code, const char* msg);

}  // namespace hj
