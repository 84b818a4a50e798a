// hj_launch.h -- thread layouts of the fused particle pass and its grid rule
// (host only, no CUDA: the rules are checked on the CPU as well).
#pragma once

#include <cstdint>

namespace hj {

// Particles one block of the fused pass may deposit per turn (the packed CIC
// counter keeps a 20-bit count per cell).
constexpr int64_t kMaxBlockParticles = (1 << 20) - 8;

// Thread layouts of the fused pass (particles/thread x threads/block; the next
// group prefetched into registers except in 3): 0 = 4 x 512, 1 = 2 x 1024,
// 2 = 2 x 768, 3 = 2 x 512 without prefetch, 4 = 2 x 512 at 64 registers (two
// blocks per SM where shared memory allows), 5 = 4 x 256 at 128 registers
// (two blocks per SM: one block's set-up and write-out overlap the other's
// particles).
constexpr int kNumPassCfgs = 6;       // thread layouts of the fused pass
constexpr int kPassLayoutMask = 7;    // layout bits of a pass configuration
constexpr int kPassN32 = 8;           // + one 32-bit NGP counter per bin (else 16-bit pairs)
constexpr int kPassFastNormals = 16;  // + single-precision quantum-excitation normals
// Launch-only bit (never in a caller's configuration): the pass's hot window
// holds fewer than all B + 1 cells, so its deposits are range-checked.
constexpr int kPassWindowed = 32;

inline int pass_cfg_threads(int cfg) {
  const int l = cfg & kPassLayoutMask;
  return l == 1 ? 1024 : (l == 2 ? 768 : (l == 5 ? 256 : 512));
}
inline int pass_cfg_ppt(int cfg) {
  const int l = cfg & kPassLayoutMask;
  return (l == 0 || l == 5) ? 4 : 2;
}
// Layouts that keep two blocks on an SM (each takes at most half of it).
inline bool pass_cfg_two_blocks(int cfg) {
  const int l = cfg & kPassLayoutMask;
  return l == 4 || l == 5;
}
// Entries of a warp's staging queue of particles whose Float64 normal takes
// the ziggurat's slow path (the fused pass finishes them 32 at a time).
constexpr int kDeferStage = 64;
inline bool pass_cfg_valid(int cfg) {
  return cfg >= 0 && (cfg & ~(kPassLayoutMask | kPassN32 | kPassFastNormals)) == 0 &&
         (cfg & kPassLayoutMask) < kNumPassCfgs;
}

// A caller's layout request: -1 = automatic; kPassAutoFast = the automatic
// layout with single-precision normals; otherwise a valid configuration.
constexpr int kPassAutoFast = kPassFastNormals | kPassLayoutMask;
inline bool pass_request_valid(int r) { return r == -1 || r == kPassAutoFast || pass_cfg_valid(r); }
// The configuration a request gives for bins B, `automatic` being the
// library's choice for them.
inline int resolve_pass_request(int r, int automatic) {
  if (r == -1) return automatic;
  if (r == kPassAutoFast) return automatic | kPassFastNormals;
  return r;
}

// Blocks of the particle pass: enough to fill the GPU, but each block should
// move at least B/2 particles, since it writes a B-bin partial histogram
// that the merge reads back (B/2 measured best for 1e5-1e7 particles at 4096
// and 16384 bins).
inline int track_grid_size(int64_t n, int B, int num_sms, int blocks_per_sm, int cfg) {
  int64_t per_block = (int64_t)pass_cfg_ppt(cfg) * pass_cfg_threads(cfg);
  if (per_block < (int64_t)B / 2) per_block = (int64_t)B / 2;
  int64_t g = (n + per_block - 1) / per_block;
  int64_t cap = (int64_t)num_sms * blocks_per_sm;
  if (g > cap) g = cap;
  // The packed CIC counter holds at most kMaxBlockParticles per block and
  // turn.  Block b takes the groups of PPT particles b·T + t + k·g·T: at most
  // ceil((n / PPT) / (g·T)) steps of T·PPT particles, and block 0 also the
  // n mod PPT tail.  So g is raised until no block takes more steps than fit.
  const int64_t threads = pass_cfg_threads(cfg);
  const int64_t steps = kMaxBlockParticles / ((int64_t)pass_cfg_ppt(cfg) * threads);
  const int64_t groups = n / pass_cfg_ppt(cfg);
  const int64_t need = (groups + steps * threads - 1) / (steps * threads);
  if (g < need) g = need;
  if (g < 1) g = 1;
  return (int)g;
}

}  // namespace hj
