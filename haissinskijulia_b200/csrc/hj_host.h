// hj_host.h -- host-side table builders (hj_host.cpp), not part of the ABI.
#pragma once

#include <cstdint>

#include "../../include/haissinski_gpu.h"

namespace hj {
double host_wake_function(double c, const hj_wake& w);
double host_delta(double x, double sigma);
void host_wake_tables(const double* centers, int64_t B, const hj_wake& w, double* W,
                      double* lam);
void host_twiddles(int64_t P, double* tw_interleaved);
void host_rf_table(double V, double phi_s, int64_t M, double* tab_interleaved);
// Tables of the device's Float64 normals: a 2048-layer ziggurat for the
// density f(x) = exp(-x²/2), x >= 0 (G. Marsaglia and W. W. Tsang, "The
// Ziggurat Method for Generating Random Variables", J. Stat. Softw. 5(8),
// 2000), as hj_device.cuh (zig_fast, zig_slow) samples it.  Layer 0 is the
// base: the rectangle [0, r) x [0, f(r)) plus the tail x >= r, of area v;
// layer i >= 1 is the rectangle [0, X_i) x [f(X_i), f(X_{i+1})), also of
// area v, with X_1 = r, X_2048 = 0 and X_0 = v / f(r).
constexpr int kZigLayers = 2048;
struct NormalTables {
  // (X_i, D_i): layer i's width and its fast-acceptance bound D_i = 1 + K_i 2^-52,
  // K_i = ceil(2^52 X_{i+1} / X_i): a draw U = m 2^-52 of layer i with
  // 1 + m 2^-52 < D_i lies under the curve whatever its height.
  double xd[kZigLayers][2];
  double f[kZigLayers + 1];   // f(X_i), f(X_2048) = 1: the wedge tests
  double r;                   // X_1: where the tail begins
  double v;                   // the common area of the layers
};
// Solves for r in extended precision (bisection on the layer recursion
// X_{i+1} = sqrt(-2 ln(f(X_i) + v / X_i)) until X_2048 = 0) and fills the
// tables, each entry rounded once.
void host_normal_tables(NormalTables* t);
}  // namespace hj
