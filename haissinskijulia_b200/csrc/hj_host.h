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
// Tables of the device's double-precision Box-Muller transform
// (hj_device.cuh, box_muller_f64).
constexpr int kNormalTableRows = 128;
struct NormalTables {
  double lr[kNormalTableRows][2];   // logarithm: (r_j, -ln r_j), r_j = 1/(1 + (j + 1/2)/128)
  double sc[kNormalTableRows][2];   // angles: (sin θ_j, cos θ_j), θ_j = 2π (j + 1/2)/128
  double ln2_hi, ln2_lo; // ln 2: high part of 42 bits, and the rest
  double twopi_hi, twopi_lo;   // 2π: double, and the rest
};
// Fills the tables in extended precision (logl, sinl, cosl), each entry
// rounded once.
void host_normal_tables(NormalTables* t);
}  // namespace hj
