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
}  // namespace hj
