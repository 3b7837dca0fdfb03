// PML damping profile shared by the host set-up and the device-built body,
// so both give the same planes.
#pragma once

#include <cmath>

namespace fdmap {

// damping in one direction at coordinate x (rates.f90:2065-2068):
// sigma*|max(0, lo - x, x - hi)|^n, or sigma itself when n = 0
#ifdef __CUDACC__
__host__ __device__
#endif
inline double pml_damping(double sigma, double n, double lo, double hi, double x) {
  if (!(n > 0.0)) return sigma;
  return sigma * pow(fabs(fmax(0.0, fmax(lo - x, x - hi))), n);
}

}  // namespace fdmap
