// stats.cuh - the physical-space moment terms of a statistics substep, shared by the x pass
// (transforms2.cu) and the statistics kernels (stats.cu).
#pragma once

#include "kmm_internal.h"

namespace kmm {

// Adds the moment terms of one physical point (dft_x_realspace.f90:128-155) to s:
//   s[0..2]  u^3,  v^3,  w^3          s[3..5]   u^4, v^4, w^4
//   s[6..8]  u^6,  v^6,  w^6          s[9..11]  u^8, v^8, w^8
//   s[12..14] u^10, v^10, w^10        s[15] -u u v,  s[16] -v w w,  s[17] -u v v
// with the raw velocities (the reference's mean subtraction is commented out).
__device__ __forceinline__ void moment_terms(double (&s)[kNumMoments], double u, double v, double w) {
  const double x[3] = {u, v, w};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double x2 = x[c] * x[c], x4 = x2 * x2, x8 = x4 * x4;
    s[c] += x2 * x[c];
    s[3 + c] += x4;
    s[6 + c] += x4 * x2;
    s[9 + c] += x8;
    s[12 + c] += x8 * x2;
  }
  s[15] -= u * u * v;
  s[16] -= v * w * w;
  s[17] -= u * v * v;
}

}  // namespace kmm
