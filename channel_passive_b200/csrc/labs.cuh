// labs.cuh - device LABS routines for one (kx, kz) system per thread.
//
// Restates the generic packed-band routines of module_labs.f90 (which its hand-unrolled
// BW = 1..10 variants specialise): fixed_bandec (:3487-3636, Crout LU without pivoting,
// pivots kept in L, unit U), fixed_banbks (:4252-4318, forward then backward substitution)
// and LABS_mat_mul_bw (:4687-4722).  BW is a template parameter so every inner loop has a
// compile-time trip count.  Indices are 1-based as in the reference.
//
// A thread's vectors are strided lines (stride = number of modes): lane t of a warp owns
// mode m0 + t, so each access of element i by a warp is one contiguous run.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace kmm {

__host__ __device__ __forceinline__ double2 z2(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ double2 zadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 zsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 zscale(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ double2 zdiv(double2 a, double2 b) {
  const double d = b.x * b.x + b.y * b.y;
  return make_double2((a.x * b.x + a.y * b.y) / d, (a.y * b.x - a.x * b.y) / d);
}

// (The helpers above, Line<double2>, BandM and the three routines below also compile for the
// host, where the restart reconstructions of initial_step.f90 use them with stride 1.)

// Strided complex line; storage double2 or float2, arithmetic always in double.
template <typename T> struct Line;
template <> struct Line<double2> {
  double2 *p;
  int64_t s;
  __host__ __device__ __forceinline__ double2 ld(int i) const { return p[(i - 1) * (int)s]; }
  __host__ __device__ __forceinline__ void st(int i, double2 v) const { p[(i - 1) * (int)s] = v; }
};
template <> struct Line<float2> {
  float2 *p;
  int64_t s;
  __device__ __forceinline__ double2 ld(int i) const {
    float2 v = p[(i - 1) * (int)s];
    return make_double2((double)v.x, (double)v.y);
  }
  __device__ __forceinline__ void st(int i, double2 v) const {
    p[(i - 1) * (int)s] = make_float2((float)v.x, (float)v.y);
  }
};
using DLine = Line<double2>;

// Band shared by all modes: A(r, j) = a[(j-1)*(2BW+1) + r-1].
template <int BW> struct BandS {
  const double *a;
  __device__ __forceinline__ double g(int r, int j) const { return __ldg(a + (j - 1) * (2 * BW + 1) + (r - 1)); }
};
// Band owned by one mode: A(r, j) = p[((j-1)*(2BW+1) + r-1) * s].
template <int BW> struct BandM {
  double *p;
  int64_t s;
  __host__ __device__ __forceinline__ double g(int r, int j) const {
    return p[((int64_t)(j - 1) * (2 * BW + 1) + (r - 1)) * s];
  }
  __host__ __device__ __forceinline__ void set(int r, int j, double v) const {
    p[((int64_t)(j - 1) * (2 * BW + 1) + (r - 1)) * s] = v;
  }
};

// fixed_bandec, module_labs.f90:3487-3636.
template <int BW>
__host__ __device__ __noinline__ void labs_lu(BandM<BW> A, int n) {
  constexpr int bw = BW, m = BW + 1;
  for (int i = 1; i <= bw; ++i) {  // upper region
    const double dummy = 1.0 / A.g(m, i);
#pragma unroll
    for (int j = 1; j <= bw; ++j) {
      if (j > bw + 1 - i) break;
      double acc = A.g(m + j, i);
      for (int k = 1; k <= i - 1; ++k) acc -= A.g(m - k, i) * A.g(m + j + k, i - k);
      A.set(m + j, i, dummy * acc);
    }
    for (int j = bw + 2 - i; j <= bw; ++j) {
      double acc = A.g(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A.g(m - k, i) * A.g(m + j + k, i - k);
      for (int k = bw - j + 1; k <= i - 1; ++k) acc -= A.g(m - k, i) * A.g(m + bw - i - j + 1, i - k);
      A.set(m + j, i, dummy * acc);
    }
    for (int j = i; j <= bw; ++j) {
      double acc = A.g(m - j, i);
      for (int k = 1; k <= i - 1; ++k) acc -= A.g(m - k, i) * A.g(m - j, i - k);
      A.set(m - j, i, dummy * acc);
    }
    for (int j = 1; j <= bw + 1 - i; ++j) {
      double acc = A.g(m + 1 - j, i + j);
      for (int k = 1; k <= i; ++k) acc -= A.g(m + 1 - j - k, i + j) * A.g(m + k, i + 1 - k);
      A.set(m + 1 - j, i + j, acc);
    }
    for (int j = bw + 2 - i; j <= bw; ++j) {
      double acc = A.g(m + 1 - j, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A.g(m + 1 - j - k, i + j) * A.g(m + k, i + 1 - k);
      A.set(m + 1 - j, i + j, acc);
    }
  }
  for (int i = m; i <= 2 * bw; ++i) {  // sub-upper region
    const double dummy = 1.0 / A.g(m, i);
    for (int j = 1; j <= 2 * bw + 1 - i; ++j) {
      double acc = A.g(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A.g(m - k, i) * A.g(m + j + k, i - k);
      for (int k = bw - j + 1; k <= bw; ++k) acc -= A.g(m - k, i) * A.g(2 * m - i - j, i - k);
      A.set(m + j, i, dummy * acc);
    }
    for (int j = 2 * bw + 2 - i; j <= bw; ++j) {
      double acc = A.g(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A.g(m - k, i) * A.g(m + j + k, i - k);
      A.set(m + j, i, dummy * acc);
    }
    for (int j = 1; j <= bw; ++j) {
      double acc = A.g(m - j + 1, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A.g(m - j + 1 - k, i + j) * A.g(m + k, i - k + 1);
      A.set(m - j + 1, i + j, acc);
    }
  }
  for (int i = 2 * bw + 1; i <= n - 2 * bw - 1; ++i) {  // centre region
    const double dummy = 1.0 / A.g(m, i);
#pragma unroll
    for (int j = 1; j <= bw; ++j) {
      double acc = A.g(m + j, i);
#pragma unroll
      for (int k = 1; k <= bw - j; ++k) acc -= A.g(m - k, i) * A.g(m + j + k, i - k);
      A.set(m + j, i, dummy * acc);
    }
#pragma unroll
    for (int j = 1; j <= bw; ++j) {
      double acc = A.g(m - j + 1, i + j);
#pragma unroll
      for (int k = 1; k <= bw - j + 1; ++k) acc -= A.g(m + 1 - j - k, i + j) * A.g(m + k, i + 1 - k);
      A.set(m - j + 1, i + j, acc);
    }
  }
  for (int i = n - 2 * bw; i <= n - bw - 1; ++i) {  // sub-lower region
    const double dummy = 1.0 / A.g(m, i);
    for (int j = 1; j <= bw; ++j) {
      double acc = A.g(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A.g(m - k, i) * A.g(m + j + k, i - k);
      A.set(m + j, i, dummy * acc);
    }
    for (int j = 1; j <= n - bw - i; ++j) {
      double acc = A.g(m - j + 1, i + j);
      for (int k = 1; k <= bw - j + 1; ++k) acc -= A.g(m + 1 - j - k, i + j) * A.g(m + k, i + 1 - k);
      A.set(m - j + 1, i + j, acc);
    }
    for (int j = n - bw - i + 1; j <= bw + 1; ++j) {
      double acc = A.g(m - j + 1, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A.g(m + 1 - j - k, i + j) * A.g(m + k, i + 1 - k);
      for (int k = bw + 2 - j; k <= i - n + 2 * bw + 1; ++k)
        acc -= A.g(m + n - bw - 1 + k - i, i + j) * A.g(m + k, i + 1 - k);
      A.set(m - j + 1, i + j, acc);
    }
    for (int j = bw + 2; j <= n - i; ++j) {
      double acc = A.g(m + n - bw - 1 - i, i + j);
      for (int k = 1; k <= i - n + 2 * bw + 1; ++k)
        acc -= A.g(m + n - bw - 1 - i + k, i + j) * A.g(m + k, i + 1 - k);
      A.set(m + n - bw - 1 - i, i + j, acc);
    }
  }
  for (int i = n - bw; i <= n - 1; ++i) {  // lower region
    const double dummy = 1.0 / A.g(m, i);
    for (int j = 1; j <= n - i; ++j) {
      double acc = A.g(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A.g(m - k, i) * A.g(m + j + k, i - k);
      A.set(m + j, i, dummy * acc);
    }
    for (int j = 1; j <= n - i; ++j) {
      double acc = A.g(m - j + 1, i + j);
      for (int k = 1; k <= 1 + bw - j; ++k) acc -= A.g(m + 1 - j - k, i + j) * A.g(m + k, i + 1 - k);
      for (int k = 2 + bw - j; k <= bw; ++k) acc -= A.g(m + n - bw - 1 - i + k, i + j) * A.g(m + k, i + 1 - k);
      A.set(m - j + 1, i + j, acc);
    }
  }
}

// fixed_banbks, module_labs.f90:4252-4318 (complex right-hand side, in place).
template <int BW, typename BandT, typename LineT>
__host__ __device__ __noinline__ void labs_bs(BandT A, LineT b, int n) {
  constexpr int bw = BW, m = BW + 1;
  for (int i = 1; i <= bw; ++i) {
    double2 acc = b.ld(i);
    for (int j = 1; j <= i - 1; ++j) acc = zsub(acc, zscale(A.g(m - i + j, i), b.ld(j)));
    const double d = A.g(m, i);
    b.st(i, z2(acc.x / d, acc.y / d));
  }
  for (int i = bw + 1; i <= n - bw; ++i) {
    double2 acc = b.ld(i);
#pragma unroll
    for (int j = 1; j <= bw; ++j) acc = zsub(acc, zscale(A.g(m - bw - 1 + j, i), b.ld(i - bw - 1 + j)));
    const double d = A.g(m, i);
    b.st(i, z2(acc.x / d, acc.y / d));
  }
  for (int i = 1; i <= bw; ++i) {
    const int r = n - bw + i;
    double2 acc = b.ld(r);
    for (int j = 1; j <= i; ++j) acc = zsub(acc, zscale(A.g(m + bw + 1 - j, r), b.ld(n - 2 * bw - 1 + j)));
    for (int j = i + 1; j <= i + bw; ++j) acc = zsub(acc, zscale(A.g(m - bw + j - i - 1, r), b.ld(n - 2 * bw - 1 + j)));
    const double d = A.g(m, r);
    b.st(r, z2(acc.x / d, acc.y / d));
  }
  for (int i = 1; i <= bw - 1; ++i) {
    double2 acc = b.ld(n - i);
    for (int j = 1; j <= i; ++j) acc = zsub(acc, zscale(A.g(m + j, n - i), b.ld(n - i + j)));
    b.st(n - i, acc);
  }
  for (int i = n - bw; i >= bw + 1; --i) {
    double2 acc = b.ld(i);
#pragma unroll
    for (int j = 1; j <= bw; ++j) acc = zsub(acc, zscale(A.g(m + j, i), b.ld(i + j)));
    b.st(i, acc);
  }
  for (int i = 1; i <= bw; ++i) {
    const int r = bw + 1 - i;
    double2 acc = b.ld(r);
    for (int j = 1; j <= bw; ++j) acc = zsub(acc, zscale(A.g(m + j, r), b.ld(r + j)));
    for (int j = bw + 1; j <= bw + i; ++j) acc = zsub(acc, zscale(A.g(m + i - j, r), b.ld(r + j)));
    b.st(r, acc);
  }
}

// LABS_mat_mul_bw, module_labs.f90:4687-4722: b = A x (x and b distinct).
template <int BW, typename BandT, typename XT, typename BT>
__host__ __device__ __noinline__ void labs_mat_mul(BandT A, XT x, BT b, int n) {
  constexpr int bw = BW;
  for (int j = 1; j <= bw; ++j) {
    double2 acc = z2(0.0, 0.0);
    for (int i = 1 - j; i <= bw; ++i) acc = zadd(acc, zscale(A.g(bw + 1 + i, j), x.ld(j + i)));
    for (int i = 1; i <= bw + 1 - j; ++i) acc = zadd(acc, zscale(A.g(bw + 2 - j - i, j), x.ld(j + bw + i)));
    b.st(j, acc);
  }
  for (int j = bw + 1; j <= n - bw; ++j) {
    double2 acc = z2(0.0, 0.0);
#pragma unroll
    for (int i = -bw; i <= bw; ++i) acc = zadd(acc, zscale(A.g(bw + 1 + i, j), x.ld(j + i)));
    b.st(j, acc);
  }
  for (int j = n - bw + 1; j <= n; ++j) {
    double2 acc = z2(0.0, 0.0);
    for (int i = -bw; i <= n - j; ++i) acc = zadd(acc, zscale(A.g(bw + 1 + i, j), x.ld(j + i)));
    for (int i = 1; i <= j - n + bw; ++i) acc = zadd(acc, zscale(A.g(n + bw + 1 - j + i, j), x.ld(j - bw - i)));
    b.st(j, acc);
  }
}

}  // namespace kmm
