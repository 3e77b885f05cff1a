// fft.cuh - batched in-place mixed-radix (2,3,4,5) complex FFTs on shared-memory lines.
//
// Replaces the FFTW 1-D plans of module_ppdfftw.f90:456-477 (c2c length nz32 both
// directions, r2c / c2r length nx32).  Unnormalised, FFTW sign convention:
// forward = exp(-i 2 pi jk/n), backward = exp(+i 2 pi jk/n).
//
// Shared-memory layout: element (position p, line l) at buf[p * ls + l], so the lines of a
// batch are interleaved and consecutive threads touch consecutive words.
//  * dit():  input at the digit-reversed positions pos[i] (written by the loader), output in
//            natural order.  Pass q combines r_q sub-transforms of length L_{q-1}.
//  * dif():  natural-order input, output frequency k at position pos[k] (read by the storer).
// The radix list and pos table come from the host plan (api.cu: make_fft_plan).
#pragma once

#include <cuda_runtime.h>

#include "kmm_internal.h"

namespace kmm {

template <typename R> struct Cpx;
template <> struct Cpx<double> { using T = double2; };
template <> struct Cpx<float> { using T = float2; };

template <typename C> __device__ __forceinline__ C cmake(double a, double b);
template <> __device__ __forceinline__ double2 cmake<double2>(double a, double b) { return make_double2(a, b); }
template <> __device__ __forceinline__ float2 cmake<float2>(double a, double b) { return make_float2((float)a, (float)b); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { C r; r.x = a.x + b.x; r.y = a.y + b.y; return r; }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { C r; r.x = a.x - b.x; r.y = a.y - b.y; return r; }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  C r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// multiply by (s * i), s = +1 or -1
template <typename C> __device__ __forceinline__ C cmul_si(C a, int s) {
  C r;
  if (s > 0) { r.x = -a.y; r.y = a.x; } else { r.x = a.y; r.y = -a.x; }
  return r;
}

template <typename R> __device__ __forceinline__ typename Cpx<R>::T twiddle(const FftPlan &pl, int t, int sign);
template <> __device__ __forceinline__ double2 twiddle<double>(const FftPlan &pl, int t, int sign) {
  double2 w = __ldg(pl.tw64 + t);
  if (sign > 0) w.y = -w.y;
  return w;
}
template <> __device__ __forceinline__ float2 twiddle<float>(const FftPlan &pl, int t, int sign) {
  float2 w = __ldg(pl.tw32 + t);
  if (sign > 0) w.y = -w.y;
  return w;
}

// In-register r-point DFT, v[0..r-1] -> v[0..r-1], sign = -1 forward, +1 backward.
template <typename R>
__device__ __forceinline__ void small_dft(typename Cpx<R>::T *v, int r, int sign, const FftPlan &pl) {
  using C = typename Cpx<R>::T;
  if (r == 2) {
    C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  } else if (r == 4) {
    C a0 = v[0], a1 = v[1], a2 = v[2], a3 = v[3];
    C s02 = cadd(a0, a2), d02 = csub(a0, a2), s13 = cadd(a1, a3), d13 = cmul_si(csub(a1, a3), sign);
    v[0] = cadd(s02, s13);
    v[2] = csub(s02, s13);
    v[1] = cadd(d02, d13);
    v[3] = csub(d02, d13);
  } else if (r == 3) {
    const R h = (R)0.86602540378443864676;  // sin(2 pi / 3)
    C a0 = v[0], t1 = cadd(v[1], v[2]), t2 = csub(v[1], v[2]);
    C m;
    m.x = a0.x - (R)0.5 * t1.x;
    m.y = a0.y - (R)0.5 * t1.y;
    C q = cmul_si(t2, sign);
    q.x *= h;
    q.y *= h;
    v[0] = cadd(a0, t1);
    v[1] = cadd(m, q);
    v[2] = csub(m, q);
  } else {  // generic (radix 5): twiddles from the length-n table
    C in[5];
    for (int j = 0; j < r; ++j) in[j] = v[j];
    const int step = pl.n / r;
    for (int s = 0; s < r; ++s) {
      C acc = in[0];
      for (int j = 1; j < r; ++j) acc = cadd(acc, cmul(in[j], twiddle<R>(pl, (j * s % r) * step, sign)));
      v[s] = acc;
    }
  }
}

// Decimation in time over nl lines; input at pos[], output natural.  Call with all threads
// of the block; ends with a __syncthreads().
template <typename R>
__device__ void fft_dit(typename Cpx<R>::T *buf, int ls, int nl, const FftPlan &pl, int sign) {
  using C = typename Cpx<R>::T;
  const int n = pl.n;
  int lp = 1;
  for (int q = 0; q < pl.npass; ++q) {
    const int r = pl.radix[q];
    const int lq = lp * r;
    const int tstep = n / lq;
    const int nb = n / r;
    for (int w = threadIdx.x; w < nb * nl; w += blockDim.x) {
      const int l = w % nl, b = w / nl;
      const int g = b / lp, k = b - g * lp;
      const int base = g * lq + k;
      C v[5];
      for (int j = 0; j < r; ++j) {
        C x = buf[(base + j * lp) * ls + l];
        v[j] = (j == 0 || k == 0) ? x : cmul(x, twiddle<R>(pl, (j * k * tstep) % n, sign));
      }
      small_dft<R>(v, r, sign, pl);
      for (int j = 0; j < r; ++j) buf[(base + j * lp) * ls + l] = v[j];
    }
    __syncthreads();
    lp = lq;
  }
}

// Decimation in frequency over nl lines; input natural, output frequency k at pos[k].
template <typename R>
__device__ void fft_dif(typename Cpx<R>::T *buf, int ls, int nl, const FftPlan &pl, int sign) {
  using C = typename Cpx<R>::T;
  const int n = pl.n;
  int lq = n;
  for (int q = pl.npass - 1; q >= 0; --q) {
    const int r = pl.radix[q];
    const int lp = lq / r;
    const int tstep = n / lq;
    const int nb = n / r;
    for (int w = threadIdx.x; w < nb * nl; w += blockDim.x) {
      const int l = w % nl, b = w / nl;
      const int g = b / lp, k = b - g * lp;
      const int base = g * lq + k;
      C v[5];
      for (int j = 0; j < r; ++j) v[j] = buf[(base + j * lp) * ls + l];
      small_dft<R>(v, r, sign, pl);
      for (int j = 0; j < r; ++j)
        buf[(base + j * lp) * ls + l] =
            (j == 0 || k == 0) ? v[j] : cmul(v[j], twiddle<R>(pl, (j * k * tstep) % n, sign));
    }
    __syncthreads();
    lq = lp;
  }
}

}  // namespace kmm
