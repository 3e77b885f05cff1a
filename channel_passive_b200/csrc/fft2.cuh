// fft2.cuh - compile-time four-step FFTs for the 3/2-padded line lengths.
//
// A line of length N = N1 * N2 (natural order in shared memory) is transformed as
//   X[k2 + N2 k1] = sum_{n1} W_N^{n1 k2} W_{N1}^{n1 k1} [ sum_{n2} x[n1 + N1 n2] W_{N2}^{n2 k2} ]
// step 1: thread n1 loads x[n1 + N1 n2] (n2 < N2) into registers, runs an N2-point DFT,
//         multiplies by W_N^{n1 k2} and stores y at n1 + (N1+1) k2 (padded, conflict-free);
// step 2: thread k2 loads y[n1 + (N1+1) k2] (n1 < N1), runs an N1-point DFT and stores X at
//         k2 + N2 k1 (natural order).
// The small DFTs are Stockham autosort passes over register arrays whose indices are all
// compile-time constants, so no index arithmetic or digit reversal happens at run time.
// Sign convention: forward exp(-i 2 pi jk / M), backward exp(+i ...), unnormalised (FFTW's).
#pragma once

#include <cuda_runtime.h>

#include "fft.cuh"

namespace kmm {

// Twiddles exp(-i 2 pi t / M) of the register DFT sizes, filled by the host (api.cu).
constexpr int kRegSizes[] = {2, 3, 4, 6, 8, 9, 12, 16, 18, 24, 32};
constexpr int kNumRegSizes = 11;
constexpr int reg_tw_offset(int M) {
  int off = 0;
  for (int i = 0; i < kNumRegSizes; ++i) {
    if (kRegSizes[i] == M) return off;
    off += kRegSizes[i];
  }
  return -1;
}
constexpr int kRegTwTotal = 2 + 3 + 4 + 6 + 8 + 9 + 12 + 16 + 18 + 24 + 32;
// Defined in the one translation unit that includes this header (transforms2.cu).  The float2
// copy lets FP32 DFTs take their twiddles as constant operands without conversions.
__constant__ double2 c_regtw[kRegTwTotal];
__constant__ float2 c_regtw32[kRegTwTotal];

// First radix of the Stockham factorisation of M (4s first, then 2, then 3).
constexpr int first_radix(int M) { return (M % 4 == 0 && M != 8 && M != 32) || M == 4 ? 4 : (M % 2 == 0 ? 2 : 3); }

template <typename C, int M>
__device__ __forceinline__ C twr(int t, int sign) {
  constexpr int off = reg_tw_offset(M);  // evaluated at compile time: the table offset of size M
  static_assert(off >= 0, "register DFT size without a twiddle table");
  if constexpr (sizeof(C) == sizeof(float2)) {
    const float2 w = c_regtw32[off + t];
    return cmake<C>(w.x, sign > 0 ? -w.y : w.y);
  } else {
    const double2 w = c_regtw[off + t];
    return cmake<C>(w.x, sign > 0 ? -w.y : w.y);
  }
}

// One Stockham pass of radix R over M points: Ns = size of the sub-transforms already done.
template <typename C, int M, int R, int Ns>
__device__ __forceinline__ void stockham_pass(const C (&in)[M], C (&out)[M], int sign) {
  constexpr int Q = M / R;
#pragma unroll
  for (int idx = 0; idx < Q; ++idx) {
    const int k = idx % Ns;
    C a[R];
#pragma unroll
    for (int p = 0; p < R; ++p) {
      a[p] = in[idx + p * Q];
      if (p > 0 && k > 0) a[p] = cmul(a[p], twr<C, M>((p * k * (M / (Ns * R))) % M, sign));
    }
    if (R == 2) {
      const C x0 = a[0], x1 = a[1];
      a[0] = cadd(x0, x1);
      a[1] = csub(x0, x1);
    } else if (R == 4) {
      const C s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]), s13 = cadd(a[1], a[3]);
      const C d13 = cmul_si(csub(a[1], a[3]), sign);
      a[0] = cadd(s02, s13);
      a[2] = csub(s02, s13);
      a[1] = cadd(d02, d13);
      a[3] = csub(d02, d13);
    } else {  // R == 3
      using R_t = decltype(a[0].x);
      const R_t h = (R_t)0.86602540378443864676;  // sin(2 pi / 3)
      const C a0 = a[0], t1 = cadd(a[1], a[2]), t2 = csub(a[1], a[2]);
      C mm;
      mm.x = a0.x - (R_t)0.5 * t1.x;
      mm.y = a0.y - (R_t)0.5 * t1.y;
      C q = cmul_si(t2, sign);
      q.x *= h;
      q.y *= h;
      a[0] = cadd(a0, t1);
      a[1] = cadd(mm, q);
      a[2] = csub(mm, q);
    }
#pragma unroll
    for (int p = 0; p < R; ++p) out[(idx / Ns) * Ns * R + k + p * Ns] = a[p];
  }
}

template <typename C, int M, int Ns>
struct RegDft {
  // transforms v in place (natural order in and out); Ns = sub-transform size done so far
  static __device__ __forceinline__ void run(C (&v)[M], int sign) {
    constexpr int rem = M / Ns;
    constexpr int R = first_radix(rem);
    C t[M];
    stockham_pass<C, M, R, Ns>(v, t, sign);
#pragma unroll
    for (int i = 0; i < M; ++i) v[i] = t[i];
    RegDft<C, M, Ns * R>::run(v, sign);
  }
};
template <typename C, int M>
struct RegDft<C, M, M> {
  static __device__ __forceinline__ void run(C (&)[M], int) {}
};

template <typename C, int M>
__device__ __forceinline__ void reg_dft(C (&v)[M], int sign) {
  RegDft<C, M, 1>::run(v, sign);
}

// Four-step transform of nl lines of length N1*N2, natural order in and out.  The lines are
// line-major in shared memory: a (line l at a + l*lda, the input and the output) and b (the
// intermediate, line l at b + l*ldb, ldb >= (N1+1)*N2).  tw = exp(-i 2 pi t / N), t < N.
// Every thread of the block calls it; it ends with a barrier.
template <typename R, int N1, int N2>
__device__ __forceinline__ void fft4(typename Cpx<R>::T *a, int lda, typename Cpx<R>::T *b, int ldb, int nl,
                                     const typename Cpx<R>::T *tw, int sign) {
  using C = typename Cpx<R>::T;
  for (int it = threadIdx.x; it < nl * N1; it += blockDim.x) {
    const int l = it / N1, n1 = it - l * N1;
    const C *x = a + l * lda;
    C v[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) v[n2] = x[n1 + N1 * n2];
    reg_dft<C, N2>(v, sign);
    C *y = b + l * ldb;
    y[n1] = v[0];
#pragma unroll
    for (int k2 = 1; k2 < N2; ++k2) {
      C val = v[k2];
      if (n1 > 0) {
        C w = tw[n1 * k2];
        if (sign > 0) w.y = -w.y;
        val = cmul(val, w);
      }
      y[n1 + (N1 + 1) * k2] = val;
    }
  }
  __syncthreads();
  for (int it = threadIdx.x; it < nl * N2; it += blockDim.x) {
    const int l = it / N2, k2 = it - l * N2;
    const C *y = b + l * ldb;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = y[n1 + (N1 + 1) * k2];
    reg_dft<C, N1>(v, sign);
    C *X = a + l * lda;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) X[k2 + N2 * k1] = v[k1];
  }
  __syncthreads();
}

// The same transform in place: NL lines at a + l*lda with lda >= (N1+1)*N2, launched with NT
// threads.  Every thread keeps its step-1 (and step-2) work items in registers across a
// barrier before it overwrites the line, so no second buffer is needed.
template <int N1, int N2>
constexpr int ip_lda() {
  return ((N1 + 1) * N2) | 1;
}

template <typename R, int N1, int N2, int NL, int NT>
__device__ __forceinline__ void fft4_ip(typename Cpx<R>::T *a, int lda, const typename Cpx<R>::T *tw, int sign) {
  using C = typename Cpx<R>::T;
  constexpr int I1 = (NL * N1 + NT - 1) / NT, I2 = (NL * N2 + NT - 1) / NT;
  {
    C v[I1][N2];
#pragma unroll
    for (int i = 0; i < I1; ++i) {
      const int it = threadIdx.x + i * NT;
      if (I1 * NT == NL * N1 || it < NL * N1) {
        const int l = it / N1, n1 = it - l * N1;
        const C *x = a + l * lda;
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) v[i][n2] = x[n1 + N1 * n2];
        reg_dft<C, N2>(v[i], sign);
        if (n1 > 0) {
#pragma unroll
          for (int k2 = 1; k2 < N2; ++k2) {
            C w = tw[n1 * k2];
            if (sign > 0) w.y = -w.y;
            v[i][k2] = cmul(v[i][k2], w);
          }
        }
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < I1; ++i) {
      const int it = threadIdx.x + i * NT;
      if (I1 * NT == NL * N1 || it < NL * N1) {
        const int l = it / N1, n1 = it - l * N1;
        C *y = a + l * lda;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) y[n1 + (N1 + 1) * k2] = v[i][k2];
      }
    }
    __syncthreads();
  }
  {
    C v[I2][N1];
#pragma unroll
    for (int i = 0; i < I2; ++i) {
      const int it = threadIdx.x + i * NT;
      if (I2 * NT == NL * N2 || it < NL * N2) {
        const int l = it / N2, k2 = it - l * N2;
        const C *y = a + l * lda;
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) v[i][n1] = y[n1 + (N1 + 1) * k2];
        reg_dft<C, N1>(v[i], sign);
      }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < I2; ++i) {
      const int it = threadIdx.x + i * NT;
      if (I2 * NT == NL * N2 || it < NL * N2) {
        const int l = it / N2, k2 = it - l * N2;
        C *X = a + l * lda;
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) X[k2 + N2 * k1] = v[i][k1];
      }
    }
    __syncthreads();
  }
}

}  // namespace kmm
