// transforms2.cu - the substep's transforms with compile-time four-step FFTs (fft2.cuh).
//
// Same contracts as transforms.cu (k_zinv / k_xphys / k_zfwd: y_to_x, dft_x_realspace and
// x_to_y with rescale_data folded in) for the line lengths N = N1 * N2 listed in fft4_shape;
// the launchers fall back to the generic kernels of transforms.cu for other lengths.  Lines
// are line-major in shared memory with an odd leading dimension, natural order in and out, so
// the 3/2 padding and truncation read and write plain positions k and N - k.
#include <cuda_runtime.h>

#include "fft2.cuh"
#include "kmm_internal.h"

namespace kmm {

namespace {

constexpr int kT2 = 256;

template <typename C> __device__ __forceinline__ C ld_as(const double2 *p) {
  const double2 v = *p;
  return cmake<C>(v.x, v.y);
}
template <typename R> __device__ __forceinline__ const typename Cpx<R>::T *tw_of(const FftPlan &pl);
template <> __device__ __forceinline__ const double2 *tw_of<double>(const FftPlan &pl) { return pl.tw64; }
template <> __device__ __forceinline__ const float2 *tw_of<float>(const FftPlan &pl) { return pl.tw32; }

constexpr int lda_of(int N) { return N | 1; }
constexpr int ldb_of(int N1, int N2) { return ((N1 + 1) * N2) | 1; }

// y_to_x: grid (ceil(nxh/KB), ny, nfield)
template <typename R, int N1, int N2, int KB>
__global__ void __launch_bounds__(kT2) k_zinv2(const double2 *__restrict__ src, typename Cpx<R>::T *__restrict__ dst,
                                               FftPlan pl, int nz, int nxh, int64_t ns, int64_t nm) {
  using C = typename Cpx<R>::T;
  constexpr int N = N1 * N2, LDA = lda_of(N), LDB = ldb_of(N1, N2);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + KB * LDA;
  const int nh = nz / 2;
  const int kx0 = blockIdx.x * KB, y = blockIdx.y, f = blockIdx.z;
  const double2 *sp = src + f * ns + (int64_t)y * nz * nxh;
  for (int w = threadIdx.x; w < N * KB; w += blockDim.x) {
    const int l = w % KB, p = w / KB;
    int kzi = -1;
    if (p < nh) kzi = p;
    else if (p > 2 * nh) kzi = p - nh;
    C v = cmake<C>(0.0, 0.0);
    if (kzi >= 0 && kx0 + l < nxh) v = ld_as<C>(sp + (int64_t)kzi * nxh + kx0 + l);
    a[l * LDA + p] = v;
  }
  __syncthreads();
  fft4<R, N1, N2>(a, LDA, b, LDB, KB, tw_of<R>(pl), +1);
  C *dp = dst + f * nm + (int64_t)y * N * nxh;
  for (int w = threadIdx.x; w < N * KB; w += blockDim.x) {
    const int l = w % KB, z = w / KB;
    if (kx0 + l < nxh) dp[(int64_t)z * nxh + kx0 + l] = a[l * LDA + z];
  }
}

// x_to_y: grid (ceil(nxh/KB), ny, nfield)
template <typename R, int N1, int N2, int KB, typename D>
__global__ void __launch_bounds__(kT2) k_zfwd2(const typename Cpx<R>::T *__restrict__ src, D *__restrict__ dst,
                                               FftPlan pl, int nz, int nxh, int64_t ns, int64_t nm, double scale) {
  using C = typename Cpx<R>::T;
  constexpr int N = N1 * N2, LDA = lda_of(N), LDB = ldb_of(N1, N2);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *a = reinterpret_cast<C *>(smem_raw);
  C *b = a + KB * LDA;
  const int nh = nz / 2;
  const int kx0 = blockIdx.x * KB, y = blockIdx.y, f = blockIdx.z;
  const C *sp = src + f * nm + (int64_t)y * N * nxh;
  for (int w = threadIdx.x; w < N * KB; w += blockDim.x) {
    const int l = w % KB, z = w / KB;
    a[l * LDA + z] = (kx0 + l < nxh) ? sp[(int64_t)z * nxh + kx0 + l] : cmake<C>(0.0, 0.0);
  }
  __syncthreads();
  fft4<R, N1, N2>(a, LDA, b, LDB, KB, tw_of<R>(pl), -1);
  D *dp = dst + f * ns + (int64_t)y * nz * nxh;
  for (int w = threadIdx.x; w < nz * KB; w += blockDim.x) {
    const int l = w % KB, kzi = w / KB;
    if (kx0 + l >= nxh) continue;
    const int k = (kzi < nh) ? kzi : (kzi == nh ? -1 : kzi + nh);
    D out;
    if (k < 0) {
      out.x = 0;
      out.y = 0;
    } else {
      const C v = a[l * LDA + k];
      out.x = (decltype(out.x))(scale * (double)v.x);
      out.y = (decltype(out.y))(scale * (double)v.y);
    }
    dp[(int64_t)kzi * nxh + kx0 + l] = out;
  }
}

struct X2Args {
  int ny, nz32, nxh;
  int64_t nm;
  double dxr, dzr;
  const double *dyr;
  int substep;
  DevScalars *dsc;
};

// dft_x_realspace: grid (ceil(nz32/ZB), ny); MID slots 0..3 = u, v, w, theta in,
// slots 0..7 = f1, f2, f3, f4, f5, f7, f8, f9 out (a block owns its rows).
template <typename R, int N1, int N2, int ZB>
__global__ void __launch_bounds__(kT2) k_xphys2(typename Cpx<R>::T *__restrict__ mid, FftPlan pl, X2Args a_) {
  using C = typename Cpx<R>::T;
  constexpr int N = N1 * N2, LDA = lda_of(N), LDB = ldb_of(N1, N2);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *a = reinterpret_cast<C *>(smem_raw);  // 4*ZB lines: (u,v) ZB, (w,theta) ZB, then f57, f89
  C *b = a + 4 * ZB * LDA;
  const int nxh = a_.nxh;
  const int z0 = blockIdx.x * ZB, y = blockIdx.y;
  const int64_t row0 = ((int64_t)y * a_.nz32 + z0) * nxh;
  for (int w = threadIdx.x; w < 2 * ZB * N; w += blockDim.x) {
    const int L = w / N, p = w - L * N;
    a[L * LDA + p] = cmake<C>(0.0, 0.0);
  }
  __syncthreads();
  // Z_k = X1_k + i X2_k and its Hermitian mirror at N - k; DC imaginary parts dropped (c2r)
  for (int w = threadIdx.x; w < 2 * ZB * nxh; w += blockDim.x) {
    const int k = w % nxh, t = w / nxh, l = t % ZB, bsel = t / ZB;
    if (z0 + l >= a_.nz32) continue;
    const int64_t off = row0 + (int64_t)l * nxh + k;
    const int fa = bsel ? 2 : 0, fb = bsel ? 3 : 1;
    const C x1 = mid[fa * a_.nm + off], x2 = mid[fb * a_.nm + off];
    C *line = a + (bsel * ZB + l) * LDA;
    if (k == 0) {
      line[0] = cmake<C>(x1.x, x2.x);
    } else {
      C zk, zm;
      zk.x = x1.x - x2.y; zk.y = x1.y + x2.x;
      zm.x = x1.x + x2.y; zm.y = x2.x - x1.y;
      line[k] = zk;
      line[N - k] = zm;
    }
  }
  __syncthreads();
  fft4<R, N1, N2>(a, LDA, b, LDB, 2 * ZB, tw_of<R>(pl), +1);
  const double dyr = a_.dyr[y];
  double vmax = 0.0;
  int bad = 0;
  for (int w = threadIdx.x; w < ZB * N; w += blockDim.x) {
    const int l = w / N, p = w - l * N;
    const C uv = a[l * LDA + p], wt = a[(ZB + l) * LDA + p];
    const R u = uv.x, v = uv.y, ww = wt.x, t = wt.y;
    const R bv2 = v * v;
    C f12, f34, f57, f89;
    f12.x = u * u - bv2; f12.y = u * v;
    f34.x = ww * ww - bv2; f34.y = v * ww;
    f57.x = u * ww; f57.y = u * t;
    f89.x = v * t; f89.y = ww * t;
    a[l * LDA + p] = f12;
    a[(ZB + l) * LDA + p] = f34;
    a[(2 * ZB + l) * LDA + p] = f57;
    a[(3 * ZB + l) * LDA + p] = f89;
    if (a_.substep == 1 && z0 + l < a_.nz32) {
      const double vel = (fabs((double)u) * a_.dxr) + (fabs((double)v) * dyr) + (fabs((double)ww) * a_.dzr);
      if (!isfinite(vel)) bad = 1;
      else vmax = fmax(vmax, vel);
    }
  }
  __syncthreads();
  fft4<R, N1, N2>(a, LDA, b, LDB, 4 * ZB, tw_of<R>(pl), -1);
  for (int w = threadIdx.x; w < 4 * ZB * nxh; w += blockDim.x) {
    const int k = w % nxh, t = w / nxh, l = t % ZB, bsel = t / ZB;
    if (z0 + l >= a_.nz32) continue;
    const C *line = a + (bsel * ZB + l) * LDA;
    const C zk = line[k], zm = line[k == 0 ? 0 : N - k];
    C A, B;
    A.x = (R)0.5 * (zk.x + zm.x); A.y = (R)0.5 * (zk.y - zm.y);
    B.x = (R)0.5 * (zk.y + zm.y); B.y = (R)0.5 * (zm.x - zk.x);
    const int64_t off = row0 + (int64_t)l * nxh + k;
    mid[(2 * bsel) * a_.nm + off] = A;
    mid[(2 * bsel + 1) * a_.nm + off] = B;
  }
  if (a_.substep == 1) {
    __shared__ double red[kT2 / 32];
    __shared__ int redbad;
    if (threadIdx.x == 0) redbad = 0;
    __syncthreads();
    if (bad) atomicOr(&redbad, 1);
    for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
      for (int i = 0; i < (int)(blockDim.x >> 5); ++i) m = fmax(m, red[i]);
      atomicMax(&a_.dsc->velmax_bits, (unsigned long long)__double_as_longlong(m));
      if (redbad) atomicOr(&a_.dsc->nonfinite, 1);
    }
  }
}

// ---- dispatch over the supported lengths ------------------------------------------------
template <typename F> bool with_shape(int N, F &&f) {
  switch (N) {
    case 12: f.template operator()<3, 4>(); return true;
    case 24: f.template operator()<4, 6>(); return true;
    case 36: f.template operator()<6, 6>(); return true;
    case 48: f.template operator()<6, 8>(); return true;
    case 72: f.template operator()<8, 9>(); return true;
    case 96: f.template operator()<8, 12>(); return true;
    case 144: f.template operator()<12, 12>(); return true;
    case 192: f.template operator()<12, 16>(); return true;
    case 288: f.template operator()<16, 18>(); return true;
    case 384: f.template operator()<16, 24>(); return true;
    case 576: f.template operator()<24, 24>(); return true;
    default: return false;
  }
}

template <typename K> void set_smem(K kern, int optin) {
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) return;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
}

template <typename R> constexpr int zkb() { return sizeof(R) == 8 ? 8 : 16; }

template <typename R, int N1, int N2>
size_t xphys_zb_bytes(int zb) {
  using C = typename Cpx<R>::T;
  return sizeof(C) * (size_t)4 * zb * (lda_of(N1 * N2) + ldb_of(N1, N2));
}

}  // namespace

cudaError_t fill_regtw() {
  double2 h[kRegTwTotal];
  int off = 0;
  for (int i = 0; i < kNumRegSizes; ++i) {
    const int M = kRegSizes[i];
    for (int t = 0; t < M; ++t) {
      const long double ang = -2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)M;
      h[off + t] = make_double2((double)cosl(ang), (double)sinl(ang));
    }
    off += M;
  }
  return cudaMemcpyToSymbol(c_regtw, h, sizeof(h));
}

bool fft4_supported(int N) {
  return with_shape(N, [&]<int A, int B>() {});
}

cudaError_t prepare_transforms2() {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const cudaError_t e = fill_regtw();
  if (e != cudaSuccess) return e;
  for (int N : {12, 24, 36, 48, 72, 96, 144, 192, 288, 384, 576}) {
    with_shape(N, [&]<int N1, int N2>() {
      set_smem(k_zinv2<double, N1, N2, 8>, optin);
      set_smem(k_zinv2<float, N1, N2, 16>, optin);
      set_smem(k_zfwd2<double, N1, N2, 8, double2>, optin);
      set_smem(k_zfwd2<float, N1, N2, 16, float2>, optin);
      set_smem(k_zfwd2<float, N1, N2, 16, double2>, optin);
      set_smem(k_xphys2<double, N1, N2, 4>, optin);
      set_smem(k_xphys2<double, N1, N2, 2>, optin);
      set_smem(k_xphys2<double, N1, N2, 1>, optin);
      set_smem(k_xphys2<float, N1, N2, 8>, optin);
      set_smem(k_xphys2<float, N1, N2, 4>, optin);
      set_smem(k_xphys2<float, N1, N2, 2>, optin);
      set_smem(k_xphys2<float, N1, N2, 1>, optin);
    });
  }
  return cudaSuccess;
}

// Returns cudaErrorNotSupported when the length has no four-step shape (caller falls back).
cudaError_t launch_zinv2(Handle &h, const double2 *src, void *mid, int nfield, cudaStream_t st) {
  cudaError_t err = cudaErrorNotSupported;
  const int N = h.nz32;
  auto go = [&]<typename R>() {
    with_shape(N, [&]<int N1, int N2>() {
      using C = typename Cpx<R>::T;
      constexpr int KB = zkb<R>();
      const size_t smem = sizeof(C) * (size_t)KB * (lda_of(N1 * N2) + ldb_of(N1, N2));
      dim3 grid((unsigned)((h.nxh + KB - 1) / KB), (unsigned)h.ny, (unsigned)nfield);
      k_zinv2<R, N1, N2, KB><<<grid, kT2, smem, st>>>(src, reinterpret_cast<C *>(mid), h.pz, h.nz, h.nxh, h.ns, h.nm);
      err = cudaGetLastError();
    });
  };
  if (h.mixed) go.template operator()<float>();
  else go.template operator()<double>();
  return err;
}

cudaError_t launch_zfwd2(Handle &h, const void *mid, void *dst, int nfield, double scale, bool dst_fp64,
                         cudaStream_t st) {
  cudaError_t err = cudaErrorNotSupported;
  const int N = h.nz32;
  auto go = [&]<typename R, typename D>() {
    with_shape(N, [&]<int N1, int N2>() {
      using C = typename Cpx<R>::T;
      constexpr int KB = zkb<R>();
      const size_t smem = sizeof(C) * (size_t)KB * (lda_of(N1 * N2) + ldb_of(N1, N2));
      dim3 grid((unsigned)((h.nxh + KB - 1) / KB), (unsigned)h.ny, (unsigned)nfield);
      k_zfwd2<R, N1, N2, KB, D><<<grid, kT2, smem, st>>>(reinterpret_cast<const C *>(mid), reinterpret_cast<D *>(dst),
                                                         h.pz, h.nz, h.nxh, h.ns, h.nm, scale);
      err = cudaGetLastError();
    });
  };
  if (h.mixed) {
    if (dst_fp64) go.template operator()<float, double2>();
    else go.template operator()<float, float2>();
  } else {
    go.template operator()<double, double2>();
  }
  return err;
}

cudaError_t launch_xphys2(Handle &h, void *mid, int substep, cudaStream_t st) {
  cudaError_t err = cudaErrorNotSupported;
  const int N = h.nx32;
  X2Args a;
  a.ny = h.ny;
  a.nz32 = h.nz32;
  a.nxh = h.nxh;
  a.nm = h.nm;
  a.dxr = h.dxr;
  a.dzr = h.dzr;
  a.dyr = h.dops + ops_offsets(h.bw, h.ny).dyr;
  a.substep = substep;
  a.dsc = h.dsc;
  auto go = [&]<typename R>() {
    with_shape(N, [&]<int N1, int N2>() {
      using C = typename Cpx<R>::T;
      const size_t lim = 200 * 1024;
      auto launch = [&]<int ZB>() {
        const size_t smem = xphys_zb_bytes<R, N1, N2>(ZB);
        dim3 grid((unsigned)((h.nz32 + ZB - 1) / ZB), (unsigned)h.ny);
        k_xphys2<R, N1, N2, ZB><<<grid, kT2, smem, st>>>(reinterpret_cast<C *>(mid), h.px, a);
        err = cudaGetLastError();
      };
      if (sizeof(R) == 4 && xphys_zb_bytes<R, N1, N2>(8) <= lim) launch.template operator()<8>();
      else if (xphys_zb_bytes<R, N1, N2>(4) <= lim) launch.template operator()<4>();
      else if (xphys_zb_bytes<R, N1, N2>(2) <= lim) launch.template operator()<2>();
      else launch.template operator()<1>();
    });
  };
  if (h.mixed) go.template operator()<float>();
  else go.template operator()<double>();
  return err;
}

}  // namespace kmm
