// transforms.cu - the spectral <-> physical round trip of one substep.
//
//   k_zinv   y_to_x  (y_to_x.f90:21-50): Y-planes -> pad kz (module_ppdfftw.f90:846-854)
//            -> backward c2c along z -> MID (= the reference X-pencil).  The y->z->x
//            pencil transposes (on_node_*order_*, module_ppdfftw.f90:883-1146) become the
//            shared-memory staging of a (kz x kx-block) tile.
//   k_xphys  dft_x_realspace (dft_x_realspace.f90:68-213): pad kx, c2r, the nonlinear
//            products, CFL maximum, r2c, truncate; two real lines share one complex FFT.
//   k_zfwd   x_to_y (x_to_y.f90:21-46): forward c2c along z, keep 1..nz/2, zero the kz
//            Nyquist, shift the negative modes down (module_ppdfftw.f90:809-818), and
//            rescale_data's 1/(nx32 nz32) (rescale_data.f90:31-33) in the same store.
#include <cuda_runtime.h>

#include <cfloat>

#include "fft.cuh"
#include "kmm_internal.h"

namespace kmm {

namespace {

constexpr int kThreads = 256;

template <typename C> __device__ __forceinline__ C load_as(const double2 *p) {
  double2 v = *p;
  return cmake<C>(v.x, v.y);
}


// ---------------------------------------------------------------------------------------
// z inverse: grid (ceil(nxh/KB), ny, nfield); src planes [f][y][kz][kx] double2;
// dst MID [f][y][z32][kx] R2.
template <typename R, int KB>
__global__ void __launch_bounds__(kThreads) k_zinv(const double2 *__restrict__ src,
                                                   typename Cpx<R>::T *__restrict__ dst,
                                                   FftPlan pl, int ny, int nz, int nxh,
                                                   int64_t ns, int64_t nm) {
  using C = typename Cpx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int n = pl.n, nh = nz / 2;
  const int kx0 = blockIdx.x * KB, y = blockIdx.y, f = blockIdx.z;
  const double2 *sp = src + f * ns + (int64_t)y * nz * nxh;
  for (int w = threadIdx.x; w < n * KB; w += blockDim.x) {
    const int l = w % KB, p = w / KB;
    int kzi = -1;
    if (p < nh) kzi = p;
    else if (p > 2 * nh) kzi = p - nh;
    C v = cmake<C>(0.0, 0.0);
    if (kzi >= 0 && kx0 + l < nxh) v = load_as<C>(sp + (int64_t)kzi * nxh + kx0 + l);
    buf[__ldg(pl.pos + p) * KB + l] = v;
  }
  __syncthreads();
  fft_dit<R>(buf, KB, KB, pl, +1);
  C *dp = dst + f * nm + (int64_t)y * n * nxh;
  for (int w = threadIdx.x; w < n * KB; w += blockDim.x) {
    const int l = w % KB, z = w / KB;
    if (kx0 + l < nxh) dp[(int64_t)z * nxh + kx0 + l] = buf[z * KB + l];
  }
}

// ---------------------------------------------------------------------------------------
// z forward: grid (ceil(nxh/KB), ny, nfield); src MID R2, dst planes (R2 or double2).
template <typename R, int KB, typename D>
__global__ void __launch_bounds__(kThreads) k_zfwd(const typename Cpx<R>::T *__restrict__ src,
                                                   D *__restrict__ dst, FftPlan pl, int ny,
                                                   int nz, int nxh, int64_t ns, int64_t nm,
                                                   double scale) {
  using C = typename Cpx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  const int n = pl.n, nh = nz / 2;
  const int kx0 = blockIdx.x * KB, y = blockIdx.y, f = blockIdx.z;
  const C *sp = src + f * nm + (int64_t)y * n * nxh;
  for (int w = threadIdx.x; w < n * KB; w += blockDim.x) {
    const int l = w % KB, z = w / KB;
    buf[z * KB + l] = (kx0 + l < nxh) ? sp[(int64_t)z * nxh + kx0 + l] : cmake<C>(0.0, 0.0);
  }
  __syncthreads();
  fft_dif<R>(buf, KB, KB, pl, -1);
  D *dp = dst + f * ns + (int64_t)y * nz * nxh;
  for (int w = threadIdx.x; w < nz * KB; w += blockDim.x) {
    const int l = w % KB, kzi = w / KB;
    if (kx0 + l >= nxh) continue;
    int k = (kzi < nh) ? kzi : (kzi == nh ? -1 : kzi + nh);
    D out;
    if (k < 0) {
      out.x = 0;
      out.y = 0;
    } else {
      C v = buf[__ldg(pl.pos + k) * KB + l];
      out.x = (decltype(out.x))(scale * (double)v.x);
      out.y = (decltype(out.y))(scale * (double)v.y);
    }
    dp[(int64_t)kzi * nxh + kx0 + l] = out;
  }
}

// ---------------------------------------------------------------------------------------
// x physical step: grid (ceil(nz32/ZB), ny).  MID slots 0..3 = u, v, w, theta on entry;
// slots 0..7 = f1, f2, f3, f4, f5, f7, f8, f9 on exit (in place: a block owns its rows).
struct XArgs {
  int ny, nz32, nxh;
  int64_t nm;
  double dxr, dzr;
  const double *dyr;
  int substep;
  DevScalars *dsc;
};

template <typename R, int ZB>
__global__ void __launch_bounds__(kThreads) k_xphys(typename Cpx<R>::T *__restrict__ mid,
                                                    FftPlan pl, XArgs a) {
  using C = typename Cpx<R>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *buf = reinterpret_cast<C *>(smem_raw);
  constexpr int LS = 4 * ZB;  // 4 buffers of ZB lines interleaved
  const int n = pl.n, nxh = a.nxh;
  const int z0 = blockIdx.x * ZB, y = blockIdx.y;
  const int64_t row0 = ((int64_t)y * a.nz32 + z0) * nxh;
  // zero the two inverse buffers
  for (int w = threadIdx.x; w < n * 2 * ZB; w += blockDim.x) {
    const int p = w / (2 * ZB), L = w % (2 * ZB);
    buf[p * LS + L] = cmake<C>(0.0, 0.0);
  }
  __syncthreads();
  // pack (u,v) -> line b=0, (w,theta) -> b=1: Z_k = X1_k + i X2_k and its Hermitian mirror;
  // the DC imaginary parts are dropped as FFTW's c2r does.
  for (int w = threadIdx.x; w < 2 * ZB * nxh; w += blockDim.x) {
    const int k = w % nxh, t = w / nxh, l = t % ZB, b = t / ZB;
    if (z0 + l >= a.nz32) continue;
    const int64_t off = row0 + (int64_t)l * nxh + k;
    const int fa = (b == 0) ? 0 : 2, fb = (b == 0) ? 1 : 3;
    C x1 = mid[fa * a.nm + off], x2 = mid[fb * a.nm + off];
    const int L = b * ZB + l;
    if (k == 0) {
      buf[__ldg(pl.pos) * LS + L] = cmake<C>(x1.x, x2.x);
    } else {
      C zk, zm;
      zk.x = x1.x - x2.y; zk.y = x1.y + x2.x;
      zm.x = x1.x + x2.y; zm.y = x2.x - x1.y;
      buf[__ldg(pl.pos + k) * LS + L] = zk;
      buf[__ldg(pl.pos + (n - k)) * LS + L] = zm;
    }
  }
  __syncthreads();
  fft_dit<R>(buf, LS, 2 * ZB, pl, +1);
  // products (dft_x_realspace.f90:109-123) and the CFL maximum (:125-127)
  const double dyr = a.dyr[y];
  double vmax = 0.0;
  int bad = 0;
  for (int w = threadIdx.x; w < n * ZB; w += blockDim.x) {
    const int p = w / ZB, l = w % ZB;
    C uv = buf[p * LS + l], wt = buf[p * LS + ZB + l];
    const R u = uv.x, v = uv.y, ww = wt.x, t = wt.y;
    const R bv2 = v * v;
    C f12, f34, f57, f89;
    f12.x = u * u - bv2; f12.y = u * v;
    f34.x = ww * ww - bv2; f34.y = v * ww;
    f57.x = u * ww; f57.y = u * t;
    f89.x = v * t; f89.y = ww * t;
    buf[p * LS + l] = f12;
    buf[p * LS + ZB + l] = f34;
    buf[p * LS + 2 * ZB + l] = f57;
    buf[p * LS + 3 * ZB + l] = f89;
    if (a.substep == 1 && z0 + l < a.nz32) {
      double vel = (fabs((double)u) * a.dxr) + (fabs((double)v) * dyr) + (fabs((double)ww) * a.dzr);
      if (!isfinite(vel)) bad = 1;
      else vmax = fmax(vmax, vel);
    }
  }
  __syncthreads();
  fft_dif<R>(buf, LS, 4 * ZB, pl, -1);
  // unpack the pairs and keep kx < nxh
  for (int w = threadIdx.x; w < 4 * ZB * nxh; w += blockDim.x) {
    const int k = w % nxh, t = w / nxh, l = t % ZB, b = t / ZB;
    if (z0 + l >= a.nz32) continue;
    const int L = b * ZB + l;
    C zk = buf[__ldg(pl.pos + k) * LS + L];
    C zm = buf[__ldg(pl.pos + ((n - k) % n)) * LS + L];
    C A, B;
    A.x = (R)0.5 * (zk.x + zm.x); A.y = (R)0.5 * (zk.y - zm.y);
    B.x = (R)0.5 * (zk.y + zm.y); B.y = (R)0.5 * (zm.x - zk.x);
    const int64_t off = row0 + (int64_t)l * nxh + k;
    mid[(2 * b) * a.nm + off] = A;
    mid[(2 * b + 1) * a.nm + off] = B;
  }
  if (a.substep == 1) {
    // block max of the CFL velocity
    __shared__ double red[kThreads / 32];
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
      atomicMax(&a.dsc->velmax_bits, (unsigned long long)__double_as_longlong(m));
      if (redbad) atomicOr(&a.dsc->nonfinite, 1);
    }
  }
}

// ---------------------------------------------------------------------------------------
__global__ void k_begin_substep(DevScalars *dsc, int substep) {
  if (substep == 1) {
    dsc->velmax_bits = 0ull;
    dsc->nonfinite = 0;
  }
}

// dt update after the x step of substep 1 (dft_x_realspace.f90:489-498).
__global__ void k_update_dt(DevScalars *dsc, double dt_factor, double cflx, int fixed_dt) {
  const double velmax = __longlong_as_double((long long)dsc->velmax_bits);
  double dt = dsc->dt;
  dsc->dt_prev = dt;
  if (dsc->nonfinite) {
    dsc->err = KMM_ERR_NONFINITE;
    return;
  }
  if (!fixed_dt) dt = dt_factor * dt + (1.0 - dt_factor) * cflx / velmax;
  if (!(dt > 1e-14) || dt > 1e5) {
    dsc->err = KMM_ERR_DT;
    return;
  }
  dsc->dt = dt;
}

// ---------------------------------------------------------------------------------------
// Reference layout [f][mode][y] <-> planes [f][y][mode] (a batched 2-D transpose).
__global__ void k_transpose(const double2 *__restrict__ src, double2 *__restrict__ dst,
                            int64_t rows, int64_t cols) {
  // src (rows x cols) row-major per field -> dst (cols x rows)
  __shared__ double2 tile[32][33];
  const int64_t f = blockIdx.z;
  const int64_t c0 = (int64_t)blockIdx.x * 32, r0 = (int64_t)blockIdx.y * 32;
  const double2 *s = src + f * rows * cols;
  double2 *d = dst + f * rows * cols;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int64_t r = r0 + i, c = c0 + threadIdx.x;
    if (r < rows && c < cols) tile[i][threadIdx.x] = s[r * cols + c];
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    int64_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < rows && c < cols) d[c * rows + r] = tile[threadIdx.x][i];
  }
}

__global__ void k_d2f(const double2 *__restrict__ src, float2 *__restrict__ dst, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = make_float2((float)src[i].x, (float)src[i].y);
}

// Opt-in dynamic shared memory = the device limit minus the kernel's static shared memory.
template <typename K> void set_smem_limit(K kern, int bytes) {
  cudaFuncAttributes fa;
  if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) return;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes - (int)fa.sharedSizeBytes);
}

}  // namespace

// ---------------------------------------------------------------------------------------
cudaError_t launch_ref_to_planes(const double2 *src, double2 *dst, int nfield, int64_t nmodes,
                                 int ny, cudaStream_t st) {
  dim3 grid((unsigned)((ny + 31) / 32), (unsigned)((nmodes + 31) / 32), (unsigned)nfield);
  k_transpose<<<grid, dim3(32, 8), 0, st>>>(src, dst, nmodes, ny);
  return cudaGetLastError();
}

cudaError_t launch_planes_to_ref(const double2 *src, double2 *dst, int nfield, int64_t nmodes,
                                 int ny, cudaStream_t st) {
  dim3 grid((unsigned)((nmodes + 31) / 32), (unsigned)((ny + 31) / 32), (unsigned)nfield);
  k_transpose<<<grid, dim3(32, 8), 0, st>>>(src, dst, ny, nmodes);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t zinv_impl(Handle &h, const double2 *src, void *mid, int nfield, cudaStream_t st) {
  using C = typename Cpx<R>::T;
  constexpr int KB = sizeof(R) == 8 ? 8 : 16;
  const size_t smem = sizeof(C) * (size_t)h.pz.n * KB;
  auto kern = k_zinv<R, KB>;
  dim3 grid((unsigned)((h.nxh + KB - 1) / KB), (unsigned)h.ny, (unsigned)nfield);
  kern<<<grid, kThreads, smem, st>>>(src, reinterpret_cast<C *>(mid), h.pz, h.ny, h.nz, h.nxh,
                                     h.ns, h.nm);
  return cudaGetLastError();
}

cudaError_t launch_zinv(Handle &h, const double2 *src, void *mid, int nfield, cudaStream_t st, bool fp64) {
  const cudaError_t e = launch_zinv2(h, src, mid, nfield, st, fp64);
  if (e != cudaErrorNotSupported) return e;
  return (h.mixed && !fp64) ? zinv_impl<float>(h, src, mid, nfield, st)
                            : zinv_impl<double>(h, src, mid, nfield, st);
}

template <typename R, typename D>
static cudaError_t zfwd_impl(Handle &h, const void *mid, void *dst, int nfield, double scale,
                             cudaStream_t st) {
  using C = typename Cpx<R>::T;
  constexpr int KB = sizeof(R) == 8 ? 8 : 16;
  const size_t smem = sizeof(C) * (size_t)h.pz.n * KB;
  auto kern = k_zfwd<R, KB, D>;
  dim3 grid((unsigned)((h.nxh + KB - 1) / KB), (unsigned)h.ny, (unsigned)nfield);
  kern<<<grid, kThreads, smem, st>>>(reinterpret_cast<const C *>(mid), reinterpret_cast<D *>(dst),
                                     h.pz, h.ny, h.nz, h.nxh, h.ns, h.nm, scale);
  return cudaGetLastError();
}

cudaError_t launch_zfwd(Handle &h, const void *mid, void *dst, int nfield, double scale,
                        bool dst_fp64, cudaStream_t st, bool fp64) {
  const cudaError_t e = launch_zfwd2(h, mid, dst, nfield, scale, dst_fp64, st, fp64);
  if (e != cudaErrorNotSupported) return e;
  if (h.mixed && !fp64)
    return dst_fp64 ? zfwd_impl<float, double2>(h, mid, dst, nfield, scale, st)
                    : zfwd_impl<float, float2>(h, mid, dst, nfield, scale, st);
  return zfwd_impl<double, double2>(h, mid, dst, nfield, scale, st);
}

template <typename R, int ZB>
static cudaError_t xphys_zb(Handle &h, void *mid, int substep, cudaStream_t st) {
  using C = typename Cpx<R>::T;
  const size_t smem = sizeof(C) * (size_t)h.px.n * 4 * ZB;
  auto kern = k_xphys<R, ZB>;
  XArgs a;
  a.ny = h.ny;
  a.nz32 = h.nz32;
  a.nxh = h.nxh;
  a.nm = h.nm;
  a.dxr = h.dxr;
  a.dzr = h.dzr;
  a.dyr = h.dops + ops_offsets(h.bw, h.ny).dyr;
  a.substep = substep;
  a.dsc = h.dsc;
  dim3 grid((unsigned)((h.nz32 + ZB - 1) / ZB), (unsigned)h.ny);
  kern<<<grid, kThreads, smem, st>>>(reinterpret_cast<C *>(mid), h.px, a);
  return cudaGetLastError();
}

template <typename R>
static cudaError_t xphys_impl(Handle &h, void *mid, int substep, cudaStream_t st) {
  // largest line batch whose 4 buffers fit in 200 KB of shared memory
  const size_t per = sizeof(typename Cpx<R>::T) * (size_t)h.px.n * 4;
  const size_t lim = 200 * 1024;
  if (per * 8 <= lim) return xphys_zb<R, 8>(h, mid, substep, st);
  if (per * 4 <= lim) return xphys_zb<R, 4>(h, mid, substep, st);
  if (per * 2 <= lim) return xphys_zb<R, 2>(h, mid, substep, st);
  return xphys_zb<R, 1>(h, mid, substep, st);
}

cudaError_t launch_xphys(Handle &h, void *mid, int substep, cudaStream_t st) {
  const cudaError_t e = launch_xphys2(h, mid, substep, st);
  if (e != cudaErrorNotSupported || h.nsc != 1) return e;  // a second scalar needs a four-step length
  return h.mixed ? xphys_impl<float>(h, mid, substep, st) : xphys_impl<double>(h, mid, substep, st);
}

void convert_planes_d2f(const double2 *src, float2 *dst, int64_t n, cudaStream_t st) {
  k_d2f<<<1184, 256, 0, st>>>(src, dst, n);
}

void prepare_kernels(Handle &h) {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (optin <= 0) optin = 48 * 1024;
  (void)h;
  set_smem_limit(k_zinv<double, 8>, optin);
  set_smem_limit(k_zinv<float, 16>, optin);
  set_smem_limit(k_zfwd<double, 8, double2>, optin);
  set_smem_limit(k_zfwd<float, 16, float2>, optin);
  set_smem_limit(k_zfwd<float, 16, double2>, optin);
  set_smem_limit(k_xphys<double, 8>, optin);
  set_smem_limit(k_xphys<double, 4>, optin);
  set_smem_limit(k_xphys<double, 2>, optin);
  set_smem_limit(k_xphys<double, 1>, optin);
  set_smem_limit(k_xphys<float, 8>, optin);
  set_smem_limit(k_xphys<float, 4>, optin);
  set_smem_limit(k_xphys<float, 2>, optin);
  set_smem_limit(k_xphys<float, 1>, optin);
}

cudaError_t launch_begin_substep(Handle &h, int substep, cudaStream_t st) {
  k_begin_substep<<<1, 1, 0, st>>>(h.dsc, substep);
  return cudaGetLastError();
}

cudaError_t launch_update_dt(Handle &h, int substep, cudaStream_t st) {
  if (substep != 1) return cudaSuccess;
  k_update_dt<<<1, 1, 0, st>>>(h.dsc, h.cfg.dt_factor, h.cflx, h.cfg.fixed_dt);
  return cudaGetLastError();
}

}  // namespace kmm
