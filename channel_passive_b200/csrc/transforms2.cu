// transforms2.cu - the substep's transforms with compile-time four-step FFTs (fft2.cuh).
//
// Same contracts as transforms.cu (k_zinv / k_xphys / k_zfwd: y_to_x, dft_x_realspace and
// x_to_y with rescale_data folded in) for the line lengths N = N1 * N2 listed in with_shape;
// the launchers fall back to the generic kernels of transforms.cu for other lengths.  Lines
// are line-major in shared memory with the odd leading dimension (N1+1)*N2 | 1 and are
// transformed in place (fft4_ip), natural order in and out, so the 3/2 padding and truncation
// read and write plain positions k and N - k.
#include <cuda.h>
#include <cuda_runtime.h>

#include "fft2.cuh"
#include "kmm_internal.h"
#include "stats.cuh"

namespace kmm {

namespace {

template <typename C> __device__ __forceinline__ C ld_as(const double2 *p) {
  const double2 v = *p;
  return cmake<C>(v.x, v.y);
}
template <typename R> __device__ __forceinline__ const typename Cpx<R>::T *tw_of(const FftPlan &pl);
template <> __device__ __forceinline__ const double2 *tw_of<double>(const FftPlan &pl) { return pl.tw64; }
template <> __device__ __forceinline__ const float2 *tw_of<float>(const FftPlan &pl) { return pl.tw32; }

// Threads of a z-transform block: one per (line, step-1 or step-2 work item).
template <int N1, int N2, int KB>
constexpr int z_threads() {
  return KB * (N1 > N2 ? N1 : N2);
}

// The z position of padded index p (3/2 rule of ppdfftw_dft_z_inverse, module_ppdfftw.f90:846-854):
// kz index for p < nz/2 and p > nz, -1 for the zero band nz/2..nz.
__device__ __forceinline__ int zpad_src(int p, int nh) { return p < nh ? p : (p > 2 * nh ? p - nh : -1); }

// ---- TMA staging of the z-transform input tiles (cp.async.bulk.tensor, no multicast) -------
// A block's input tile (its KB kx columns of all rows of one (field, y) plane) is copied into
// shared memory as 3-D tensor boxes of (2 KB scalars, tile_rows(n) rows, 1 plane); the copies
// complete on an mbarrier whose wait has an iteration limit.
constexpr int kTmaWaitIters = 1 << 20;

// Rows of one TMA box over n rows: n split into ceil(n / 256) equal boxes (0 if they are not equal).
__host__ __device__ constexpr int tile_rows(int n) {
  const int nb = (n + 255) / 256;
  return n % nb == 0 ? n / nb : 0;
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// bounded wait for phase 0 of `bar`; false if it gave up
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar) {
  for (int it = 0; it < kTmaWaitIters; ++it)
    if (mbar_try_wait(bar, 0)) return true;
  return false;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// Copies a block's tile (KB columns x n rows of element E) into `base`, in tile_rows(n)-row boxes,
// and waits for it.  Thread 0 arms the barrier and issues the copies; every thread waits (the
// completed phase makes the bytes visible to it).  Returns false, for the whole block, if the
// wait gave up: the error flag is set and the block should leave.
template <typename E, int KB>
__device__ __forceinline__ bool tma_tile(unsigned char *base, const CUtensorMap *map, int n, int x, int plane,
                                         uint64_t *bar, int *err) {
  if (threadIdx.x == 0) mbar_init(bar, 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    const int rows = tile_rows(n);
    mbar_expect_tx(bar, (unsigned)(KB * n * sizeof(E)));
    for (int r0 = 0; r0 < n; r0 += rows) tma_load_3d(base + (size_t)r0 * KB * sizeof(E), map, x, r0, plane, bar);
  }
  const bool ok = mbar_wait_bounded(bar);
  if (__syncthreads_or(!ok)) {
    // the copy did not complete: flag it and give it one more bounded wait before the block leaves
    if (threadIdx.x == 0) atomicCAS(err, 0, KMM_ERR_TIMEOUT);
    mbar_wait_bounded(bar);
    return false;
  }
  return true;
}

// Dynamic shared memory of a z kernel with TMA: the larger of the tile and the FFT lines (the lines
// overlay the tile once every thread has taken its inputs), plus 128 bytes so that the tile can
// start on a 128-byte shared address.
template <typename R, int N1, int N2, int KB, typename E>
constexpr size_t z_smem_tma(int n) {
  const size_t tile = (size_t)KB * n * sizeof(E);
  const size_t lines = (size_t)KB * ip_lda<N1, N2>() * sizeof(typename Cpx<R>::T);
  return (tile > lines ? tile : lines) + 128;
}

// y_to_x: grid (ceil(nxh/KB), ny, nfield).  Thread (l, n1) of step 1 reads its N2 points
// x[n1 + N1*n2] of kx line l straight from the Y-pencil (16 consecutive kx per row: one coalesced
// run) or, with TMA, from the block's tile in shared memory, transforms them in registers and
// leaves them in shared memory; thread (l, k2) of step 2 finishes the line and writes
// X[k2 + N2*k1] straight into the X-pencil slab.
template <typename R, int N1, int N2, int KB, bool TMA = false>
__global__ void __launch_bounds__(z_threads<N1, N2, KB>()) k_zinv2(const double2 *__restrict__ src,
                                                                  typename Cpx<R>::T *__restrict__ dst,
                                                                  FftPlan pl, int nz, int nxh, int64_t ns,
                                                                  int64_t nm, const __grid_constant__ CUtensorMap tmap,
                                                                  int ny, int *err) {
  using C = typename Cpx<R>::T;
  constexpr int N = N1 * N2, LD = ip_lda<N1, N2>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // with TMA the tile (and the lines over it) starts on the next 128-byte shared address
  unsigned char *base = TMA ? smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u) : smem_raw;
  C *a = reinterpret_cast<C *>(base);
  const int nh = nz / 2;
  const int kx0 = blockIdx.x * KB, y = blockIdx.y, f = blockIdx.z;
  const int l = threadIdx.x % KB, item = threadIdx.x / KB;
  const bool live = kx0 + l < nxh;
  const C *tw = tw_of<R>(pl);
  C v[N2];
  if constexpr (TMA) {
    __shared__ __align__(8) uint64_t bar;
    if (!tma_tile<double2, KB>(base, &tmap, nz, 2 * kx0, f * ny + y, &bar, err)) return;
    const double2 *tile = reinterpret_cast<const double2 *>(base);
    if (item < N1) {
      const int n1 = item;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) {
        const int kzi = zpad_src(n1 + N1 * n2, nh);
        v[n2] = (live && kzi >= 0) ? ld_as<C>(tile + kzi * KB + l) : cmake<C>(0.0, 0.0);
      }
    }
    __syncthreads();  // the FFT lines overlay the tile
  } else {
    if (item < N1) {
      const int n1 = item;
      const double2 *sp = src + f * ns + (int64_t)y * nz * nxh + kx0 + l;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) {
        const int kzi = zpad_src(n1 + N1 * n2, nh);
        v[n2] = (live && kzi >= 0) ? ld_as<C>(sp + (int64_t)kzi * nxh) : cmake<C>(0.0, 0.0);
      }
    }
  }
  if (item < N1) {
    const int n1 = item;
    reg_dft<C, N2>(v, +1);
    C *yl = a + l * LD;
    yl[n1] = v[0];
#pragma unroll
    for (int k2 = 1; k2 < N2; ++k2) {
      C w = tw[n1 * k2];
      w.y = -w.y;
      yl[n1 + (N1 + 1) * k2] = n1 > 0 ? cmul(v[k2], w) : v[k2];
    }
  }
  __syncthreads();
  if (item < N2 && live) {
    const int k2 = item;
    const C *yl = a + l * LD;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = yl[n1 + (N1 + 1) * k2];
    reg_dft<C, N1>(v, +1);
    C *dp = dst + f * nm + (int64_t)y * N * nxh + kx0 + l;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) dp[(int64_t)(k2 + N2 * k1) * nxh] = v[k1];
  }
}

// x_to_y: grid (ceil(nxh/KB), ny, nfield).  The mirror of k_zinv2: step 1 reads the X-pencil
// slab, step 2 writes the kept frequencies (truncation of ppdfftw_dft_z_forward,
// module_ppdfftw.f90:811-817) with the kz Nyquist row zeroed and the rescale folded in.
// With TMA, step 1 takes its points from the block's tile of the slab (KB kx columns of the N
// rows of one (field, y) plane), which the FFT lines then overlay.
template <typename R, int N1, int N2, int KB, typename D, bool TMA = false>
__global__ void __launch_bounds__(z_threads<N1, N2, KB>()) k_zfwd2(const typename Cpx<R>::T *__restrict__ src,
                                                                  D *__restrict__ dst, FftPlan pl, int nz, int nxh,
                                                                  int64_t ns, int64_t nm, double scale,
                                                                  const __grid_constant__ CUtensorMap tmap, int ny,
                                                                  int *err) {
  using C = typename Cpx<R>::T;
  constexpr int N = N1 * N2, LD = ip_lda<N1, N2>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char *base = TMA ? smem_raw + ((128u - (smem_u32(smem_raw) & 127u)) & 127u) : smem_raw;
  C *a = reinterpret_cast<C *>(base);
  const int nh = nz / 2;
  const int kx0 = blockIdx.x * KB, y = blockIdx.y, f = blockIdx.z;
  const int l = threadIdx.x % KB, item = threadIdx.x / KB;
  const bool live = kx0 + l < nxh;
  const C *tw = tw_of<R>(pl);
  C v[N2];
  if constexpr (TMA) {
    __shared__ __align__(8) uint64_t bar;
    if (!tma_tile<C, KB>(base, &tmap, N, 2 * kx0, f * ny + y, &bar, err)) return;
    const C *tile = reinterpret_cast<const C *>(base);
    if (item < N1) {
      const int n1 = item;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) v[n2] = live ? tile[(n1 + N1 * n2) * KB + l] : cmake<C>(0.0, 0.0);
    }
    __syncthreads();  // the FFT lines overlay the tile
  } else {
    if (item < N1) {
      const int n1 = item;
      const C *sp = src + f * nm + (int64_t)y * N * nxh + kx0 + l;
#pragma unroll
      for (int n2 = 0; n2 < N2; ++n2) v[n2] = live ? sp[(int64_t)(n1 + N1 * n2) * nxh] : cmake<C>(0.0, 0.0);
    }
  }
  if (item < N1) {
    const int n1 = item;
    reg_dft<C, N2>(v, -1);
    C *yl = a + l * LD;
    yl[n1] = v[0];
#pragma unroll
    for (int k2 = 1; k2 < N2; ++k2) yl[n1 + (N1 + 1) * k2] = n1 > 0 ? cmul(v[k2], tw[n1 * k2]) : v[k2];
  }
  __syncthreads();
  if (item < N2 && live) {
    const int k2 = item;
    const C *yl = a + l * LD;
    C v[N1];
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) v[n1] = yl[n1 + (N1 + 1) * k2];
    reg_dft<C, N1>(v, -1);
    D *dp = dst + f * ns + (int64_t)y * nz * nxh + kx0 + l;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) {
      const int k = k2 + N2 * k1;
      int kzi = -1;
      D out;
      if (k < nh || k > 2 * nh) {
        kzi = k < nh ? k : k - nh;
        out.x = (decltype(out.x))(scale * (double)v[k1].x);
        out.y = (decltype(out.y))(scale * (double)v[k1].y);
      } else if (k == nh) {  // the kz Nyquist row is zeroed (module_ppdfftw.f90:811-817)
        kzi = nh;
        out.x = 0;
        out.y = 0;
      }
      if (kzi >= 0) dp[(int64_t)kzi * nxh] = out;
    }
  }
}

struct X2Args {
  int ny, nz32, nxh;
  float rnxh;  // 1 / nxh: the loops below split w into (w / nxh, w % nxh) without an integer divide
  int64_t nm;
  double dxr, dzr;
  const double *dyr;
  int substep;
  DevScalars *dsc;
  double *mom;  // STAT only, may be null: per-block moment sums [ny][gridDim.x][kNumMoments]
};

// dft_x_realspace: grid (ceil(nz32/ZB), ny), NT threads; MID slots 0..3 = u, v, w, theta in,
// slots 0..7 = f1, f2, f3, f4, f5, f7, f8, f9 out (a block owns its rows).
// STAT: the statistics-step products for the pressure instead (f1..f6 with f6 = v v,
// dft_x_realspace.f90:192-199): packed lines (f1, f2), (f3, f4), (f5, f6); no CFL, and only
// slots 0..5 are written.  With a_.mom set, each block also writes the sums over its physical
// points of the moments of dft_x_realspace.f90:128-155 (moment_terms), in FP64.
#ifndef KMM_X576_MINB
#define KMM_X576_MINB 5
#endif
// Resident blocks asked of the compiler: at N = 576 the FP32 step pass otherwise takes 140
// registers a thread, 3 blocks (12 warps) an SM.  5 blocks (96 registers, a 200-byte spill) took
// the pass from 2.35 to 2.01 ms on the 384x257x384 grid (4 blocks, no spill: 2.04 ms).  The
// statistics variant keeps the default: a cap spills more there.
// At N = 288 (16 x 18) the FP32 step pass took 80 registers, 6 blocks an SM; 8 blocks (64
// registers, a 56-byte spill) took it from 0.2345 to 0.2155 ms on the 192x129x192 grid
// (7 blocks: 0.2167 ms).
#ifndef KMM_X288_MINB
#define KMM_X288_MINB 8
#endif
// The FP64 step pass at N = 288 took 152 registers with 64 threads, 6 blocks (12 warps) an SM;
// 8 blocks (128 registers, a 64-byte spill) took it from 0.3887 to 0.3712 ms.
#ifndef KMM_X288_MINB_FP64
#define KMM_X288_MINB_FP64 8
#endif
template <typename R, int N, bool STAT, int NS = 1, int V = 0> constexpr int x_min_blocks() {
  if (STAT || V != 0) return 1;  // the caps below were measured for the default shape
  // two scalars, FP32 at N = 576: 210 registers uncapped (2 blocks an SM); 3 blocks fit the
  // shared memory of the six packed lines per row
  if (NS != 1) return (sizeof(R) == 4 && N >= 576) ? 3 : 1;
  if (sizeof(R) != 4) return N == 288 ? KMM_X288_MINB_FP64 : 1;
  return N >= 576 ? KMM_X576_MINB : N == 288 ? KMM_X288_MINB : 1;
}

// NS = 2: a second passive scalar theta2 in MID slot 4; its products u theta2, v theta2, w theta2
// go to slots 8, 9, 10, formed like f7..f9 (a third packed input line (theta2, 0) and two packed
// output lines (u theta2, v theta2), (w theta2, 0)).
template <typename R, int N1, int N2, int ZB, int NT, bool STAT = false, int NS = 1, int V = 0>
__global__ void __launch_bounds__(NT, (x_min_blocks<R, N1 * N2, STAT, NS, V>())) k_xphys2(typename Cpx<R>::T *__restrict__ mid, FftPlan pl, X2Args a_) {
  using C = typename Cpx<R>::T;
  constexpr int N = N1 * N2, LD = ip_lda<N1, N2>();
  constexpr int NIN = 1 + NS, NOUT = 2 + 2 * NS;  // packed input and output lines per row
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *a = reinterpret_cast<C *>(smem_raw);  // NOUT*ZB lines: (u,v) ZB, (w,theta) ZB, [(theta2,0) ZB,] then outputs
  const int nxh = a_.nxh;
  const int z0 = blockIdx.x * ZB, y = blockIdx.y;
  const int64_t row0 = ((int64_t)y * a_.nz32 + z0) * nxh;
  for (int w = threadIdx.x; w < NIN * ZB * N; w += NT) {
    const int L = w / N, p = w - L * N;
    a[L * LD + p] = cmake<C>(0.0, 0.0);
  }
  __syncthreads();
  // Z_k = X1_k + i X2_k and its Hermitian mirror at N - k; DC imaginary parts dropped (c2r)
  for (int w = threadIdx.x; w < NIN * ZB * nxh; w += NT) {
    // exact: (w + 0.5) / nxh stays at least 0.5 / nxh away from an integer, far above float rounding
    const int t = (int)(((float)w + 0.5f) * a_.rnxh), k = w - t * nxh, l = t % ZB, bsel = t / ZB;
    if (z0 + l >= a_.nz32) continue;
    const int64_t off = row0 + (int64_t)l * nxh + k;
    const int fa = bsel == 0 ? 0 : bsel == 1 ? 2 : 4, fb = bsel == 0 ? 1 : 3;
    const C x1 = mid[fa * a_.nm + off];
    const C x2 = bsel < 2 ? mid[fb * a_.nm + off] : cmake<C>(0.0, 0.0);
    C *line = a + (bsel * ZB + l) * LD;
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
  fft4_ip<R, N1, N2, NIN * ZB, NT>(a, LD, tw_of<R>(pl), +1);
  const double dyr = a_.dyr[y];
  double vmax = 0.0;
  int bad = 0;
  double ms[STAT ? kNumMoments : 1] = {};
  for (int w = threadIdx.x; w < ZB * N; w += NT) {
    const int l = w / N, p = w - l * N;
    const C uv = a[l * LD + p], wt = a[(ZB + l) * LD + p];
    const R u = uv.x, v = uv.y, ww = wt.x, t = wt.y;
    R t2 = 0;
    if constexpr (NS == 2) t2 = a[(2 * ZB + l) * LD + p].x;
    if constexpr (STAT) {
      if (a_.mom && z0 + l < a_.nz32) moment_terms(ms, (double)u, (double)v, (double)ww);
    }
    const R bv2 = v * v;
    C f12, f34, f57, f89;
    f12.x = u * u - bv2; f12.y = u * v;
    f34.x = ww * ww - bv2; f34.y = v * ww;
    if constexpr (STAT) {
      f57.x = u * ww; f57.y = bv2;
      f89.x = 0; f89.y = 0;
    } else {
      f57.x = u * ww; f57.y = u * t;
      f89.x = v * t; f89.y = ww * t;
    }
    a[l * LD + p] = f12;
    a[(ZB + l) * LD + p] = f34;
    a[(2 * ZB + l) * LD + p] = f57;
    a[(3 * ZB + l) * LD + p] = f89;
    if constexpr (NS == 2) {
      C g12, g3;
      g12.x = u * t2; g12.y = v * t2;
      g3.x = ww * t2; g3.y = 0;
      a[(4 * ZB + l) * LD + p] = g12;
      a[(5 * ZB + l) * LD + p] = g3;
    }
    if (!STAT && a_.substep == 1 && z0 + l < a_.nz32) {
      const double vel = (fabs((double)u) * a_.dxr) + (fabs((double)v) * dyr) + (fabs((double)ww) * a_.dzr);
      if (!isfinite(vel)) bad = 1;
      else vmax = fmax(vmax, vel);
    }
  }
  __syncthreads();
  fft4_ip<R, N1, N2, NOUT * ZB, NT>(a, LD, tw_of<R>(pl), -1);
  for (int w = threadIdx.x; w < (STAT ? 3 : NOUT) * ZB * nxh; w += NT) {
    // exact: (w + 0.5) / nxh stays at least 0.5 / nxh away from an integer, far above float rounding
    const int t = (int)(((float)w + 0.5f) * a_.rnxh), k = w - t * nxh, l = t % ZB, bsel = t / ZB;
    if (z0 + l >= a_.nz32) continue;
    const C *line = a + (bsel * ZB + l) * LD;
    const C zk = line[k], zm = line[k == 0 ? 0 : N - k];
    C A, B;
    A.x = (R)0.5 * (zk.x + zm.x); A.y = (R)0.5 * (zk.y - zm.y);
    B.x = (R)0.5 * (zk.y + zm.y); B.y = (R)0.5 * (zm.x - zk.x);
    const int64_t off = row0 + (int64_t)l * nxh + k;
    mid[(2 * bsel) * a_.nm + off] = A;
    if (2 * bsel + 1 < 11) mid[(2 * bsel + 1) * a_.nm + off] = B;  // slot 11 would be the zero partner
  }
  if constexpr (STAT) {
    if (a_.mom) {
      // fixed-order block sum: lanes by shuffles, then warps in order
      __shared__ double mred[NT / 32][kNumMoments];
#pragma unroll
      for (int i = 0; i < kNumMoments; ++i) {
        double x = ms[i];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0) mred[threadIdx.x >> 5][i] = x;
      }
      __syncthreads();
      if (threadIdx.x < kNumMoments) {
        double x = 0.0;
        for (int j = 0; j < NT / 32; ++j) x += mred[j][threadIdx.x];
        a_.mom[((int64_t)y * gridDim.x + blockIdx.x) * kNumMoments + threadIdx.x] = x;
      }
    }
  }
  if (!STAT && a_.substep == 1) {
    __shared__ double red[NT / 32];
    __shared__ int redbad;
    if (threadIdx.x == 0) redbad = 0;
    __syncthreads();
    if (bad) atomicOr(&redbad, 1);
    for (int o = 16; o > 0; o >>= 1) vmax = fmax(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = vmax;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
      for (int i = 0; i < NT / 32; ++i) m = fmax(m, red[i]);
      atomicMax(&a_.dsc->velmax_bits, (unsigned long long)__double_as_longlong(m));
      if (redbad) atomicOr(&a_.dsc->nonfinite, 1);
    }
  }
}

// Transpose of the x pass at a base state (the discrete adjoint; FP64), one block per x-line
// row (z, y).  With <a, b> = Re sum conj(a) b over the kept kx coefficients and the plain sum
// over physical points, the pass's three parts transpose as
//   r2c + truncate  ->  lambda_phys(x) = Re sum_{k < nxh} lambda_k e^{+ikx}: a c2r of
//                       b_0 = lambda_0, b_k = lambda_k / 2 (the same packed c2r as the forward);
//   products        ->  their linearisation at the base u, v, w, theta (a c2r of base_mid);
//   pad + c2r       ->  an r2c with weight 1 at kx = 0 (its imaginary part dropped) and 2 above.
// base_mid slots 0..3 = u, v, w, theta of the base state (x-spectral, z-physical); lmid slots
// 0..7 = lambda of f1..f5, f7..f9 on entry, multiplied by `scale` (the rescale of x_to_y), and
// lambda of u, v, w, theta in slots 0..3 on exit.
template <int N1, int N2>
__global__ void __launch_bounds__(128) k_xadj2(const double2 *__restrict__ base_mid, double2 *__restrict__ lmid,
                                              FftPlan pl, int nz32, int nxh, float rnxh, int64_t nm, double scale) {
  using C = double2;
  constexpr int N = N1 * N2, LD = ip_lda<N1, N2>(), NT = 128;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C *a = reinterpret_cast<C *>(smem_raw);  // 6 lines: base (u,v) (w,t); lambda (f1,f2) (f3,f4) (f5,f7) (f8,f9)
  const int z = blockIdx.x, y = blockIdx.y;
  const int64_t row0 = ((int64_t)y * nz32 + z) * nxh;
  for (int w = threadIdx.x; w < 6 * N; w += NT) a[(w / N) * LD + (w % N)] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int w = threadIdx.x; w < 6 * nxh; w += NT) {
    const int t = (int)(((float)w + 0.5f) * rnxh), k = w - t * nxh;  // line t = 0..5, exact split
    C x1, x2;
    if (t < 2) {
      x1 = base_mid[(2 * t) * nm + row0 + k];
      x2 = base_mid[(2 * t + 1) * nm + row0 + k];
    } else {
      const double f = (k == 0 ? 1.0 : 0.5) * scale;
      const C l1 = lmid[(2 * (t - 2)) * nm + row0 + k], l2 = lmid[(2 * (t - 2) + 1) * nm + row0 + k];
      x1 = make_double2(f * l1.x, f * l1.y);
      x2 = make_double2(f * l2.x, f * l2.y);
    }
    C *line = a + t * LD;
    if (k == 0) {
      line[0] = make_double2(x1.x, x2.x);
    } else {
      line[k] = make_double2(x1.x - x2.y, x1.y + x2.x);
      line[N - k] = make_double2(x1.x + x2.y, x2.x - x1.y);
    }
  }
  __syncthreads();
  fft4_ip<double, N1, N2, 6, NT>(a, LD, tw_of<double>(pl), +1);
  for (int p = threadIdx.x; p < N; p += NT) {
    const C uv = a[p], wt = a[LD + p];
    const double u = uv.x, v = uv.y, w = wt.x, t = wt.y;
    const C l12 = a[2 * LD + p], l34 = a[3 * LD + p], l57 = a[4 * LD + p], l89 = a[5 * LD + p];
    // f1 = uu - vv, f2 = uv, f3 = ww - vv, f4 = vw, f5 = uw, f7 = u t, f8 = v t, f9 = w t
    const double lu = 2.0 * u * l12.x + v * l12.y + w * l57.x + t * l57.y;
    const double lv = -2.0 * v * l12.x + u * l12.y - 2.0 * v * l34.x + w * l34.y + t * l89.x;
    const double lw = 2.0 * w * l34.x + v * l34.y + u * l57.x + t * l89.y;
    const double lt = u * l57.y + v * l89.x + w * l89.y;
    a[2 * LD + p] = make_double2(lu, lv);
    a[3 * LD + p] = make_double2(lw, lt);
  }
  __syncthreads();
  fft4_ip<double, N1, N2, 2, NT>(a + 2 * LD, LD, tw_of<double>(pl), -1);
  for (int w = threadIdx.x; w < 2 * nxh; w += NT) {
    const int t = (int)(((float)w + 0.5f) * rnxh), k = w - t * nxh;
    const C *line = a + (2 + t) * LD;
    const C zk = line[k], zm = line[k == 0 ? 0 : N - k];
    C A = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
    C B = make_double2(0.5 * (zk.y + zm.y), 0.5 * (zm.x - zk.x));
    if (k == 0) {
      A.y = 0.0;
      B.y = 0.0;
    } else {
      A = make_double2(2.0 * A.x, 2.0 * A.y);
      B = make_double2(2.0 * B.x, 2.0 * B.y);
    }
    lmid[(2 * t) * nm + row0 + k] = A;
    lmid[(2 * t + 1) * nm + row0 + k] = B;
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

// Lines per block (KB: z transforms, one thread per line and work item) and rows per block and
// threads (ZB, ZT: x pass), tuned at N = 288 on B200: a line needs (N1+1)*N2 | 1 complex values
// of shared memory, so these choices keep 39 KB or less per block.
template <typename R> struct TCfg;
template <> struct TCfg<float> {
  static constexpr int KB = 16, ZB = 2, ZT = 128;
};
template <> struct TCfg<double> {
  static constexpr int KB = 8, ZB = 1, ZT = 64;
};

// Tile-shape variants the autotuner (kmm_autotune) times on the handle's grid; variant 0 is the
// hand-tuned TCfg.  The others are built for lengths of kMinTunedLength points and more only
// (shorter lines fall back to variant 0 at compile time).
constexpr int kMinTunedLength = 96;
template <typename R, int V> struct ZVar;  // z transforms: lines per block
template <> struct ZVar<float, 0> { static constexpr int KB = TCfg<float>::KB; };
template <> struct ZVar<float, 1> { static constexpr int KB = 8; };
template <> struct ZVar<float, 2> { static constexpr int KB = 32; };
template <> struct ZVar<double, 0> { static constexpr int KB = TCfg<double>::KB; };
template <> struct ZVar<double, 1> { static constexpr int KB = 4; };
template <> struct ZVar<double, 2> { static constexpr int KB = 16; };
template <typename R, int V> struct XVar;  // x pass: rows per block and threads
template <> struct XVar<float, 0> { static constexpr int ZB = TCfg<float>::ZB, ZT = TCfg<float>::ZT; };
template <> struct XVar<float, 1> { static constexpr int ZB = 1, ZT = 128; };
template <> struct XVar<float, 2> { static constexpr int ZB = 4, ZT = 256; };
template <> struct XVar<double, 0> { static constexpr int ZB = TCfg<double>::ZB, ZT = TCfg<double>::ZT; };
template <> struct XVar<double, 1> { static constexpr int ZB = 1, ZT = 128; };
template <> struct XVar<double, 2> { static constexpr int ZB = 2, ZT = 128; };
template <int N, int V> constexpr int tuned_variant() { return N < kMinTunedLength ? 0 : V; }

// Runs f.template operator()<V>() for the runtime variant v (0..2).
template <typename F> void with_variant(int v, F &&f) {
  switch (v) {
    case 1: f.template operator()<1>(); break;
    case 2: f.template operator()<2>(); break;
    default: f.template operator()<0>(); break;
  }
}

template <typename R, int N1, int N2, int KB = TCfg<R>::KB>
constexpr size_t z_smem() {
  return sizeof(typename Cpx<R>::T) * (size_t)KB * ip_lda<N1, N2>();
}
template <typename R, int N1, int N2, int NS = 1, int ZB = TCfg<R>::ZB>
constexpr size_t x_smem() {
  return sizeof(typename Cpx<R>::T) * (size_t)(2 + 2 * NS) * ZB * ip_lda<N1, N2>();
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
  cudaError_t e = cudaMemcpyToSymbol(c_regtw, h, sizeof(h));
  if (e != cudaSuccess) return e;
  float2 h32[kRegTwTotal];
  for (int i = 0; i < kRegTwTotal; ++i) h32[i] = make_float2((float)h[i].x, (float)h[i].y);
  return cudaMemcpyToSymbol(c_regtw32, h32, sizeof(h32));
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
      using D = TCfg<double>;
      set_smem(k_xphys2<double, N1, N2, D::ZB, D::ZT, true>, optin);
      set_smem(k_xadj2<N1, N2>, optin);
      for (int v = 0; v < 3; ++v)
        with_variant(v, [&]<int V>() {
          constexpr int VV = tuned_variant<N1 * N2, V>();
          using ZF = ZVar<float, VV>;
          using ZD = ZVar<double, VV>;
          using XF = XVar<float, VV>;
          using XD = XVar<double, VV>;
          set_smem(k_zinv2<double, N1, N2, ZD::KB>, optin);
          set_smem(k_zinv2<float, N1, N2, ZF::KB>, optin);
          set_smem(k_zfwd2<double, N1, N2, ZD::KB, double2>, optin);
          set_smem(k_zfwd2<float, N1, N2, ZF::KB, float2>, optin);
          set_smem(k_zfwd2<float, N1, N2, ZF::KB, double2>, optin);
          set_smem(k_zinv2<double, N1, N2, ZD::KB, true>, optin);
          set_smem(k_zinv2<float, N1, N2, ZF::KB, true>, optin);
          set_smem(k_zfwd2<double, N1, N2, ZD::KB, double2, true>, optin);
          set_smem(k_zfwd2<float, N1, N2, ZF::KB, float2, true>, optin);
          set_smem(k_zfwd2<float, N1, N2, ZF::KB, double2, true>, optin);
          set_smem(k_xphys2<double, N1, N2, XD::ZB, XD::ZT, false, 1, VV>, optin);
          set_smem(k_xphys2<float, N1, N2, XF::ZB, XF::ZT, false, 1, VV>, optin);
          set_smem(k_xphys2<double, N1, N2, XD::ZB, XD::ZT, false, 2, VV>, optin);
          set_smem(k_xphys2<float, N1, N2, XF::ZB, XF::ZT, false, 2, VV>, optin);
        });
    });
  }
  return cudaSuccess;
}

// The driver's tensor-map encoder (cuTensorMapEncodeTiled), fetched once through the runtime.
using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled() {
  static const EncodeTiledFn fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return reinterpret_cast<EncodeTiledFn>(p);
  }();
  return fn;
}

int opt_in_smem() {
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return 0;
  return optin;
}

// The tile map of a z kernel's input: `base` holds nfield planes per y of n rows x nxh complex
// elements of es-byte scalars (a (2 nxh, n, nfield ny) tensor of scalars); a box is KB complex
// columns by tile_rows(n) rows of one plane.  The rules of a tiled map, checked here: base and
// strides (2 nxh es, 2 nxh es n) multiples of 16 bytes, box extents <= 256, inner box 2 KB es
// bytes a multiple of 16, every copy's x coordinate 2 kx0 scalars (kx0 a multiple of KB) a
// multiple of 16 bytes, and every box's shared destination (r0 KB 2 es bytes past a 128-byte
// aligned tile) on a 128-byte boundary.  False where the grid or the encoder does not allow it;
// the caller then loads per thread.
bool z_tile_map(const void *base, int nxh, int n, int nfield, int ny, int KB, size_t es, CUtensorMap *m) {
  const EncodeTiledFn fn = encode_tiled();
  const int rows = tile_rows(n);
  if (!fn || 2 * KB > 256 || rows == 0 || (2 * KB * es) % 16 != 0 || (2 * (size_t)nxh * es) % 16 != 0 ||
      ((size_t)rows * KB * 2 * es) % 128 != 0 || (reinterpret_cast<uintptr_t>(base) & 15u) != 0)
    return false;
  const cuuint64_t dims[3] = {2ull * (cuuint64_t)nxh, (cuuint64_t)n, (cuuint64_t)nfield * (cuuint64_t)ny};
  const cuuint64_t strides[2] = {2ull * es * (cuuint64_t)nxh, 2ull * es * (cuuint64_t)nxh * (cuuint64_t)n};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * KB), (cuuint32_t)rows, 1u}, ones[3] = {1u, 1u, 1u};
  return fn(m, es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
            const_cast<void *>(base), dims, strides, box, ones, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// y_to_x through TMA: only from the state S (the map covers its 3 + nsc fields)
template <typename R, int N1, int N2, int KB>
bool zinv_tma_map(const Handle &h, const double2 *src, int nfield, CUtensorMap *m) {
  return h.tune.ztma && src == h.S && nfield <= 3 + h.nsc &&
         z_smem_tma<R, N1, N2, KB, double2>(h.nz) <= (size_t)opt_in_smem() &&
         z_tile_map(h.S, h.nxh, h.nz, 3 + h.nsc, h.ny, KB, sizeof(double), m);
}

// x_to_y through TMA: only from the slab MID (the map covers its 5 + 3 nsc fields)
template <typename R, int N1, int N2, int KB>
bool zfwd_tma_map(const Handle &h, const void *mid, int nfield, CUtensorMap *m) {
  const int nprod = 5 + 3 * h.nsc;
  return h.tune.ztma && mid == h.MID && nfield <= nprod &&
         z_smem_tma<R, N1, N2, KB, typename Cpx<R>::T>(N1 * N2) <= (size_t)opt_in_smem() &&
         z_tile_map(h.MID, h.nxh, N1 * N2, nprod, h.ny, KB, sizeof(R), m);
}

// Returns cudaErrorNotSupported when the length has no four-step shape (caller falls back).
cudaError_t launch_zinv2(Handle &h, const double2 *src, void *mid, int nfield, cudaStream_t st, bool fp64) {
  cudaError_t err = cudaErrorNotSupported;
  auto go = [&]<typename R>() {
    with_shape(h.nz32, [&]<int N1, int N2>() {
      with_variant(h.tune.z, [&]<int V>() {
        using C = typename Cpx<R>::T;
        constexpr int KB = ZVar<R, tuned_variant<N1 * N2, V>()>::KB;
        dim3 grid((unsigned)((h.nxh + KB - 1) / KB), (unsigned)h.ny, (unsigned)nfield);
        CUtensorMap tmap{};
        if (zinv_tma_map<R, N1, N2, KB>(h, src, nfield, &tmap))
          k_zinv2<R, N1, N2, KB, true><<<grid, z_threads<N1, N2, KB>(), z_smem_tma<R, N1, N2, KB, double2>(h.nz),
                                         st>>>(src, reinterpret_cast<C *>(mid), h.pz, h.nz, h.nxh, h.ns, h.nm, tmap,
                                               h.ny, &h.dsc->err);
        else
          k_zinv2<R, N1, N2, KB, false><<<grid, z_threads<N1, N2, KB>(), z_smem<R, N1, N2, KB>(), st>>>(
              src, reinterpret_cast<C *>(mid), h.pz, h.nz, h.nxh, h.ns, h.nm, tmap, h.ny, &h.dsc->err);
        err = cudaGetLastError();
      });
    });
  };
  if (h.mixed && !fp64) go.template operator()<float>();
  else go.template operator()<double>();
  return err;
}

cudaError_t launch_zfwd2(Handle &h, const void *mid, void *dst, int nfield, double scale, bool dst_fp64,
                         cudaStream_t st, bool fp64) {
  cudaError_t err = cudaErrorNotSupported;
  auto go = [&]<typename R, typename D>() {
    with_shape(h.nz32, [&]<int N1, int N2>() {
      with_variant(h.tune.z, [&]<int V>() {
        using C = typename Cpx<R>::T;
        constexpr int KB = ZVar<R, tuned_variant<N1 * N2, V>()>::KB;
        dim3 grid((unsigned)((h.nxh + KB - 1) / KB), (unsigned)h.ny, (unsigned)nfield);
        CUtensorMap tmap{};
        if (zfwd_tma_map<R, N1, N2, KB>(h, mid, nfield, &tmap))
          k_zfwd2<R, N1, N2, KB, D, true><<<grid, z_threads<N1, N2, KB>(), z_smem_tma<R, N1, N2, KB, C>(N1 * N2),
                                            st>>>(reinterpret_cast<const C *>(mid), reinterpret_cast<D *>(dst), h.pz,
                                                  h.nz, h.nxh, h.ns, h.nm, scale, tmap, h.ny, &h.dsc->err);
        else
          k_zfwd2<R, N1, N2, KB, D, false><<<grid, z_threads<N1, N2, KB>(), z_smem<R, N1, N2, KB>(), st>>>(
              reinterpret_cast<const C *>(mid), reinterpret_cast<D *>(dst), h.pz, h.nz, h.nxh, h.ns, h.nm, scale,
              tmap, h.ny, &h.dsc->err);
        err = cudaGetLastError();
      });
    });
  };
  if (h.mixed && !fp64) {
    if (dst_fp64) go.template operator()<float, double2>();
    else go.template operator()<float, float2>();
  } else {
    go.template operator()<double, double2>();
  }
  return err;
}

bool z_tma_possible(const Handle &h, int zvar) {
  bool ok = false;
  auto go = [&]<typename R>() {
    with_shape(h.nz32, [&]<int N1, int N2>() {
      with_variant(zvar, [&]<int V>() {
        constexpr int KB = ZVar<R, tuned_variant<N1 * N2, V>()>::KB;
        CUtensorMap m{};
        ok = z_smem_tma<R, N1, N2, KB, double2>(h.nz) <= (size_t)opt_in_smem() &&
             z_tile_map(h.S, h.nxh, h.nz, 3 + h.nsc, h.ny, KB, sizeof(double), &m);
      });
    });
  };
  if (h.mixed) go.template operator()<float>();
  else go.template operator()<double>();
  return ok;
}

cudaError_t launch_xadj2(Handle &h, const double2 *base_mid, double2 *lmid, double scale, cudaStream_t st) {
  cudaError_t err = cudaErrorNotSupported;
  if (h.mixed) return err;
  with_shape(h.nx32, [&]<int N1, int N2>() {
    const dim3 grid((unsigned)h.nz32, (unsigned)h.ny);
    const size_t smem = sizeof(double2) * 6 * (size_t)ip_lda<N1, N2>();
    k_xadj2<N1, N2><<<grid, 128, smem, st>>>(base_mid, lmid, h.px, h.nz32, h.nxh, 1.0f / (float)h.nxh, h.nm, scale);
    err = cudaGetLastError();
  });
  return err;
}

void tile_shapes(const Handle &h, int zvar, int xvar, int *z_lines, int *x_rows, int *x_threads) {
  *z_lines = *x_rows = *x_threads = 0;
  auto zf = [&]<typename R>() {
    with_shape(h.nz32, [&]<int N1, int N2>() {
      with_variant(zvar, [&]<int V>() { *z_lines = ZVar<R, tuned_variant<N1 * N2, V>()>::KB; });
    });
    with_shape(h.nx32, [&]<int N1, int N2>() {
      with_variant(xvar, [&]<int V>() {
        using T = XVar<R, tuned_variant<N1 * N2, V>()>;
        *x_rows = T::ZB;
        *x_threads = T::ZT;
      });
    });
  };
  if (h.mixed) zf.template operator()<float>();
  else zf.template operator()<double>();
}

int xphys2_row_blocks(const Handle &h) {
  constexpr int zb = TCfg<double>::ZB;  // the statistics x pass computes in FP64 on every handle
  return (h.nz32 + zb - 1) / zb;
}

cudaError_t launch_xphys2(Handle &h, void *mid, int substep, cudaStream_t st, bool stat, double *mom) {
  cudaError_t err = cudaErrorNotSupported;
  X2Args a;
  a.ny = h.ny;
  a.nz32 = h.nz32;
  a.nxh = h.nxh;
  a.rnxh = 1.0f / (float)h.nxh;
  a.nm = h.nm;
  a.dxr = h.dxr;
  a.dzr = h.dzr;
  a.dyr = h.dops + ops_offsets(h.bw, h.ny).dyr;
  a.substep = substep;
  a.dsc = h.dsc;
  a.mom = stat ? mom : nullptr;
  auto go = [&]<typename R>() {
    with_shape(h.nx32, [&]<int N1, int N2>() {
      using C = typename Cpx<R>::T;
      if constexpr (sizeof(R) == 8) {
        if (stat) {
          // the statistics variant keeps the default shape: its moment sums are laid out per row block
          using T = TCfg<R>;
          dim3 grid((unsigned)((h.nz32 + T::ZB - 1) / T::ZB), (unsigned)h.ny);
          k_xphys2<R, N1, N2, T::ZB, T::ZT, true><<<grid, T::ZT, x_smem<R, N1, N2>(), st>>>(reinterpret_cast<C *>(mid), h.px, a);
          err = cudaGetLastError();
          return;
        }
      }
      with_variant(h.tune.x, [&]<int V>() {
        constexpr int VV = tuned_variant<N1 * N2, V>();
        using T = XVar<R, VV>;
        dim3 grid((unsigned)((h.nz32 + T::ZB - 1) / T::ZB), (unsigned)h.ny);
        if (h.nsc == 2)
          k_xphys2<R, N1, N2, T::ZB, T::ZT, false, 2, VV><<<grid, T::ZT, x_smem<R, N1, N2, 2, T::ZB>(), st>>>(
              reinterpret_cast<C *>(mid), h.px, a);
        else
          k_xphys2<R, N1, N2, T::ZB, T::ZT, false, 1, VV><<<grid, T::ZT, x_smem<R, N1, N2, 1, T::ZB>(), st>>>(
              reinterpret_cast<C *>(mid), h.px, a);
        err = cudaGetLastError();
      });
    });
  };
  // the statistics products run in FP64 on every handle: a diagnostic off the step's path, whose
  // y derivatives of third moments and pressure covariances would carry FP32 rounding of the
  // physical velocities past 1e-5 of the line
  if (h.mixed && !stat) go.template operator()<float>();
  else go.template operator()<double>();
  return err;
}

}  // namespace kmm
