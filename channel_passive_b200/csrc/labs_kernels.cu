// labs_kernels.cu - per-mode kernels outside the substep: the RK store initialisation of
// set_initial_data_uvw (initial_step.f90:139-179) and batched LABS routines (fixed_bandec,
// fixed_banbks, LABS_mat_mul_bw of module_labs.f90) on caller buffers for the unit tests.
// Mode m = kz_index * nxh + kx; element y of a line sits at y * nmodes + m.
#include <cuda_runtime.h>

#include "kmm_internal.h"
#include "labs.cuh"

namespace kmm {

namespace {

struct InitArgs {
  int ny, nxh, nz;
  int64_t nmodes, ns;
  double2 *S, *RK, *scratch;
  const double *d2, *d0lu;
  double lmfxr, lmfzr;
};

__device__ __forceinline__ DLine dline(double2 *base, int64_t off, int64_t m, int64_t stride) {
  return DLine{base + off + m, stride};
}

// set_initial_data_uvw, initial_step.f90:139-179.
template <int BW>
__global__ void k_init_stores(InitArgs a) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes) return;
  const int ny = a.ny;
  DLine Su = dline(a.S, 0 * a.ns, m, a.nmodes), Sv = dline(a.S, 1 * a.ns, m, a.nmodes);
  DLine Sw = dline(a.S, 2 * a.ns, m, a.nmodes), St = dline(a.S, 3 * a.ns, m, a.nmodes);
  DLine R1 = dline(a.RK, 0 * a.ns, m, a.nmodes), R2 = dline(a.RK, 1 * a.ns, m, a.nmodes);
  DLine R3 = dline(a.RK, 2 * a.ns, m, a.nmodes);
  if (m == 0) {
    for (int i = 1; i <= ny; ++i) {
      R1.st(i, Su.ld(i));
      R2.st(i, Sw.ld(i));
      R3.st(i, St.ld(i));
    }
    return;
  }
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;
  const double kx = kxi * a.lmfxr, kz = kzint * a.lmfzr;
  DLine c = dline(a.scratch, 0, m, a.nmodes);
  for (int i = 1; i <= ny; ++i) c.st(i, Sv.ld(i));
  labs_bs<BW>(BandS<BW>{a.d0lu}, c, ny);
  labs_mat_mul<BW>(BandS<BW>{a.d2}, c, R2, ny);
  const double k2 = kx * kx + kz * kz;
  for (int i = 1; i <= ny; ++i) {
    R2.st(i, zsub(R2.ld(i), zscale(k2, Sv.ld(i))));
    R1.st(i, zsub(zmul(z2(0.0, kz), Su.ld(i)), zmul(z2(0.0, kx), Sw.ld(i))));
    R3.st(i, St.ld(i));
  }
}

// Batched LABS kernels for the unit tests (row 18).
template <int BW>
__global__ void k_labs_lu(double *a, int ny, int nm) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nm) labs_lu<BW>(BandM<BW>{a + m, nm}, ny);
}
template <int BW>
__global__ void k_labs_bs(const double *a, double2 *b, int ny, int nm) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nm) labs_bs<BW>(BandM<BW>{const_cast<double *>(a) + m, nm}, DLine{b + m, nm}, ny);
}
template <int BW>
__global__ void k_labs_mm(const double *band, const double2 *x, double2 *b, int ny, int nm) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nm)
    labs_mat_mul<BW>(BandS<BW>{band}, DLine{const_cast<double2 *>(x) + m, nm}, DLine{b + m, nm}, ny);
}

InitArgs make_init_args(Handle &h) {
  InitArgs a;
  const OpsOffsets off = ops_offsets(h.bw, h.ny);
  a.ny = h.ny;
  a.nxh = h.nxh;
  a.nz = h.nz;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.S = h.S;
  a.RK = h.RK;
  a.scratch = h.zc;
  a.d2 = h.dops + off.d2;
  a.d0lu = h.dops + off.d0lu;
  a.lmfxr = h.lmfxr;
  a.lmfzr = h.lmfzr;
  return a;
}

template <int BW>
cudaError_t init_bw(Handle &h, cudaStream_t st) {
  const InitArgs a = make_init_args(h);
  const int threads = 128;
  k_init_stores<BW><<<(unsigned)((h.nmodes + threads - 1) / threads), threads, 0, st>>>(a);
  return cudaGetLastError();
}

template <template <int> class F, typename... Args>
cudaError_t dispatch_bw(int bw, Args &&...args) {
  switch (bw) {
    case 2: return F<2>::run(args...);
    case 3: return F<3>::run(args...);
    case 4: return F<4>::run(args...);
    case 5: return F<5>::run(args...);
    case 6: return F<6>::run(args...);
    case 7: return F<7>::run(args...);
    default: return cudaErrorInvalidValue;
  }
}

template <int BW> struct InitRun {
  static cudaError_t run(Handle &h, cudaStream_t st) { return init_bw<BW>(h, st); }
};
template <int BW> struct LuRun {
  static cudaError_t run(Handle &h, double *a, int nm, cudaStream_t st) {
    k_labs_lu<BW><<<(nm + 127) / 128, 128, 0, st>>>(a, h.ny, nm);
    return cudaGetLastError();
  }
};
template <int BW> struct BsRun {
  static cudaError_t run(Handle &h, const double *a, double2 *b, int nm, cudaStream_t st) {
    k_labs_bs<BW><<<(nm + 127) / 128, 128, 0, st>>>(a, b, h.ny, nm);
    return cudaGetLastError();
  }
};
template <int BW> struct MmRun {
  static cudaError_t run(Handle &h, const double *band, const double2 *x, double2 *b, int nm, cudaStream_t st) {
    k_labs_mm<BW><<<(nm + 127) / 128, 128, 0, st>>>(band, x, b, h.ny, nm);
    return cudaGetLastError();
  }
};

}  // namespace

cudaError_t launch_init_stores(Handle &h, cudaStream_t st) { return dispatch_bw<InitRun>(h.bw, h, st); }
cudaError_t launch_labs_lu(Handle &h, double *a, int nmodes, cudaStream_t st) {
  return dispatch_bw<LuRun>(h.bw, h, a, nmodes, st);
}
cudaError_t launch_labs_bs(Handle &h, const double *a, double2 *b, int nmodes, cudaStream_t st) {
  return dispatch_bw<BsRun>(h.bw, h, a, b, nmodes, st);
}
cudaError_t launch_labs_mat_mul(Handle &h, int which, const double2 *x, double2 *b, int nmodes,
                                cudaStream_t st) {
  OpsOffsets off = ops_offsets(h.bw, h.ny);
  const double *band = h.dops + (which == 0 ? off.d0 : which == 1 ? off.d1 : off.d2);
  return dispatch_bw<MmRun>(h.bw, h, band, x, b, nmodes, st);
}

}  // namespace kmm
