// labs_kernels.cu - per-mode kernels outside the substep: the RK store initialisation of
// set_initial_data_uvw (initial_step.f90:139-179) and batched LABS routines (fixed_bandec,
// fixed_banbks, LABS_mat_mul_bw of module_labs.f90) on caller buffers for the unit tests.
// Mode m = kz_index * nxh + kx; element y of a line sits at y * nmodes + m.
#include <cuda_runtime.h>

#include "kmm_internal.h"
#include "labs.cuh"
#include "sweeps.cuh"

namespace kmm {

namespace {

struct InitArgs {
  int ny, nxh, nz, nsc;
  int64_t nmodes, ns;
  double2 *S, *RK, *scratch;
  const double *tabs;  // offset tables T0, T1, T2, L0, U0
  double lmfxr, lmfzr;
};

__device__ __forceinline__ DLine dline(double2 *base, int64_t off, int64_t m, int64_t stride) {
  return DLine{base + off + m, stride};
}

// set_initial_data_uvw, initial_step.f90:139-179: RK_STORE 1 = i kz u - i kx w,
// RK_STORE 2 = D2 D0^{-1} v - k^2 v, RK_STORE 3 = theta; the mean mode stores U, W, Theta.  One
// thread per mode: the D0 solve of v runs through the fixed D0 profile LU (sweeps.cuh) and D2 of
// it is emitted from the backward window.  PHI_ONLY: RK_STORE 2 of the modes other than (0,0),
// which needs v alone (k_init_elem does the rest), so it can start before u, w, theta arrive.
template <int BW, bool PHI_ONLY = false>
__global__ void __launch_bounds__(128) k_init_stores(InitArgs a) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes || (PHI_ONLY && m == 0)) return;
  const int n = a.ny;
  const int64_t nm = a.nmodes;
  const DLine Su = dline(a.S, 0 * a.ns, m, nm), Sv = dline(a.S, 1 * a.ns, m, nm);
  const DLine Sw = dline(a.S, 2 * a.ns, m, nm), St = dline(a.S, 3 * a.ns, m, nm);
  const DLine R1 = dline(a.RK, 0 * a.ns, m, nm), R2 = dline(a.RK, 1 * a.ns, m, nm);
  const DLine R3 = dline(a.RK, 2 * a.ns, m, nm);
  if (m == 0) {
    for (int i = 1; i <= n; ++i) {
      R1.st(i, Su.ld(i));
      R2.st(i, Sw.ld(i));
      R3.st(i, St.ld(i));
    }
    if (a.nsc == 2) {  // the second scalar's store is the scalar, as RK_STORE 3 is theta
      const DLine S4 = dline(a.S, 4 * a.ns, m, nm), R4 = dline(a.RK, 3 * a.ns, m, nm);
      for (int i = 1; i <= n; ++i) R4.st(i, S4.ld(i));
    }
    return;
  }
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;
  const double kx = kxi * a.lmfxr, kz = kzint * a.lmfzr;
  const double k2 = kx * kx + kz * kz;
  const Tabs<BW> tb = tabs_at<BW>(a.tabs, n);
  const DLine Z = dline(a.scratch, 0, m, nm);
  auto ufix = [&](int r, int e) { return tb.u0[(r - 1) * 2 * BW + e - 1]; };
  fwd_fixed<BW, 1>(tb, n, [&](int r, double2 *b) { b[0] = Sv.ld(r); },
                   [&](int r, const double2 *z) { Z.st(r, z[0]); },
                   [&](int r) { pf_l1(Sv.p + (r - 1) * (int)nm); });
  bwd_emit<BW, 1, 0>(n, ufix, [&](int r, double2 *zc, double *) { zc[0] = Z.ld(r); },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        R2.st(q, zsub(mvc<BW>(tb.t2, q, r, wc[0]), zscale(k2, Sv.ld(q))));
        if constexpr (!PHI_ONLY) {
          R1.st(q, zsub(zmul(z2(0.0, kz), Su.ld(q)), zmul(z2(0.0, kx), Sw.ld(q))));
          R3.st(q, St.ld(q));
          if (a.nsc == 2) a.RK[3 * a.ns + (q - 1) * nm + m] = a.S[4 * a.ns + (q - 1) * nm + m];
        }
      },
      [&](int r) {
        pf_l1(Z.p + (r - 1) * (int)nm);
        if (r <= n - 2 * BW) {
          const int64_t o = (r + BW - 1) * (int)nm;
          pf_l1(Sv.p + o);
          if constexpr (PHI_ONLY) return;
          pf_l1(Su.p + o);
          pf_l1(Sw.p + o);
          pf_l1(St.p + o);
        }
      });
}

// The element-wise rest of set_initial_data_uvw beside k_init_stores<BW, true>: RK_STORE 1 =
// i kz u - i kx w and RK_STORE 3 = theta, and the mean mode's stores U, W, Theta
// (initial_step.f90:139-179).  One thread per (mode, y).
__global__ void __launch_bounds__(256) k_init_elem(InitArgs a) {
  const int64_t nm = a.nmodes, ns = a.ns;
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= nm) return;
  const int64_t o = (int64_t)blockIdx.y * nm + m;
  const double2 u = a.S[o], w = a.S[2 * ns + o];
  if (m == 0) {
    a.RK[o] = u;
    a.RK[ns + o] = w;
  } else {
    const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
    const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;
    const double kx = kxi * a.lmfxr, kz = kzint * a.lmfzr;
    a.RK[o] = zsub(zmul(z2(0.0, kz), u), zmul(z2(0.0, kx), w));
  }
  a.RK[2 * ns + o] = a.S[3 * ns + o];
  if (a.nsc == 2) a.RK[3 * ns + o] = a.S[4 * ns + o];
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
  a.nsc = h.nsc;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.S = h.S;
  a.RK = h.RK;
  a.scratch = h.zc;
  a.tabs = h.dops + off.t0;
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
template <int BW> struct InitPhiRun {
  static cudaError_t run(Handle &h, cudaStream_t st) {
    const InitArgs a = make_init_args(h);
    k_init_stores<BW, true><<<(unsigned)((h.nmodes + 127) / 128), 128, 0, st>>>(a);
    return cudaGetLastError();
  }
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
cudaError_t launch_init_phi(Handle &h, cudaStream_t st) { return dispatch_bw<InitPhiRun>(h.bw, h, st); }
cudaError_t launch_init_elem(Handle &h, cudaStream_t st) {
  const InitArgs a = make_init_args(h);
  const dim3 grid((unsigned)((h.nmodes + 255) / 256), (unsigned)h.ny);
  k_init_elem<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}
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
