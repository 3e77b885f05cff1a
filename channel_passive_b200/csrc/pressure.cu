// pressure.cu - the pressure of a state (get_pressure / cal_pressure / solve_ppe,
// get_pressure.f90:1-137), computed on the device the way a statistics step does it
// (time_march.f90:47-110): <vv> from the state (get_statistics_1 -> get_uv), the substep-1
// products with f6 = v v (y_to_x, dft_x_realspace on a statistics substep, x_to_y,
// rescale_data), then per (kx, kz)
//   rhs = kx^2 f1 + kz^2 f3 + k^2 f6 + 2 kx kz f5 - D2 D0^{-1} f6 - 2 D1 D0^{-1} g,
//   g = i kx f2 + i kz f4 on rows 2..ny-1 and D0^{-1} f6 on rows 1, ny (as the reference
//   leaves them), rhs on rows 1, ny = the wall values stat_PPE_boundary = nu d2v/dy2 of the
//   state's v (get_y_dir_deriv_of_field_with_PPE_BC, get_statistics.f90:689-719; stats.cu
//   k_ydiff computes them),
//   (D2 - k^2 D0 with D1 rows at the walls) c = rhs,  p = D0 c,
// and p = -<vv> for the (0,0) mode.  One thread per mode runs the six sweeps (sweeps.cuh): this
// is a diagnostic of statistics steps, not part of the time step, and its products are formed in
// FP64 on every handle.  In FP32 (a mixed handle's step precision) the y derivatives of the
// third-moment and pressure-covariance averages, whose terms cancel to about 1e-2 of their size,
// carried the rounding of the physical velocities to 1.2e-5 of the line.
#include <cuda_runtime.h>

#include "kmm_internal.h"
#include "sweeps.cuh"

namespace kmm {

namespace {

struct PpeArgs {
  int ny, nxh, nz;
  int64_t nmodes, ns;
  const double2 *P;   // products f1..f6 in slots 0..5
  double2 *zl;        // 2 complex scratch lines
  const double2 *bc;  // [2][nmodes] wall values of rows 1 and ny
  double *ub;         // U factor region
  const double *tabs;
  double lmfxr, lmfzr;
  double2 *out;       // pressure planes [y][mode]
};

template <int BW>
__global__ void __launch_bounds__(128) k_ppe(PpeArgs a) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0 || m >= a.nmodes) return;
  const int n = a.ny;
  const int64_t nm = a.nmodes, ns = a.ns;
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;
  const double kx = kxi * a.lmfxr, kz = kzint * a.lmfzr;
  const double k2 = kx * kx + kz * kz, kxkz = kx * kz;
  const Tabs<BW> tb = tabs_at<BW>(a.tabs, n);
  const double2 *P = a.P + m;
  auto prod = [&](int slot, int r) { return P[slot * ns + (r - 1) * (int)nm]; };
  auto pfp = [&](int slot, int r) { pf_l1(P + slot * ns + (r - 1) * (int)nm); };
  const DLine Z{a.zl + m, nm}, Rh{a.zl + ns + m, nm}, Pout{a.out + m, nm};
  const UBand<BW> ub = make_uband<BW>(a.ub + m, nm, ns);
  auto ufix = [&](int r, int e) { return tb.u0[(r - 1) * 2 * BW + e - 1]; };

  // c6 = D0^{-1} f6; rhs = kx^2 f1 + kz^2 f3 + k^2 f6 + 2 kx kz f5 - D2 c6 on rows 2..ny-1
  fwd_fixed<BW, 1>(tb, n, [&](int r, double2 *b) { b[0] = prod(5, r); },
                   [&](int r, const double2 *z) { Z.st(r, z[0]); }, [&](int r) { pfp(5, r); });
  double2 c6_1 = z2(0.0, 0.0), c6_n = z2(0.0, 0.0);
  bwd_emit<BW, 1, 0>(n, ufix, [&](int r, double2 *zc, double *) { zc[0] = Z.ld(r); },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        if (q == 1) c6_1 = wc[0][0];       // emitted at step r = 1
        if (q == n) c6_n = wc[0][2 * BW];  // emitted at step r = n - 2BW
        double2 rh = z2(0.0, 0.0);
        if (q != 1 && q != n) {
          const double2 f1 = prod(0, q), f3 = prod(2, q), f5 = prod(4, q), f6 = prod(5, q);
          const double2 d2 = mvc<BW>(tb.t2, q, r, wc[0]);
          rh.x = kx * kx * f1.x + kz * kz * f3.x + k2 * f6.x + 2.0 * kxkz * f5.x;
          rh.y = kx * kx * f1.y + kz * kz * f3.y + k2 * f6.y + 2.0 * kxkz * f5.y;
          rh = zsub(rh, d2);
        }
        Rh.st(q, rh);
      },
      [&](int r) {
        pf_l1(Z.p + (r - 1) * (int)nm);
        if (r <= n - 2 * BW) {
          pfp(0, r + BW);
          pfp(2, r + BW);
          pfp(4, r + BW);
          pfp(5, r + BW);
        }
      });
  // g = i kx f2 + i kz f4 (rows 2..ny-1), c6 on rows 1, ny; rhs -= 2 D1 D0^{-1} g; the wall
  // rows take the wall values
  fwd_fixed<BW, 1>(tb, n,
      [&](int r, double2 *b) {
        if (r == 1) b[0] = c6_1;
        else if (r == n) b[0] = c6_n;
        else {
          const double2 f2 = prod(1, r), f4 = prod(3, r);
          b[0] = z2(-kx * f2.y - kz * f4.y, kx * f2.x + kz * f4.x);
        }
      },
      [&](int r, const double2 *z) { Z.st(r, z[0]); },
      [&](int r) {
        pfp(1, r);
        pfp(3, r);
      });
  bwd_emit<BW, 1, 0>(n, ufix, [&](int r, double2 *zc, double *) { zc[0] = Z.ld(r); },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        if (q == 1 || q == n) {
          Rh.st(q, a.bc[(q == 1 ? 0 : nm) + m]);
        } else {
          const double2 d1 = mvc<BW>(tb.t1, q, r, wc[0]);
          const double2 rh = Rh.ld(q);
          Rh.st(q, z2(rh.x - 2.0 * d1.x, rh.y - 2.0 * d1.y));
        }
      },
      [&](int r) {
        pf_l1(Z.p + (r - 1) * (int)nm);
        if (r <= n - 2 * BW) pf_l1(Rh.p + (r + BW - 1) * (int)nm);
      });
  // (D2 - k^2 D0, D1 rows at the walls) c = rhs; p = D0 c
  lu_fwd<BW, 1, 0>(n,
      [&](int r, double *row, bool centre) {
        if (r == 1 || r == n) {
          const double *r1 = trow<BW>(tb.t1, r);
#pragma unroll
          for (int e = -2 * BW; e <= 2 * BW; ++e) row[e + 2 * BW] = r1[e];
          return;
        }
        const double *r0 = trow<BW>(tb.t0, r), *r2 = trow<BW>(tb.t2, r);
        if (centre) {
#pragma unroll
          for (int e = -BW; e <= BW; ++e) row[e + 2 * BW] = -k2 * r0[e] + r2[e];
          return;
        }
#pragma unroll
        for (int e = -2 * BW; e <= 2 * BW; ++e) row[e + 2 * BW] = -k2 * r0[e] + r2[e];
      },
      [&](int r, double2 *bc, double *) { bc[0] = Rh.ld(r); },
      [&](int r, const double2 *zc, const double *) { Z.st(r, zc[0]); }, ub,
      [&](int r) { pf_l1(Rh.p + (r - 1) * (int)nm); });
  bwd_emit<BW, 1, 0>(n, [&](int r, int e) { return ub.get(r, e); },
      [&](int r, double2 *zc, double *) { zc[0] = Z.ld(r); },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        Pout.st(q, mvc<BW>(tb.t0, q, r, wc[0]));
      },
      [&](int r) {
        pf_l1(Z.p + (r - 1) * (int)nm);
#pragma unroll
        for (int e = 1; e <= BW; ++e) pf_l1(ub.p + (e - 1) * (int)ns + (r - 1) * (int)nm);
      });
}

// The mean mode: p(y) = -<vv>(y) with <vv> = sum over the stored modes of |v|^2, weight 1 on the
// kx = 0 plane and 2 elsewhere (get_uv, get_statistics.f90:982-1017).  One block per y.
__global__ void __launch_bounds__(256) k_mean_vv(const double2 *__restrict__ v, double2 *__restrict__ out,
                                                 int64_t nmodes, int nxh) {
  const int y = blockIdx.x;
  const double2 *row = v + (int64_t)y * nmodes;
  double acc = 0.0;
  for (int64_t m = threadIdx.x; m < nmodes; m += blockDim.x) {
    const double2 a = row[m];
    const double w = (m % nxh == 0) ? 1.0 : 2.0;
    acc += w * (a.x * a.x + a.y * a.y);
  }
  __shared__ double red[256 / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < 256 / 32; ++i) s += red[i];
    out[(int64_t)y * nmodes] = make_double2(-s, 0.0);
  }
}

template <int BW>
cudaError_t ppe_bw(Handle &h, const double2 *P, double2 *out, const double2 *bc, cudaStream_t st) {
  const OpsOffsets off = ops_offsets(h.bw, h.ny);
  PpeArgs a;
  a.ny = h.ny;
  a.nxh = h.nxh;
  a.nz = h.nz;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.P = P;
  a.zl = h.zc;
  a.bc = bc;
  a.ub = h.ub;
  a.tabs = h.dops + off.t0;
  a.lmfxr = h.lmfxr;
  a.lmfzr = h.lmfzr;
  a.out = out;
  const unsigned blocks = (unsigned)((h.nmodes + 127) / 128);
  k_ppe<BW><<<blocks, 128, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t launch_pressure(Handle &h, double2 *out, const double2 *bc, double *mom, cudaStream_t st) {
  // <vv> from the state's v before the transforms overwrite anything (get_statistics_1)
  k_mean_vv<<<h.ny, 256, 0, st>>>(h.S + h.ns, out, h.nmodes, h.nxh);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  // substep-1 products of a statistics step in FP64: f1..f6 in P slots 0..5, rescaled
  void *mid = h.mixed ? static_cast<void *>(h.mid64) : h.MID;
  double2 *P = h.mixed ? h.p64 : static_cast<double2 *>(h.P);
  if (!mid || !P) return cudaErrorInvalidValue;
  if ((e = launch_zinv(h, h.S, mid, 4, st, true)) != cudaSuccess) return e;
  if ((e = launch_xphys2(h, mid, 2, st, true, mom)) != cudaSuccess) return e;
  if ((e = launch_zfwd(h, mid, P, 6, h.rescale, true, st, true)) != cudaSuccess) return e;
  switch (h.bw) {
    case 2: return ppe_bw<2>(h, P, out, bc, st);
    case 3: return ppe_bw<3>(h, P, out, bc, st);
    case 4: return ppe_bw<4>(h, P, out, bc, st);
    case 5: return ppe_bw<5>(h, P, out, bc, st);
    case 6: return ppe_bw<6>(h, P, out, bc, st);
    case 7: return ppe_bw<7>(h, P, out, bc, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kmm
