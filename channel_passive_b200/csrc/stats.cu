// stats.cu - the statistics of a statistics step on the device: get_statistics_1
// (get_statistics.f90:9-368), write_spectra (write_energy_spectra.f90:9-399), the moment sums of
// dft_x_realspace on a statistics substep (dft_x_realspace.f90:41-57, 128-155, 238-484) and
// get_statistics_2 (get_statistics.f90:376-539), all from the state at the start of a step.
//
// Order of work (launch_statistics):
//   k_ydiff         per mode, one warp per field: du/dy, dv/dy, dw/dy = D1 D0^{-1} (u, v, w)
//                   and the pressure wall values nu (D2 D0^{-1} v) on rows 1 and ny
//   launch_pressure <vv>, the statistics-substep products with the moment sums, the PPE
//   k_spectra       one block per y: the 18 spectra in kx and in kz, the <ab> and vorticity
//                   lines (sums of the kx spectra), dissipation, pressure covariance and
//                   pressure-strain lines
//   k_mom_reduce    per y: the moment lines from the x pass's per-block sums
//   k_stat_lines    the line solves: mean-line derivatives, centre-line values, -d<..>/dy
// Every sum runs in a fixed order (no atomics), so repeated calls give identical results.
#include <cuda_runtime.h>

#include "kmm_internal.h"
#include "labs.cuh"
#include "stats.cuh"
#include "sweeps.cuh"

namespace kmm {

namespace {

// ---- y derivatives and the PPE wall values -------------------------------------------------
struct YdiffArgs {
  int ny;
  int64_t nmodes, ns;
  const double2 *S;  // state planes, fields u, v, w at 0, ns, 2 ns
  double2 *zl;       // 3 forward scratch lines
  double2 *d;        // 3 output lines
  double2 *bc;       // [2][nmodes]
  const double *tabs;
  double nu;
  int mask;
};

// get_y_dir_deriv_of_field (get_statistics.f90:658-681) for u and w and
// get_y_dir_deriv_of_field_with_PPE_BC (get_statistics.f90:689-719) for v: c = D0^{-1} f through
// the fixed D0 profile LU, D1 c emitted from the backward window; for v also
// BC1 = nu (D2(1,1) c1 + D2(1,2) c2 + D2(1,3) c3), BC2 = nu (D2(n,n-2) c_{n-2} + ... + D2(n,n) c_n).
template <int BW>
__global__ void __launch_bounds__(96) k_ydiff(YdiffArgs a) {
  const int role = threadIdx.x >> 5;
  const int64_t m = (int64_t)blockIdx.x * 32 + (threadIdx.x & 31);
  if (!((a.mask >> role) & 1) || m >= a.nmodes) return;
  const int n = a.ny;
  const int64_t nm = a.nmodes, ns = a.ns;
  const Tabs<BW> tb = tabs_at<BW>(a.tabs, n);
  const DLine F{const_cast<double2 *>(a.S) + role * ns + m, nm};
  const DLine Z{a.zl + role * ns + m, nm}, D{a.d + role * ns + m, nm};
  auto ufix = [&](int r, int e) { return tb.u0[(r - 1) * 2 * BW + e - 1]; };
  fwd_fixed<BW, 1>(tb, n, [&](int r, double2 *b) { b[0] = F.ld(r); },
                   [&](int r, const double2 *z) { Z.st(r, z[0]); },
                   [&](int r) { pf_l1(F.p + (r - 1) * (int)nm); });
  bwd_emit<BW, 1, 0>(n, ufix, [&](int r, double2 *zc, double *) { zc[0] = Z.ld(r); },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        D.st(q, mvc<BW>(tb.t1, q, r, wc[0]));
        if (role == 1 && q == 1) {  // emitted at r = 1: wc[0][j] = c_{1+j}
          const double *t2 = trow<BW>(tb.t2, 1);
          double2 s;
          s.x = t2[0] * wc[0][0].x + t2[1] * wc[0][1].x + t2[2] * wc[0][2].x;
          s.y = t2[0] * wc[0][0].y + t2[1] * wc[0][1].y + t2[2] * wc[0][2].y;
          a.bc[m] = z2(a.nu * s.x, a.nu * s.y);
        }
        if (role == 1 && q == n) {  // emitted at r = n - 2BW: wc[0][j] = c_{n-2BW+j}
          const double *t2 = trow<BW>(tb.t2, n);
          double2 s;
          s.x = t2[-2] * wc[0][2 * BW - 2].x + t2[-1] * wc[0][2 * BW - 1].x + t2[0] * wc[0][2 * BW].x;
          s.y = t2[-2] * wc[0][2 * BW - 2].y + t2[-1] * wc[0][2 * BW - 1].y + t2[0] * wc[0][2 * BW].y;
          a.bc[nm + m] = z2(a.nu * s.x, a.nu * s.y);
        }
      },
      [&](int r) { pf_l1(Z.p + (r - 1) * (int)nm); });
}

template <int BW>
cudaError_t ydiff_bw(Handle &h, int mask, cudaStream_t st) {
  YdiffArgs a;
  a.ny = h.ny;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.S = h.S;
  a.zl = h.zc;
  a.d = h.ec;
  a.bc = h.dvw;
  a.tabs = h.dops + ops_offsets(h.bw, h.ny).t0;
  a.nu = h.cfg.nu;
  a.mask = mask;
  k_ydiff<BW><<<(unsigned)((h.nmodes + 31) / 32), 96, 0, st>>>(a);
  return cudaGetLastError();
}

// ---- spectra and mode-sum lines ------------------------------------------------------------
struct SpecArgs {
  int ny, nxh, nz;
  int64_t nmodes, ns;
  const double2 *S;  // u, v, w, theta planes
  const double2 *D;  // du/dy, dv/dy, dw/dy planes
  const double2 *P;  // pressure planes
  double lmfxr, lmfzr, nu;
  double *skx, *skz, *lines;
};

__device__ __forceinline__ double re2(double2 a, double2 b) { return a.x * b.x + a.y * b.y; }
// Re a Im p - Im a Re p: Re((i a) conj(p)) / i-free form of get_turb_transport_PI1_ij
__device__ __forceinline__ double crs(double2 a, double2 p) { return a.x * p.y - a.y * p.x; }

__device__ __forceinline__ double warp_sum(double x) {
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Line index of the mode sum of each kx spectrum (get_statistics_1's get_uv calls).
__constant__ int c_spec_line[kNumSpec] = {6, 7, 9, 10, 11, 13, 12, 14, 16, 15, 21, 22, 23, 24, 26, 25, 27, 28};
// Lines of the mode-sum-only quantities: dissipation uu, vv, ww, uv; up, vp, wp, pp;
// 2 p du/dx, 2 p dv/dy, 2 p dw/dz, p du/dy + p dv/dx.
constexpr int kNumOnly = 12;
__constant__ int c_only_line[kNumOnly] = {17, 18, 19, 20, 48, 50, 52, 53, 54, 55, 56, 57};

// One block per y.  Warp w takes the kz rows w, w + NW, ...; lane l the kx = l, l + 32, ...
// E_kz(kz, y) is the warp's shuffle sum of its row; E_kx(kx, y) accumulates per warp in shared
// memory ([NW][18][nxh], each entry owned by one lane) and is summed over the warps in order.
// Spectrum pairs (write_energy_spectra.f90:76-154 in kx, :157-226 in kz): uu vv ww tt uv vw uw
// ut vt wt, ox ox, oy oy, oz oz, ox oy, ox oz, oy oz, v oz, w oy; the kz list takes ox oz for
// its "oz oz" entry, as the reference's call does (write_energy_spectra.f90:218-219).
template <int NW>
__global__ void __launch_bounds__(NW * 32) k_spectra(SpecArgs a) {
  extern __shared__ double sk[];
  const int y = blockIdx.x, lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nxh = a.nxh, nz = a.nz, ny = a.ny;
  for (int i = threadIdx.x; i < NW * kNumSpec * nxh; i += NW * 32) sk[i] = 0.0;
  __syncthreads();
  double *my = sk + wid * kNumSpec * nxh;
  double only[kNumOnly];
#pragma unroll
  for (int j = 0; j < kNumOnly; ++j) only[j] = 0.0;
  const int64_t row = (int64_t)y * a.nmodes, ns = a.ns;
  const double tnu = 2.0 * a.nu;
  for (int kz = wid; kz < nz; kz += NW) {
    const double kzw = (double)(kz <= nz / 2 ? kz : kz - nz) * a.lmfzr;
    double zs[kNumSpec];
#pragma unroll
    for (int i = 0; i < kNumSpec; ++i) zs[i] = 0.0;
    for (int kx = lane; kx < nxh; kx += 32) {
      const int64_t o = row + (int64_t)kz * nxh + kx;
      const double2 u = a.S[o], v = a.S[ns + o], w = a.S[2 * ns + o], t = a.S[3 * ns + o];
      const double2 du = a.D[o], dv = a.D[ns + o], dw = a.D[2 * ns + o], p = a.P[o];
      const double kxw = (double)kx * a.lmfxr, wt = kx == 0 ? 1.0 : 2.0;
      // get_vorticity_field (get_statistics.f90:912-948)
      const double2 ox = z2(dw.x + kzw * v.y, dw.y - kzw * v.x);
      const double2 oy = z2(-kzw * u.y + kxw * w.y, kzw * u.x - kxw * w.x);
      const double2 oz = z2(-kxw * v.y - du.x, kxw * v.x - du.y);
      double q[kNumSpec];
      q[0] = re2(u, u); q[1] = re2(v, v); q[2] = re2(w, w); q[3] = re2(t, t);
      q[4] = re2(u, v); q[5] = re2(v, w); q[6] = re2(u, w); q[7] = re2(u, t);
      q[8] = re2(v, t); q[9] = re2(t, w);
      q[10] = re2(ox, ox); q[11] = re2(oy, oy); q[12] = re2(oz, oz); q[13] = re2(ox, oy);
      q[14] = re2(ox, oz); q[15] = re2(oy, oz); q[16] = re2(v, oz); q[17] = re2(w, oy);
#pragma unroll
      for (int i = 0; i < kNumSpec; ++i) {
        const double x = wt * q[i];
        zs[i] += x;
        my[i * nxh + kx] += x;
      }
      // get_turb_transport_e_ij (get_statistics.f90:761-810)
      const double k2 = kxw * kxw + kzw * kzw;
      only[0] += tnu * wt * (k2 * q[0] + re2(du, du));
      only[1] += tnu * wt * (k2 * q[1] + re2(dv, dv));
      only[2] += tnu * wt * (k2 * q[2] + re2(dw, dw));
      only[3] += tnu * wt * (k2 * q[4] + re2(du, dv));
      // get_uv with the pressure (get_statistics.f90:466-508)
      only[4] += wt * re2(u, p);
      only[5] += wt * re2(v, p);
      only[6] += wt * re2(w, p);
      only[7] += wt * re2(p, p);
      // get_turb_transport_PI1_ij (get_statistics.f90:817-902)
      only[8] += wt * 2.0 * kxw * crs(u, p);
      only[9] += wt * 2.0 * re2(dv, p);
      only[10] += wt * 2.0 * kzw * crs(w, p);
      only[11] += wt * (kxw * crs(v, p) + re2(du, p));
    }
#pragma unroll
    for (int i = 0; i < kNumSpec; ++i) {
      const double x = warp_sum(zs[i == 12 ? 14 : i]);
      if (lane == 0) a.skz[((int64_t)i * nz + kz) * ny + y] = x;
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < kNumSpec * nxh; idx += NW * 32) {
    double x = 0.0;
    for (int w = 0; w < NW; ++w) x += sk[w * kNumSpec * nxh + idx];
    const int i = idx / nxh, kx = idx - i * nxh;
    a.skx[((int64_t)i * nxh + kx) * ny + y] = x;
    sk[idx] = x;  // warp 0's copy: only this thread touches index idx of it
  }
  __shared__ double ored[NW][kNumOnly];
#pragma unroll
  for (int j = 0; j < kNumOnly; ++j) {
    const double x = warp_sum(only[j]);
    if (lane == 0) ored[wid][j] = x;
  }
  __syncthreads();
  for (int i = wid; i < kNumSpec; i += NW) {
    double x = 0.0;
    for (int kx = lane; kx < nxh; kx += 32) x += sk[i * nxh + kx];
    x = warp_sum(x);
    if (lane == 0) {
      a.lines[c_spec_line[i] * ny + y] = x;
      if (i == 1) a.lines[8 * ny + y] = -x;  // "P" = -<vv>
    }
  }
  if (threadIdx.x < kNumOnly) {
    double x = 0.0;
    for (int w = 0; w < NW; ++w) x += ored[w][threadIdx.x];
    a.lines[c_only_line[threadIdx.x] * ny + y] = x;
  }
}

template <int NW>
size_t spectra_smem(int nxh) {
  return sizeof(double) * (size_t)NW * kNumSpec * nxh;
}

// ---- moments -------------------------------------------------------------------------------
// Per y: the x pass's per-block moment sums, summed over the blocks in order and scaled by
// rescale = 1/(nx32 nz32) (dft_x_realspace.f90:238-424): lines 29..43 (u^3 .. w^10, rows 1 and
// ny set to 0) and the transport inputs tr[j] = rescale * (sum of -u u v, -v v v, -v w w, -u v v)
// (dft_x_realspace.f90:426-484).
__global__ void k_mom_reduce(const double *__restrict__ part, int nblk, int ny, double rescale,
                             double *__restrict__ lines, double *__restrict__ tr) {
  const int y = blockIdx.x, i = threadIdx.x;
  if (i >= kNumMoments) return;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[((int64_t)y * nblk + b) * kNumMoments + i];
  if (i < 15) lines[(29 + i) * ny + y] = (y == 0 || y == ny - 1) ? 0.0 : rescale * s;
  if (i == 1) tr[1 * ny + y] = rescale * -s;
  if (i == 15) tr[0 * ny + y] = rescale * s;
  if (i == 16) tr[2 * ny + y] = rescale * s;
  if (i == 17) tr[3 * ny + y] = rescale * s;
}

// ---- line solves ---------------------------------------------------------------------------
struct LinesArgs {
  int ny;
  int64_t nmodes, ns;
  const double2 *S;
  const double *d0lu, *d1, *center;
  const double *tr;   // [4][ny] transport inputs
  double *lines;      // [58][ny]
  double *scal;       // u_center, t_center
  double2 *scr;       // [9][2][ny] scratch
  double u_gal;
};

// Nine threads, one line each, through labs_bs (D0_LU) and labs_mat_mul (D1) in the reference's
// elimination order (module_labs.f90:4252-4318, 4687-4722):
//   0 U: dUdy and U_c = u_gal + sum_k Re c_k centre_k (get_dudy_u_center, get_statistics.f90:548-581)
//   1 W: dWdy (get_dwdy, :626-652)      2 theta: dTdy and T_c (get_dtdy_t_center, :586-620)
//   3..6 -d<uuv>/dy, -d<vvv>/dy, -d<vww>/dy, -d<uvv>/dy (dft_x_realspace.f90:426-484)
//   7 -d<up>/dy, 8 -2 d<vp>/dy (get_statistics.f90:466-495)
// and the mean lines U = Re U00 + u_gal, W, Theta (get_u, get_statistics.f90:1024-1048).
template <int BW>
__global__ void k_stat_lines(LinesArgs a) {
  const int job = threadIdx.x, n = a.ny;
  if (job >= 9) return;
  const DLine c{a.scr + (int64_t)job * 2 * n, 1}, out{a.scr + (int64_t)job * 2 * n + n, 1};
  const int field = job == 0 ? 0 : (job == 1 ? 2 : 3);
  for (int r = 1; r <= n; ++r) {
    double2 x;
    if (job <= 2) x = a.S[field * a.ns + (int64_t)(r - 1) * a.nmodes];
    else if (job <= 6) x = z2(a.tr[(job - 3) * n + r - 1], 0.0);
    else x = z2(a.lines[(job == 7 ? 48 : 50) * n + r - 1], 0.0);
    c.st(r, x);
    if (job == 0) a.lines[0 * n + r - 1] = x.x + a.u_gal;
    if (job == 1) a.lines[1 * n + r - 1] = x.x;
    if (job == 2) a.lines[2 * n + r - 1] = x.x;
  }
  labs_bs<BW>(BandS<BW>{a.d0lu}, c, n);
  labs_mat_mul<BW>(BandS<BW>{a.d1}, c, out, n);
  const int dst[9] = {3, 4, 5, 44, 45, 46, 47, 49, 51};
  const double scale = job == 7 ? -1.0 : (job == 8 ? -2.0 : 1.0);
  for (int r = 1; r <= n; ++r) a.lines[dst[job] * n + r - 1] = scale * out.ld(r).x;
  if (job == 0 || job == 2) {
    double s = job == 0 ? a.u_gal : 0.0;
    for (int k = 1; k <= n; ++k) s = s + c.ld(k).x * a.center[k - 1];
    a.scal[job == 0 ? 0 : 1] = s;
  }
}

template <int BW>
cudaError_t stat_lines_bw(Handle &h, const StatLayout &L, cudaStream_t st) {
  const OpsOffsets off = ops_offsets(h.bw, h.ny);
  LinesArgs a;
  a.ny = h.ny;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.S = h.S;
  a.d0lu = h.dops + off.d0lu;
  a.d1 = h.dops + off.d1;
  a.center = h.stat + L.center;
  a.tr = h.stat + L.tr;
  a.lines = h.stat + L.lines;
  a.scal = h.stat + L.scal;
  a.scr = reinterpret_cast<double2 *>(h.stat + L.scr);
  a.u_gal = h.cfg.u_gal;
  k_stat_lines<BW><<<1, 32, 0, st>>>(a);
  return cudaGetLastError();
}

template <int NW>
cudaError_t spectra_nw(Handle &h, const StatLayout &L, cudaStream_t st) {
  SpecArgs a;
  a.ny = h.ny;
  a.nxh = h.nxh;
  a.nz = h.nz;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.S = h.S;
  a.D = h.ec;
  a.P = h.staging;
  a.lmfxr = h.lmfxr;
  a.lmfzr = h.lmfzr;
  a.nu = h.cfg.nu;
  a.skx = h.stat + L.skx;
  a.skz = h.stat + L.skz;
  a.lines = h.stat + L.lines;
  const size_t smem = spectra_smem<NW>(h.nxh);
  cudaError_t e = cudaFuncSetAttribute(k_spectra<NW>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_spectra<NW><<<h.ny, NW * 32, smem, st>>>(a);
  return cudaGetLastError();
}

constexpr size_t kSpectraSmemCap = 200 * 1024;

}  // namespace

StatLayout stat_layout(const Handle &h) {
  StatLayout L;
  int64_t o = 0;
  L.part = o;
  o += (int64_t)h.ny * xphys2_row_blocks(h) * kNumMoments;
  L.tr = o;
  o += 4 * (int64_t)h.ny;
  L.lines = o;
  o += (int64_t)KMM_STAT_NLINES * h.ny;
  L.skx = o;
  o += (int64_t)kNumSpec * h.nxh * h.ny;
  L.skz = o;
  o += (int64_t)kNumSpec * h.nz * h.ny;
  L.scal = o;
  o += 2;
  L.center = o;
  o += h.ny;
  o = (o + 1) & ~(int64_t)1;  // double2 alignment of the scratch lines
  L.scr = o;
  o += 9 * 2 * 2 * (int64_t)h.ny;
  L.total = o;
  return L;
}

cudaError_t launch_ydiff(Handle &h, int mask, cudaStream_t st) {
  switch (h.bw) {
    case 2: return ydiff_bw<2>(h, mask, st);
    case 3: return ydiff_bw<3>(h, mask, st);
    case 4: return ydiff_bw<4>(h, mask, st);
    case 5: return ydiff_bw<5>(h, mask, st);
    case 6: return ydiff_bw<6>(h, mask, st);
    case 7: return ydiff_bw<7>(h, mask, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_statistics(Handle &h, cudaStream_t st) {
  if (!h.stat) return cudaErrorInvalidValue;
  const StatLayout L = stat_layout(h);
  cudaError_t e;
  if ((e = launch_ydiff(h, 7, st)) != cudaSuccess) return e;
  if ((e = launch_pressure(h, h.staging, h.dvw, h.stat + L.part, st)) != cudaSuccess) return e;
  if (spectra_smem<8>(h.nxh) <= kSpectraSmemCap) e = spectra_nw<8>(h, L, st);
  else if (spectra_smem<4>(h.nxh) <= kSpectraSmemCap) e = spectra_nw<4>(h, L, st);
  else if (spectra_smem<2>(h.nxh) <= kSpectraSmemCap) e = spectra_nw<2>(h, L, st);
  else if (spectra_smem<1>(h.nxh) <= kSpectraSmemCap) e = spectra_nw<1>(h, L, st);
  else return cudaErrorNotSupported;
  if (e != cudaSuccess) return e;
  k_mom_reduce<<<h.ny, 32, 0, st>>>(h.stat + L.part, xphys2_row_blocks(h), h.ny, h.rescale,
                                    h.stat + L.lines, h.stat + L.tr);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  switch (h.bw) {
    case 2: return stat_lines_bw<2>(h, L, st);
    case 3: return stat_lines_bw<3>(h, L, st);
    case 4: return stat_lines_bw<4>(h, L, st);
    case 5: return stat_lines_bw<5>(h, L, st);
    case 6: return stat_lines_bw<6>(h, L, st);
    case 7: return stat_lines_bw<7>(h, L, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kmm
