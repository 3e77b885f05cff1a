// routines.cu - the reference's per-mode routines as batched device entry points, with their
// argument lists (hvhg.f90:28, solve_g.f90:28, solve_t.f90:28, solve_v_f.f90:38-39,
// solve_u_w.f90:18).  One thread per (kx, kz) mode; each runs the routine's statement sequence on
// its own lines through the reference-order LABS routines of labs.cuh, with the caller's buffers
// as the routine's scratch (buf1, buf2, buf3, D_buf), exactly as the Fortran passes them.  The
// module globals the routines read (RK_SUBSTEP, dt, RK_3_COEF, RK_STEP = 3) arrive as arguments.
//
// These are the drop-in's building blocks and its unit-test surface; the time step itself runs
// the fused role-per-warp kernels of wavespace_split.cu.
//
// Line layout: value y (1-based) of mode m at [(y - 1) * nmodes + m] (mode fastest, so a warp's
// accesses are contiguous).  D_buf: one band per mode, entry (r, j) at
// [((j - 1) * (2bw + 1) + r - 1) * nmodes + m].
#include <cuda_runtime.h>

#include <string>

#include "kmm_internal.h"
#include "labs.cuh"

namespace kmm {
namespace {

// RK3 coefficients alpha, beta, gamma, zeta per substep (module_runge_kutta.f90:34-45)
__constant__ double c_rk3[4][3] = {{29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0},
                                   {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0},
                                   {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0},
                                   {0.0, -17.0 / 60.0, -5.0 / 12.0}};
__device__ __forceinline__ double rk3c(int c, int s) { return c_rk3[c - 1][s - 1]; }
constexpr int kRkStep = 3;

struct RoutineArgs {
  int ny, nmodes, substep;
  double dt, nu, pr;
  double2 *l[10];             // the routine's line arguments, in its argument order
  const double *d0lu, *d0, *d1, *d2;
  double *dbuf;
  const double *kx, *kz;
  const double2 *vwall;       // solve_v_f: [2][nmodes] wall values, or null (zero walls)
};

__device__ __forceinline__ DLine line(const RoutineArgs &a, int i, int m) { return DLine{a.l[i] + m, a.nmodes}; }

// A (2bw+1, ny) band per mode, filled like the reference fills D_buf.
template <int BW>
__device__ __forceinline__ void fill_dirichlet(BandM<BW> D, BandS<BW> P, BandS<BW> Q, double cp, double cq,
                                               double wall_p, double wall_q, int n) {
  // rows 1 and ny: only the diagonal, wall_p P + wall_q Q; interior: cp P + cq Q
  for (int i = 1; i <= 2 * BW + 1; ++i) {
    D.set(i, 1, 0.0);
    D.set(i, n, 0.0);
  }
  D.set(BW + 1, 1, wall_p * P.g(BW + 1, 1) + wall_q * Q.g(BW + 1, 1));
  for (int j = 2; j <= n - 1; ++j)
    for (int i = 1; i <= 2 * BW + 1; ++i) D.set(i, j, cp * P.g(i, j) + cq * Q.g(i, j));
  D.set(BW + 1, n, wall_p * P.g(BW + 1, n) + wall_q * Q.g(BW + 1, n));
}

// hvhg.f90:28-163 (arguments u1 u2 u3 u4 u5 u7 u8 u9 = lines 0..7)
template <int BW>
__global__ void __launch_bounds__(128) k_ref_hvhg(RoutineArgs a) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes) return;
  const int n = a.ny;
  const DLine u1 = line(a, 0, m), u2 = line(a, 1, m), u3 = line(a, 2, m), u4 = line(a, 3, m);
  const DLine u5 = line(a, 4, m), u7 = line(a, 5, m), u8 = line(a, 6, m), u9 = line(a, 7, m);
  const BandS<BW> D0lu{a.d0lu}, D1{a.d1}, D2{a.d2};
  const double kx = a.kx[m], kz = a.kz[m];
  const double kz2 = kz * kz, kx2 = kx * kx, kxkz = kx * kz;
  // ci*kx**3 etc. are purely imaginary: i c times z = (-c z.y, c z.x)
  auto imul = [](double c, double2 z) { return z2(-c * z.y, c * z.x); };
  const double ikx3 = kx * kx * kx, ikxkz2 = kx * (kz * kz), ikx2kz = (kx * kx) * kz, ikz3 = kz * kz * kz;
  for (int i = 1; i <= n; ++i) {
    const double2 dummy = u1.ld(i);
    u1.st(i, zadd(zscale(kxkz, zsub(u1.ld(i), u3.ld(i))), zscale(kz2 - kx2, u5.ld(i))));
    u3.st(i, zsub(zsub(zscale(-kx2, dummy), zscale(2.0 * kxkz, u5.ld(i))), zscale(kz2, u3.ld(i))));
  }
  labs_bs<BW>(D0lu, u3, n);
  labs_mat_mul<BW>(D1, u3, u5, n);
  for (int i = 1; i <= n; ++i)
    u5.st(i, zadd(zadd(u5.ld(i), imul(ikx3 + ikxkz2, u2.ld(i))), imul(ikx2kz + ikz3, u4.ld(i))));
  for (int i = 1; i <= n; ++i) {
    const double2 a3 = zsub(imul(kx, u4.ld(i)), imul(kz, u2.ld(i)));
    const double2 a4 = zadd(imul(kz, u4.ld(i)), imul(kx, u2.ld(i)));
    u3.st(i, a3);
    u4.st(i, a4);
  }
  labs_bs<BW>(D0lu, u3, n);
  labs_mat_mul<BW>(D1, u3, u2, n);
  labs_bs<BW>(D0lu, u4, n);
  labs_mat_mul<BW>(D2, u4, u3, n);
  for (int i = 1; i <= n; ++i) {
    u5.st(i, zadd(u5.ld(i), u3.ld(i)));
    u1.st(i, zadd(u1.ld(i), u2.ld(i)));
  }
  for (int i = 1; i <= n; ++i) u7.st(i, zadd(imul(kx, u7.ld(i)), imul(kz, u9.ld(i))));
  labs_bs<BW>(D0lu, u8, n);
  labs_mat_mul<BW>(D1, u8, u9, n);
  for (int i = 1; i <= n; ++i) {
    const double2 t = zadd(u7.ld(i), u9.ld(i));
    u7.st(i, z2(-t.x, -t.y));
  }
}

// solve_g.f90:28-201 (IS_T = false) and solve_t.f90:28-201 (IS_T = true, nu/pr):
// lines 0..3 = u1 (or u7), store, buf1, buf2.
template <int BW, bool IS_T>
__global__ void __launch_bounds__(128) k_ref_solve_gt(RoutineArgs a) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes) return;
  const int n = a.ny, s = a.substep;
  const DLine u1 = line(a, 0, m), store = line(a, 1, m), buf1 = line(a, 2, m), buf2 = line(a, 3, m);
  const BandS<BW> D0lu{a.d0lu}, D0{a.d0}, D2{a.d2};
  const BandM<BW> Db{a.dbuf + m, a.nmodes};
  const double kx = a.kx[m], kz = a.kz[m], k2 = kx * kx + kz * kz, dt = a.dt;
  auto visc = [&](int c, int ss) {
    const double v = dt * rk3c(c, ss) * a.nu;
    return IS_T ? v / a.pr : v;
  };
  const double beta = visc(2, s);
  double dummy = 1.0 + beta * k2;
  fill_dirichlet<BW>(Db, D0, D2, dummy, -beta, dummy, -beta, n);
  labs_lu<BW>(Db, n);
  if (s == 1) {
    const double alpha = visc(1, s), gamma = dt * rk3c(3, s);
    dummy = 1.0 - alpha * k2;
    for (int i = 1; i <= n; ++i) buf1.st(i, zadd(zscale(dummy, store.ld(i)), zscale(gamma, u1.ld(i))));
    labs_bs<BW>(D0lu, store, n);
    labs_mat_mul<BW>(D2, store, buf2, n);
    for (int i = 1; i <= n; ++i) buf1.st(i, zadd(buf1.ld(i), zscale(alpha, buf2.ld(i))));
  } else {
    const double gamma = dt * rk3c(3, s);
    for (int i = 1; i <= n; ++i) buf1.st(i, zadd(store.ld(i), zscale(gamma, u1.ld(i))));
  }
  buf1.st(1, z2(0.0, 0.0));
  buf1.st(n, z2(0.0, 0.0));
  if (s != kRkStep) {
    const double zeta = dt * rk3c(4, s + 1);
    for (int i = 1; i <= n; ++i) store.st(i, zscale(zeta, u1.ld(i)));
  }
  labs_bs<BW>(Db, buf1, n);
  labs_mat_mul<BW>(D0, buf1, u1, n);
  labs_mat_mul<BW>(D2, buf1, buf2, n);
  if (s != kRkStep) {
    const double alpha = visc(1, s + 1);
    dummy = 1.0 - alpha * k2;
    for (int i = 1; i <= n; ++i)
      store.st(i, zadd(zadd(store.ld(i), zscale(dummy, u1.ld(i))), zscale(alpha, buf2.ld(i))));
  } else {
    for (int i = 1; i <= n; ++i) store.st(i, u1.ld(i));
  }
}

// solve_v_f.f90:38-375: lines 0..7 = v, dv, hv, store_phi, buf1, buf2, buf3, vold; D_buf holds
// solve_g's factored operator on entry and the v operator's on exit.  The wall values of the v
// solve (solve_v_f.f90:251-252) come from vwall when given, else zero (the reference).
template <int BW>
__global__ void __launch_bounds__(128) k_ref_solve_v_f(RoutineArgs a) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes) return;
  const int n = a.ny, s = a.substep;
  const DLine v = line(a, 0, m), dv = line(a, 1, m), hv = line(a, 2, m), sp = line(a, 3, m);
  const DLine buf1 = line(a, 4, m), buf2 = line(a, 5, m), buf3 = line(a, 6, m);
  const BandS<BW> D0lu{a.d0lu}, D0{a.d0}, D1{a.d1}, D2{a.d2};
  const BandM<BW> Db{a.dbuf + m, a.nmodes};
  const double kx = a.kx[m], kz = a.kz[m], k2 = kx * kx + kz * kz, dt = a.dt, nu = a.nu;
  // part 1: the RK right-hand side of phi
  if (s == 1) {
    const double alpha = dt * rk3c(1, s) * nu, gamma = dt * rk3c(3, s), dummy = 1.0 - alpha * k2;
    for (int i = 1; i <= n; ++i) buf1.st(i, zadd(zscale(dummy, sp.ld(i)), zscale(gamma, hv.ld(i))));
    labs_bs<BW>(D0lu, sp, n);
    labs_mat_mul<BW>(D2, sp, buf2, n);
    for (int i = 1; i <= n; ++i) buf1.st(i, zadd(buf1.ld(i), zscale(alpha, buf2.ld(i))));
  } else {
    const double gamma = dt * rk3c(3, s);
    for (int i = 1; i <= n; ++i) buf1.st(i, zadd(sp.ld(i), zscale(gamma, hv.ld(i))));
  }
  buf1.st(1, z2(0.0, 0.0));
  buf1.st(n, z2(0.0, 0.0));
  // part 2
  if (s != kRkStep) {
    const double zeta = dt * rk3c(4, s + 1);
    for (int i = 1; i <= n; ++i) sp.st(i, zscale(zeta, hv.ld(i)));
  }
  // part 3: phi_p and the unit-wall phi_h with solve_g's factors
  const double p0 = Db.g(BW + 1, 1);
  buf2.st(1, z2(p0, p0));
  for (int i = 2; i <= n; ++i) buf2.st(i, z2(0.0, 0.0));
  labs_bs<BW>(Db, buf1, n);
  labs_bs<BW>(Db, buf2, n);
  labs_mat_mul<BW>(D0, buf1, hv, n);
  labs_mat_mul<BW>(D0, buf2, buf3, n);
  labs_mat_mul<BW>(D2, buf1, dv, n);
  // part 4
  if (s != kRkStep) {
    const double alpha = dt * nu * rk3c(1, s + 1), dummy = 1.0 - alpha * k2;
    for (int i = 1; i <= n; ++i) sp.st(i, zadd(zadd(sp.ld(i), zscale(dummy, hv.ld(i))), zscale(alpha, dv.ld(i))));
  } else {
    for (int i = 1; i <= n; ++i) sp.st(i, hv.ld(i));
  }
  // part 5: D2 - k^2 D0 with D0 at the wall rows
  {
    const BandS<BW> Dz{a.d0};
    for (int i = 1; i <= 2 * BW + 1; ++i) {
      Db.set(i, 1, 0.0);
      Db.set(i, n, 0.0);
    }
    Db.set(BW + 1, 1, Dz.g(BW + 1, 1));
    for (int j = 2; j <= n - 1; ++j)
      for (int i = 1; i <= 2 * BW + 1; ++i) Db.set(i, j, -k2 * D0.g(i, j) + D2.g(i, j));
    Db.set(BW + 1, n, Dz.g(BW + 1, n));
  }
  labs_lu<BW>(Db, n);
  // part 6: v_p with the wall values, v_h from phi_h with zero walls
  hv.st(1, a.vwall ? a.vwall[m] : z2(0.0, 0.0));
  hv.st(n, a.vwall ? a.vwall[a.nmodes + m] : z2(0.0, 0.0));
  labs_bs<BW>(Db, hv, n);
  for (int i = 1; i <= n; ++i) buf1.st(i, buf3.ld(i));
  buf1.st(1, z2(0.0, 0.0));
  buf1.st(n, z2(0.0, 0.0));
  labs_bs<BW>(Db, buf1, n);
  labs_mat_mul<BW>(D0, hv, v, n);
  labs_mat_mul<BW>(D1, hv, dv, n);
  labs_mat_mul<BW>(D1, buf1, hv, n);
  const double2 h1 = hv.ld(1), hn = hv.ld(n), d1 = dv.ld(1), dn = dv.ld(n);
  const double2 den = zsub(zmul(h1, h1), zmul(hn, hn));
  const double2 C1 = zdiv(zsub(zmul(hn, dn), zmul(h1, d1)), den);
  const double2 C2 = zdiv(zsub(zmul(h1, dn), zmul(hn, d1)), den);
  for (int i = 1; i <= n; ++i) dv.st(i, zsub(zadd(dv.ld(i), zmul(C1, hv.ld(i))), zmul(C2, hv.ld(n + 1 - i))));
  // part 7
  labs_mat_mul<BW>(D2, buf2, hv, n);
  if (s != kRkStep) {
    const double alpha = dt * nu * rk3c(1, s + 1), dummy = 1.0 - alpha * k2;
    const double2 C1d = zscale(dummy, C1), C2d = zscale(dummy, C2), C1a = zscale(alpha, C1), C2a = zscale(alpha, C2);
    for (int i = 1; i <= n; ++i) {
      double2 t = sp.ld(i);
      t = zadd(t, zmul(C1d, buf3.ld(i)));
      t = zadd(t, zmul(C2d, buf3.ld(n + 1 - i)));
      t = zadd(t, zmul(C1a, hv.ld(i)));
      t = zadd(t, zmul(C2a, hv.ld(n + 1 - i)));
      sp.st(i, t);
    }
  } else {
    for (int i = 1; i <= n; ++i)
      sp.st(i, zadd(zadd(sp.ld(i), zmul(C1, buf3.ld(i))), zmul(C2, buf3.ld(n + 1 - i))));
  }
  // part 8
  labs_mat_mul<BW>(D0, buf1, hv, n);
  for (int i = 1; i <= n; ++i) v.st(i, zadd(zadd(v.ld(i), zmul(C1, hv.ld(i))), zmul(C2, hv.ld(n + 1 - i))));
}

// solve_u_w.f90:18-42: g -> u, f -> w in place (lines 0, 1).
__global__ void __launch_bounds__(128) k_ref_solve_u_w(RoutineArgs a) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes) return;
  const DLine g = line(a, 0, m), f = line(a, 1, m);
  const double kx = a.kx[m], kz = a.kz[m], k2 = kx * kx + kz * kz;
  const double2 kxx = z2(0.0, kx / k2), kzz = z2(0.0, kz / k2);
  for (int i = 1; i <= a.ny; ++i) {
    const double2 gi = g.ld(i), fi = f.ld(i);
    const double2 dxg = zmul(kxx, gi), dzg = zmul(kzz, gi), dxf = zmul(kxx, fi), dzf = zmul(kzz, fi);
    g.st(i, zsub(dxf, dzg));
    f.st(i, zadd(dxg, dzf));
  }
}

enum Routine { R_HVHG, R_SOLVE_G, R_SOLVE_T, R_SOLVE_V_F };

template <int BW>
cudaError_t launch_routine_bw(Routine r, const RoutineArgs &a, cudaStream_t st) {
  const unsigned blocks = (unsigned)((a.nmodes + 127) / 128);
  switch (r) {
    case R_HVHG: k_ref_hvhg<BW><<<blocks, 128, 0, st>>>(a); break;
    case R_SOLVE_G: k_ref_solve_gt<BW, false><<<blocks, 128, 0, st>>>(a); break;
    case R_SOLVE_T: k_ref_solve_gt<BW, true><<<blocks, 128, 0, st>>>(a); break;
    default: k_ref_solve_v_f<BW><<<blocks, 128, 0, st>>>(a); break;
  }
  return cudaGetLastError();
}

int run(Handle &h, Routine r, const RoutineArgs &a, void *stream, const char *name) {
  DeviceGuard dg(h.cfg.device);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e;
  switch (h.bw) {
    case 2: e = launch_routine_bw<2>(r, a, st); break;
    case 3: e = launch_routine_bw<3>(r, a, st); break;
    case 4: e = launch_routine_bw<4>(r, a, st); break;
    case 5: e = launch_routine_bw<5>(r, a, st); break;
    case 6: e = launch_routine_bw<6>(r, a, st); break;
    default: e = launch_routine_bw<7>(r, a, st); break;
  }
  if (e != cudaSuccess) {
    set_error(std::string(name) + ": launch failed: " + cudaGetErrorString(e));
    return KMM_ERR_CUDA;
  }
  return KMM_OK;
}

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int bad(const char *name, const char *why) {
  set_error(std::string(name) + ": " + why);
  return KMM_ERR_ARG;
}

// Common checks: every line pointer non-null and 16-byte aligned (complex doubles), bands and
// wavenumbers non-null, substep in 1..3, ny equal to the handle's.
int check_common(const Handle &h, const char *name, double *const *lines, int nl, const void *const *ptrs, int np,
                 int nmodes, int ny, int substep) {
  if (nmodes <= 0) return bad(name, "nmodes must be positive");
  if (ny != h.ny) return bad(name, "ny differs from the handle's");
  if (substep < 1 || substep > 3) return bad(name, "rk_substep must be 1, 2 or 3");
  for (int i = 0; i < nl; ++i)
    if (!lines[i] || !aligned16(lines[i])) return bad(name, "null or misaligned line argument (16-byte complex)");
  for (int i = 0; i < np; ++i)
    if (!ptrs[i]) return bad(name, "null band or wavenumber argument");
  return KMM_OK;
}

RoutineArgs base_args(const Handle &h, int nmodes, int substep, double dt) {
  RoutineArgs a{};
  a.ny = h.ny;
  a.nmodes = nmodes;
  a.substep = substep;
  a.dt = dt;
  return a;
}

}  // namespace
}  // namespace kmm

using namespace kmm;

extern "C" {

int kmm_dev_hvhg(kmm_handle *hh, double *u1, double *u2, double *u3, double *u4, double *u5, double *u7, double *u8,
                 double *u9, const double *D0_lu, const double *D1, const double *D2, const double *kx,
                 const double *kz, int64_t nx32, int64_t nz32, int nmodes, void *stream) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  (void)nx32;
  (void)nz32;  // declared by hvhg.f90:28, not read by its body
  double *lines[8] = {u1, u2, u3, u4, u5, u7, u8, u9};
  const void *ptrs[5] = {D0_lu, D1, D2, kx, kz};
  int rc = check_common(h, "kmm_dev_hvhg", lines, 8, ptrs, 5, nmodes, h.ny, 1);
  if (rc) return rc;
  RoutineArgs a = base_args(h, nmodes, 1, 0.0);
  for (int i = 0; i < 8; ++i) a.l[i] = reinterpret_cast<double2 *>(lines[i]);
  a.d0lu = D0_lu;
  a.d1 = D1;
  a.d2 = D2;
  a.kx = kx;
  a.kz = kz;
  return run(h, R_HVHG, a, stream, "kmm_dev_hvhg");
}

static int solve_gt(kmm_handle *hh, bool is_t, const char *name, double *u, double *store, double *buf1,
                    double *buf2, const double *D0_lu, const double *D0, const double *D2, double *D_buf,
                    const double *kx, const double *kz, double nu, double pr, int ny, int rk_substep, double dt,
                    int nmodes, void *stream) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  double *lines[4] = {u, store, buf1, buf2};
  const void *ptrs[6] = {D0_lu, D0, D2, D_buf, kx, kz};
  int rc = check_common(h, name, lines, 4, ptrs, 6, nmodes, ny, rk_substep);
  if (rc) return rc;
  if (!(nu > 0.0) || (is_t && !(pr > 0.0))) return bad(name, "nu and pr must be positive");
  RoutineArgs a = base_args(h, nmodes, rk_substep, dt);
  for (int i = 0; i < 4; ++i) a.l[i] = reinterpret_cast<double2 *>(lines[i]);
  a.d0lu = D0_lu;
  a.d0 = D0;
  a.d2 = D2;
  a.dbuf = D_buf;
  a.kx = kx;
  a.kz = kz;
  a.nu = nu;
  a.pr = pr;
  return run(h, is_t ? R_SOLVE_T : R_SOLVE_G, a, stream, name);
}

int kmm_dev_solve_g(kmm_handle *hh, double *u1, double *store_g, double *buf1, double *buf2, const double *D0_lu,
                    const double *D0, const double *D2, double *D_buf, const double *kx, const double *kz, double nu,
                    int ny, int rk_substep, double dt, int nmodes, void *stream) {
  return solve_gt(hh, false, "kmm_dev_solve_g", u1, store_g, buf1, buf2, D0_lu, D0, D2, D_buf, kx, kz, nu, 1.0, ny,
                  rk_substep, dt, nmodes, stream);
}

int kmm_dev_solve_t(kmm_handle *hh, double *u7, double *store_t, double *buf1, double *buf2, const double *D0_lu,
                    const double *D0, const double *D2, double *D_buf, const double *kx, const double *kz, double nu,
                    double pr, int ny, int rk_substep, double dt, int nmodes, void *stream) {
  return solve_gt(hh, true, "kmm_dev_solve_t", u7, store_t, buf1, buf2, D0_lu, D0, D2, D_buf, kx, kz, nu, pr, ny,
                  rk_substep, dt, nmodes, stream);
}

int kmm_dev_solve_v_f(kmm_handle *hh, double *v, double *dv, double *hv, double *store_phi, double *buf1,
                      double *buf2, double *buf3, const double *vold, const double *D0_lu, const double *D0,
                      const double *D1, const double *D2, double *D_buf, const double *kx, const double *kz,
                      double nu, int ny, int rk_substep, double dt, const double *vwall, int nmodes, void *stream) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  (void)vold;  // read only by the reference's commented control lines (solve_v_f.f90:253-257)
  double *lines[7] = {v, dv, hv, store_phi, buf1, buf2, buf3};
  const void *ptrs[7] = {D0_lu, D0, D1, D2, D_buf, kx, kz};
  int rc = check_common(h, "kmm_dev_solve_v_f", lines, 7, ptrs, 7, nmodes, ny, rk_substep);
  if (rc) return rc;
  if (vwall && !aligned16(vwall)) return bad("kmm_dev_solve_v_f", "misaligned vwall");
  if (!(nu > 0.0)) return bad("kmm_dev_solve_v_f", "nu must be positive");
  RoutineArgs a = base_args(h, nmodes, rk_substep, dt);
  for (int i = 0; i < 7; ++i) a.l[i] = reinterpret_cast<double2 *>(lines[i]);
  a.d0lu = D0_lu;
  a.d0 = D0;
  a.d1 = D1;
  a.d2 = D2;
  a.dbuf = D_buf;
  a.kx = kx;
  a.kz = kz;
  a.nu = nu;
  a.vwall = reinterpret_cast<const double2 *>(vwall);
  return run(h, R_SOLVE_V_F, a, stream, "kmm_dev_solve_v_f");
}

int kmm_dev_solve_u_w(kmm_handle *hh, double *g, double *f, const double *kx, const double *kz, int nmodes,
                      void *stream) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  double *lines[2] = {g, f};
  const void *ptrs[2] = {kx, kz};
  int rc = check_common(h, "kmm_dev_solve_u_w", lines, 2, ptrs, 2, nmodes, h.ny, 1);
  if (rc) return rc;
  DeviceGuard dg(h.cfg.device);
  RoutineArgs a = base_args(h, nmodes, 1, 0.0);
  a.l[0] = reinterpret_cast<double2 *>(g);
  a.l[1] = reinterpret_cast<double2 *>(f);
  a.kx = kx;
  a.kz = kz;
  k_ref_solve_u_w<<<(unsigned)((nmodes + 127) / 128), 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(std::string("kmm_dev_solve_u_w: launch failed: ") + cudaGetErrorString(e));
    return KMM_ERR_CUDA;
  }
  return KMM_OK;
}

}  // extern "C"
