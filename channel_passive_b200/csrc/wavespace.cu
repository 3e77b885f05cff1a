// wavespace.cu - the per-(kx, kz) wall-normal solves of one substep.
//
// k_wavespace restates wavespace.f90:22-113 with one thread per mode: hvhg (hvhg.f90:28-163),
// solve_g (solve_g.f90:28-201), solve_v_f (solve_v_f.f90:38-375), solve_u_w
// (solve_u_w.f90:18-42) and solve_t (solve_t.f90:28-201).  The (0,0) mode (wave00.f90:41-714)
// runs in FP64 on a dedicated extra block so it overlaps the other modes.
//
// Lines: products P[slot] (slots 0..7 = f1..f5, f7..f9), state S[0..3] = u, v, w, theta,
// stores RK[0..2]; two FP64 scratch lines per mode (buf1, buf2 of the reference) plus two
// more for solve_v_f so that phi_p / phi_h stay in FP64 whatever the product precision; the
// per-mode band D_buf lives in wband.  Mode m = kz_index * nxh + kx; element y of a line sits
// at y * nmodes + m.
#include <cuda_runtime.h>

#include "kmm_internal.h"
#include "labs.cuh"

namespace kmm {

namespace {

// RK_3_COEF(c, s), module_runge_kutta.f90:33-48.
__device__ __forceinline__ double rk3(int c, int s) {
  const double t[4][3] = {{29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0},
                          {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0},
                          {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0},
                          {0.0, -17.0 / 60.0, -5.0 / 12.0}};
  return t[c - 1][s - 1];
}

struct WsArgs {
  int ny, nxh, nz, substep;
  int64_t nmodes, ns;
  double2 *S, *RK, *wbuf, *w00;
  void *P;
  double *wband;
  const double *d0, *d1, *d2, *d0lu, *integ, *wlo, *whi;
  const float *gains;
  double2 *vwall;  // [2][nmodes] control wall velocities (bottom, top)
  double control_amp;
  double nu, pr, lmfxr, lmfzr, bulk_u, bulk_w, bulk_t, u_gal;
  DevScalars *dsc;
  const double *dt_ptr;
};

// a*D0 - b*D2 with the Dirichlet first/last rows (solve_g.f90:42-67, solve_t.f90:243-268,
// wave00.f90:58-80); a = 1 for wave00.
template <int BW>
__device__ void build_helmholtz(BandM<BW> D, BandS<BW> D0, BandS<BW> D2, double a, double b, int ny) {
  constexpr int ld = 2 * BW + 1;
  for (int i = 1; i <= ld; ++i) D.set(i, 1, 0.0);
  D.set(BW + 1, 1, a * D0.g(BW + 1, 1) - b * D2.g(BW + 1, 1));
  for (int j = 2; j <= ny - 1; ++j)
#pragma unroll
    for (int i = 1; i <= ld; ++i) D.set(i, j, a * D0.g(i, j) - b * D2.g(i, j));
  for (int i = 1; i <= ld; ++i) D.set(i, ny, 0.0);
  D.set(BW + 1, ny, a * D0.g(BW + 1, ny) - b * D2.g(BW + 1, ny));
}

template <int BW>
struct Ops {
  BandS<BW> D0, D1, D2, D0lu;
};

// hvhg.f90:56-159 in place on the product lines.  Leaves hg in u1, hv in u5, ht in u7.
template <int BW, typename PL>
__device__ void hvhg(PL u1, PL u2, PL u3, PL u4, PL u5, PL u7, PL u8, PL u9, const Ops<BW> &o,
                     double kx, double kz, int ny) {
  const double kz2 = kz * kz, kx2 = kx * kx, kxkz = kx * kz;
  const double2 ikx = z2(0.0, kx), ikz = z2(0.0, kz);
  const double2 ikx3 = z2(0.0, kx * kx * kx), ikxkz2 = z2(0.0, kx * (kz * kz));
  const double2 ikx2kz = z2(0.0, (kx * kx) * kz), ikz3 = z2(0.0, kz * kz * kz);
  for (int i = 1; i <= ny; ++i) {
    const double2 d = u1.ld(i), a3 = u3.ld(i), a5 = u5.ld(i);
    u1.st(i, zadd(zscale(kxkz, zsub(d, a3)), zscale(kz2 - kx2, a5)));
    u3.st(i, zsub(zsub(zscale(-kx2, d), zscale(2.0 * kxkz, a5)), zscale(kz2, a3)));
  }
  labs_bs<BW>(o.D0lu, u3, ny);
  labs_mat_mul<BW>(o.D1, u3, u5, ny);
  const double2 c2 = zadd(ikx3, ikxkz2), c4 = zadd(ikx2kz, ikz3);
  for (int i = 1; i <= ny; ++i) u5.st(i, zadd(zadd(u5.ld(i), zmul(c2, u2.ld(i))), zmul(c4, u4.ld(i))));
  for (int i = 1; i <= ny; ++i) {
    const double2 a2 = u2.ld(i), a4 = u4.ld(i);
    u3.st(i, zsub(zmul(ikx, a4), zmul(ikz, a2)));
    u4.st(i, zadd(zmul(ikz, a4), zmul(ikx, a2)));
  }
  labs_bs<BW>(o.D0lu, u3, ny);
  labs_mat_mul<BW>(o.D1, u3, u2, ny);
  labs_bs<BW>(o.D0lu, u4, ny);
  labs_mat_mul<BW>(o.D2, u4, u3, ny);
  for (int i = 1; i <= ny; ++i) {
    u5.st(i, zadd(u5.ld(i), u3.ld(i)));
    u1.st(i, zadd(u1.ld(i), u2.ld(i)));
  }
  for (int i = 1; i <= ny; ++i) u7.st(i, zadd(zmul(ikx, u7.ld(i)), zmul(ikz, u9.ld(i))));
  labs_bs<BW>(o.D0lu, u8, ny);
  labs_mat_mul<BW>(o.D1, u8, u9, ny);
  for (int i = 1; i <= ny; ++i) {
    const double2 v = zadd(u7.ld(i), u9.ld(i));
    u7.st(i, z2(-v.x, -v.y));
  }
}

// solve_g.f90:28-201 (pr = 0) and solve_t.f90:28-201 (pr > 0): h in hin, new field to out.
template <int BW, typename HL>
__device__ void solve_helm(HL hin, DLine out, DLine store, DLine buf1, DLine buf2, BandM<BW> Dbuf,
                           const Ops<BW> &o, double kx, double kz, double nu, double pr, int s,
                           double dt, int ny) {
  const double k2 = kx * kx + kz * kz;
  auto visc = [&](double c) { return pr > 0.0 ? dt * c * nu / pr : dt * c * nu; };
  const double beta = visc(rk3(2, s));
  double dummy = 1.0 + beta * k2;
  build_helmholtz<BW>(Dbuf, o.D0, o.D2, dummy, beta, ny);
  labs_lu<BW>(Dbuf, ny);
  if (s == 1) {
    const double alpha = visc(rk3(1, s)), gamma = dt * rk3(3, s);
    dummy = 1.0 - alpha * k2;
    for (int i = 1; i <= ny; ++i) buf1.st(i, zadd(zscale(dummy, store.ld(i)), zscale(gamma, hin.ld(i))));
    labs_bs<BW>(o.D0lu, store, ny);
    labs_mat_mul<BW>(o.D2, store, buf2, ny);
    for (int i = 1; i <= ny; ++i) buf1.st(i, zadd(buf1.ld(i), zscale(alpha, buf2.ld(i))));
  } else {
    const double gamma = dt * rk3(3, s);
    for (int i = 1; i <= ny; ++i) buf1.st(i, zadd(store.ld(i), zscale(gamma, hin.ld(i))));
  }
  buf1.st(1, z2(0.0, 0.0));
  buf1.st(ny, z2(0.0, 0.0));
  if (s != 3) {
    const double zeta = dt * rk3(4, s + 1);
    for (int i = 1; i <= ny; ++i) store.st(i, zscale(zeta, hin.ld(i)));
  }
  labs_bs<BW>(Dbuf, buf1, ny);
  labs_mat_mul<BW>(o.D0, buf1, out, ny);
  labs_mat_mul<BW>(o.D2, buf1, buf2, ny);
  if (s != 3) {
    const double alpha = visc(rk3(1, s + 1));
    dummy = 1.0 - alpha * k2;
    for (int i = 1; i <= ny; ++i)
      store.st(i, zadd(zadd(store.ld(i), zscale(dummy, out.ld(i))), zscale(alpha, buf2.ld(i))));
  } else {
    for (int i = 1; i <= ny; ++i) store.st(i, out.ld(i));
  }
}

// solve_v_f.f90:38-375.  hv (FP64 copy of h_v) is consumed; v and dv receive v and dv/dy.
template <int BW>
__device__ void solve_v_f(DLine v, DLine dv, DLine hv, DLine store_phi, DLine buf1, DLine buf2,
                          DLine buf3, BandM<BW> Dbuf, const Ops<BW> &o, double kx, double kz,
                          double nu, int s, double dt, double2 vwall_lo, double2 vwall_hi, int ny) {
  const double k2 = kx * kx + kz * kz;
  // Part 1
  if (s == 1) {
    const double alpha = dt * rk3(1, s) * nu, gamma = dt * rk3(3, s);
    const double dummy = 1.0 - alpha * k2;
    for (int i = 1; i <= ny; ++i) buf1.st(i, zadd(zscale(dummy, store_phi.ld(i)), zscale(gamma, hv.ld(i))));
    labs_bs<BW>(o.D0lu, store_phi, ny);
    labs_mat_mul<BW>(o.D2, store_phi, buf2, ny);
    for (int i = 1; i <= ny; ++i) buf1.st(i, zadd(buf1.ld(i), zscale(alpha, buf2.ld(i))));
  } else {
    const double gamma = dt * rk3(3, s);
    for (int i = 1; i <= ny; ++i) buf1.st(i, zadd(store_phi.ld(i), zscale(gamma, hv.ld(i))));
  }
  buf1.st(1, z2(0.0, 0.0));
  buf1.st(ny, z2(0.0, 0.0));
  // Part 2
  if (s != 3) {
    const double zeta = dt * rk3(4, s + 1);
    for (int i = 1; i <= ny; ++i) store_phi.st(i, zscale(zeta, hv.ld(i)));
  }
  // Part 3 (solve_g's factored matrix)
  const double p0 = Dbuf.g(BW + 1, 1);
  buf2.st(1, z2(p0, p0));
  for (int i = 2; i <= ny; ++i) buf2.st(i, z2(0.0, 0.0));
  labs_bs<BW>(Dbuf, buf1, ny);
  labs_bs<BW>(Dbuf, buf2, ny);
  labs_mat_mul<BW>(o.D0, buf1, hv, ny);
  labs_mat_mul<BW>(o.D0, buf2, buf3, ny);
  labs_mat_mul<BW>(o.D2, buf1, dv, ny);
  // Part 4
  if (s != 3) {
    const double alpha = dt * nu * rk3(1, s + 1);
    const double dummy = 1.0 - alpha * k2;
    for (int i = 1; i <= ny; ++i)
      store_phi.st(i, zadd(zadd(store_phi.ld(i), zscale(dummy, hv.ld(i))), zscale(alpha, dv.ld(i))));
  } else {
    for (int i = 1; i <= ny; ++i) store_phi.st(i, hv.ld(i));
  }
  // Part 5: D2 - k2 D0 with D0 Dirichlet rows
  {
    constexpr int ld = 2 * BW + 1;
    for (int i = 1; i <= ld; ++i) Dbuf.set(i, 1, 0.0);
    Dbuf.set(BW + 1, 1, o.D0.g(BW + 1, 1));
    for (int j = 2; j <= ny - 1; ++j)
#pragma unroll
      for (int i = 1; i <= ld; ++i) Dbuf.set(i, j, -k2 * o.D0.g(i, j) + o.D2.g(i, j));
    for (int i = 1; i <= ld; ++i) Dbuf.set(i, ny, 0.0);
    Dbuf.set(BW + 1, ny, o.D0.g(BW + 1, ny));
    labs_lu<BW>(Dbuf, ny);
  }
  // Part 6 (the wall values are the opposition-control hook, 0 without control)
  hv.st(1, vwall_lo);
  hv.st(ny, vwall_hi);
  labs_bs<BW>(Dbuf, hv, ny);
  for (int i = 1; i <= ny; ++i) buf1.st(i, buf3.ld(i));
  buf1.st(1, z2(0.0, 0.0));
  buf1.st(ny, z2(0.0, 0.0));
  labs_bs<BW>(Dbuf, buf1, ny);
  labs_mat_mul<BW>(o.D0, hv, v, ny);
  labs_mat_mul<BW>(o.D1, hv, dv, ny);
  labs_mat_mul<BW>(o.D1, buf1, hv, ny);
  const double2 h1 = hv.ld(1), hn = hv.ld(ny), d1 = dv.ld(1), dn = dv.ld(ny);
  const double2 den = zsub(zmul(h1, h1), zmul(hn, hn));
  const double2 C1 = zdiv(zsub(zmul(hn, dn), zmul(h1, d1)), den);
  const double2 C2 = zdiv(zsub(zmul(h1, dn), zmul(hn, d1)), den);
  for (int i = 1; i <= ny; ++i)
    dv.st(i, zsub(zadd(dv.ld(i), zmul(C1, hv.ld(i))), zmul(C2, hv.ld(ny + 1 - i))));
  // Part 7
  labs_mat_mul<BW>(o.D2, buf2, hv, ny);
  if (s != 3) {
    const double alpha = dt * nu * rk3(1, s + 1);
    const double dummy = 1.0 - alpha * k2;
    const double2 c1d = zscale(dummy, C1), c2d = zscale(dummy, C2);
    const double2 c1a = zscale(alpha, C1), c2a = zscale(alpha, C2);
    for (int i = 1; i <= ny; ++i) {
      double2 acc = zadd(store_phi.ld(i), zmul(c1d, buf3.ld(i)));
      acc = zadd(acc, zmul(c2d, buf3.ld(ny + 1 - i)));
      acc = zadd(acc, zmul(c1a, hv.ld(i)));
      acc = zadd(acc, zmul(c2a, hv.ld(ny + 1 - i)));
      store_phi.st(i, acc);
    }
  } else {
    for (int i = 1; i <= ny; ++i)
      store_phi.st(i, zadd(zadd(store_phi.ld(i), zmul(C1, buf3.ld(i))), zmul(C2, buf3.ld(ny + 1 - i))));
  }
  // Part 8
  labs_mat_mul<BW>(o.D0, buf1, hv, ny);
  for (int i = 1; i <= ny; ++i)
    v.st(i, zadd(zadd(v.ld(i), zmul(C1, hv.ld(i))), zmul(C2, hv.ld(ny + 1 - i))));
}

// solve_u_w.f90:18-42 in place: g -> u, f -> w.
__device__ void solve_u_w(DLine g, DLine f, double kx, double kz, int ny) {
  const double den = kx * kx + kz * kz;
  const double2 kxx = z2(0.0, kx / den), kzz = z2(0.0, kz / den);
  for (int i = 1; i <= ny; ++i) {
    const double2 gi = g.ld(i), fi = f.ld(i);
    g.st(i, zsub(zmul(kxx, fi), zmul(kzz, gi)));
    f.st(i, zadd(zmul(kxx, gi), zmul(kzz, fi)));
  }
}

template <typename PT> __device__ __forceinline__ Line<PT> pline(const WsArgs &a, int slot, int64_t m) {
  return Line<PT>{reinterpret_cast<PT *>(a.P) + slot * a.ns + m, a.nmodes};
}
__device__ __forceinline__ DLine dline(double2 *base, int64_t off, int64_t m, int64_t stride) {
  return DLine{base + off + m, stride};
}

template <int BW, typename PT>
__device__ void mode_step(const WsArgs &a, const Ops<BW> &o, int64_t m) {
  const int ny = a.ny, s = a.substep;
  const double dt = *a.dt_ptr;
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;   // set_waveno
  const double kx = kxi * a.lmfxr, kz = kzint * a.lmfzr;     // wavespace.f90:69
  DLine Su = dline(a.S, 0 * a.ns, m, a.nmodes), Sv = dline(a.S, 1 * a.ns, m, a.nmodes);
  DLine Sw = dline(a.S, 2 * a.ns, m, a.nmodes), St = dline(a.S, 3 * a.ns, m, a.nmodes);
  DLine Rg = dline(a.RK, 0 * a.ns, m, a.nmodes), Rp = dline(a.RK, 1 * a.ns, m, a.nmodes);
  DLine Rt = dline(a.RK, 2 * a.ns, m, a.nmodes);
  DLine b1 = dline(a.wbuf, 0 * a.ns, m, a.nmodes), b2 = dline(a.wbuf, 1 * a.ns, m, a.nmodes);
  DLine b3 = dline(a.wbuf, 2 * a.ns, m, a.nmodes), hvd = dline(a.wbuf, 3 * a.ns, m, a.nmodes);
  BandM<BW> Dbuf{a.wband + m, a.nmodes};
  // opposition-control wall values from k_control_probe (zero without control)
  double2 vlo = z2(0.0, 0.0), vhi = z2(0.0, 0.0);
  if (a.control_amp != 0.0) {
    vlo = a.vwall[m];
    vhi = a.vwall[a.nmodes + m];
  }
  Line<PT> u1 = pline<PT>(a, 0, m), u2 = pline<PT>(a, 1, m), u3 = pline<PT>(a, 2, m),
           u4 = pline<PT>(a, 3, m), u5 = pline<PT>(a, 4, m), u7 = pline<PT>(a, 5, m),
           u8 = pline<PT>(a, 6, m), u9 = pline<PT>(a, 7, m);
  hvhg<BW>(u1, u2, u3, u4, u5, u7, u8, u9, o, kx, kz, ny);
  // g: hg (u1) -> Su
  solve_helm<BW>(u1, Su, Rg, b1, b2, Dbuf, o, kx, kz, a.nu, 0.0, s, dt, ny);
  // v, dv/dy: hv (u5) in FP64
  for (int i = 1; i <= ny; ++i) hvd.st(i, u5.ld(i));
  solve_v_f<BW>(Sv, Sw, hvd, Rp, b1, b2, b3, Dbuf, o, kx, kz, a.nu, s, dt, vlo, vhi, ny);
  solve_u_w(Su, Sw, kx, kz, ny);
  // theta: ht (u7) -> St
  solve_helm<BW>(u7, St, Rt, b1, b2, Dbuf, o, kx, kz, a.nu, a.pr, s, dt, ny);
}

// wave00.f90:41-685 for the mean mode, one thread, FP64 scratch lines w00[0..5].
template <int BW, typename PT>
__device__ void wave00(const WsArgs &a, const Ops<BW> &o) {
  const int ny = a.ny, s = a.substep;
  const double dt = *a.dt_ptr, nu = a.nu, pr = a.pr;
  const int64_t m = 0;
  DLine Su = dline(a.S, 0 * a.ns, m, a.nmodes), Sv = dline(a.S, 1 * a.ns, m, a.nmodes);
  DLine Sw = dline(a.S, 2 * a.ns, m, a.nmodes), St = dline(a.S, 3 * a.ns, m, a.nmodes);
  DLine R1 = dline(a.RK, 0 * a.ns, m, a.nmodes), R2 = dline(a.RK, 1 * a.ns, m, a.nmodes);
  DLine R3 = dline(a.RK, 2 * a.ns, m, a.nmodes);
  DLine uv{a.w00 + 0 * ny, 1}, vw{a.w00 + 1 * ny, 1}, vt{a.w00 + 2 * ny, 1};
  DLine dflux{a.w00 + 3 * ny, 1}, buf1{a.w00 + 4 * ny, 1}, tmp{a.w00 + 5 * ny, 1};
  BandM<BW> Dbuf{a.wband + m, a.nmodes};
  {
    Line<PT> p2 = pline<PT>(a, 1, m), p4 = pline<PT>(a, 3, m), p8 = pline<PT>(a, 6, m);
    for (int i = 1; i <= ny; ++i) {
      uv.st(i, p2.ld(i));
      vw.st(i, p4.ld(i));
      vt.st(i, p8.ld(i));
    }
  }
  auto wall_grad = [&](DLine c) {  // wave00.f90:210-211 with LABS_D1_B
    return o.D1.g(BW + 1, 1) * c.ld(1).x + o.D1.g(BW + 2, 1) * c.ld(2).x -
           o.D1.g(BW, ny) * c.ld(ny - 1).x - o.D1.g(BW + 1, ny) * c.ld(ny).x;
  };
  // One mean line: U (visc = nu, gal = u_gal, forced), W (unforced), Theta (nu/pr, forced).
  auto mean_line = [&](DLine store, DLine flux, DLine out, double visc, double bulk, double gal,
                       bool forced, double &phi_out) {
    build_helmholtz<BW>(Dbuf, o.D0, o.D2, 1.0, dt * rk3(2, s) * visc, ny);
    labs_lu<BW>(Dbuf, ny);
    if (s == 1) {
      for (int i = 1; i <= ny; ++i) tmp.st(i, store.ld(i));
      labs_bs<BW>(o.D0lu, tmp, ny);
      labs_bs<BW>(o.D0lu, flux, ny);
      labs_mat_mul<BW>(o.D2, tmp, buf1, ny);
      labs_mat_mul<BW>(o.D1, flux, dflux, ny);
      const double alpha = dt * rk3(1, s) * visc, gamma = dt * rk3(3, s);
      for (int i = 2; i <= ny; ++i)
        buf1.st(i, zsub(zadd(store.ld(i), zscale(alpha, buf1.ld(i))), zscale(gamma, dflux.ld(i))));
    } else {
      labs_bs<BW>(o.D0lu, flux, ny);
      labs_mat_mul<BW>(o.D1, flux, dflux, ny);
      const double gamma = dt * rk3(3, s);
      for (int i = 2; i <= ny; ++i) buf1.st(i, zsub(store.ld(i), zscale(gamma, dflux.ld(i))));
    }
    buf1.st(1, z2(0.0, 0.0));
    for (int i = 2; i <= ny - 1; ++i) buf1.st(i, z2(buf1.ld(i).x + gal, 1.0));
    buf1.st(ny, z2(0.0, 0.0));
    labs_bs<BW>(Dbuf, buf1, ny);
    double2 integral = z2(0.0, 0.0);  // LABS_integration, module_labs.f90:401-413
    for (int i = 1; i <= ny; ++i) integral = zadd(integral, zscale(__ldg(a.integ + i - 1), buf1.ld(i)));
    double phi = (bulk - 0.5 * integral.x) / (0.5 * integral.y);  // calculate_phi
    if (!forced) phi = 0.0;
    for (int i = 1; i <= ny; ++i) {
      const double2 b = buf1.ld(i);
      buf1.st(i, z2(b.x + phi * b.y, 0.0));
    }
    labs_mat_mul<BW>(o.D0, buf1, out, ny);
    phi_out = phi;
  };
  auto mean_store = [&](DLine store, DLine out) {
    if (s != 3) {
      labs_mat_mul<BW>(o.D2, buf1, store, ny);
      return true;
    }
    for (int i = 1; i <= ny; ++i) store.st(i, out.ld(i));
    return false;
  };
  double phi;
  // U
  mean_line(R1, uv, Su, nu, a.bulk_u, a.u_gal, true, phi);
  a.dsc->phi_dpdx[s - 1] = phi;
  if (s == 3) a.dsc->wall_shear_stress = 0.5 * nu * wall_grad(buf1);
  for (int i = 1; i <= ny; ++i) Su.st(i, z2(Su.ld(i).x - a.u_gal, Su.ld(i).y));
  if (mean_store(R1, Su)) {
    const double alpha = dt * rk3(1, s + 1) * nu, zeta = dt * rk3(4, s + 1);
    for (int i = 1; i <= ny; ++i)
      R1.st(i, zsub(zadd(zscale(alpha, R1.ld(i)), Su.ld(i)), zscale(zeta, dflux.ld(i))));
  }
  // W (wave00.f90:298-443; phi forced to 0 at :396)
  mean_line(R2, vw, Sw, nu, a.bulk_w, 0.0, false, phi);
  if (mean_store(R2, Sw)) {
    const double alpha = dt * rk3(1, s + 1) * nu, zeta = dt * rk3(4, s + 1);
    for (int i = 1; i <= ny; ++i)
      R2.st(i, zsub(zadd(zscale(alpha, R2.ld(i)), Sw.ld(i)), zscale(zeta, dflux.ld(i))));
  }
  for (int i = 1; i <= ny; ++i) Sv.st(i, z2(0.0, 0.0));  // wave00.f90:462
  // Theta (wave00.f90:473-667)
  const double visc_t = nu / pr;
  mean_line(R3, vt, St, visc_t, a.bulk_t, 0.0, true, phi);
  a.dsc->phi_dtdx[s - 1] = phi;
  if (s == 3) a.dsc->wall_theta_stress = 0.5 * nu / pr * wall_grad(buf1);
  if (mean_store(R3, St)) {
    const double alpha = dt * rk3(1, s + 1) * nu / pr, zeta = dt * rk3(4, s + 1);
    for (int i = 1; i <= ny; ++i)
      R3.st(i, zsub(zadd(zscale(alpha, R3.ld(i)), St.ld(i)), zscale(zeta, dflux.ld(i))));
  }
}

// Opposition control, the build's extension at the wall rows of the v Poisson solve
// (solve_v_f.f90:251-257, where the reference's commented lines read vold).  The reference's
// vold is field 10, v after the physical round trip (dft_x_realspace.f90:123): x_to_y zeroes
// the kz Nyquist row and the c2r keeps only the Hermitian part of the kx = 0 plane, so the
// same projection is applied to the v of the substep's start.  v(y_d) = w . v with the
// precomputed weights w = D0^{-T} B(y_d); the wall value is A * gain(kx, kz) * v(y_d).
// Runs before k_wavespace, which overwrites v.
__global__ void k_control_probe(WsArgs a) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes) return;
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  double2 sl = z2(0.0, 0.0), sh = z2(0.0, 0.0);
  if (kzi != a.nz / 2 && m != 0) {
    auto probe = [&](int64_t mm, double2 &pl, double2 &ph) {
      DLine line = dline(a.S, 1 * a.ns, mm, a.nmodes);
      pl = z2(0.0, 0.0);
      ph = z2(0.0, 0.0);
      for (int i = 1; i <= a.ny; ++i) {
        const double2 vi = line.ld(i);
        pl = zadd(pl, zscale(__ldg(a.wlo + i - 1), vi));
        ph = zadd(ph, zscale(__ldg(a.whi + i - 1), vi));
      }
    };
    probe(m, sl, sh);
    if (kxi == 0) {  // (v(kz) + conj v(-kz)) / 2
      double2 pl, ph;
      probe((int64_t)((a.nz - kzi) % a.nz) * a.nxh, pl, ph);
      sl = z2(0.5 * (sl.x + pl.x), 0.5 * (sl.y - pl.y));
      sh = z2(0.5 * (sh.x + ph.x), 0.5 * (sh.y - ph.y));
    }
    const double gmul = a.control_amp * (a.gains ? (double)__ldg(a.gains + m) : 1.0);
    sl = zscale(gmul, sl);
    sh = zscale(gmul, sh);
  }
  a.vwall[m] = sl;
  a.vwall[a.nmodes + m] = sh;
}

template <int BW, typename PT>
__global__ void __launch_bounds__(128) k_wavespace(WsArgs a) {
  Ops<BW> o{BandS<BW>{a.d0}, BandS<BW>{a.d1}, BandS<BW>{a.d2}, BandS<BW>{a.d0lu}};
  if (a.dsc->err) return;  // a failed dt update leaves the state untouched
  if (blockIdx.x == gridDim.x - 1) {
    if (threadIdx.x == 0) wave00<BW, PT>(a, o);
    return;
  }
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0 || m >= a.nmodes) return;
  mode_step<BW, PT>(a, o, m);
}

// set_initial_data_uvw, initial_step.f90:139-179.
template <int BW>
__global__ void k_init_stores(WsArgs a) {
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
  DLine c = dline(a.wbuf, 0, m, a.nmodes);
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

WsArgs make_args(Handle &h, int substep, const double *dt_ptr) {
  WsArgs a;
  OpsOffsets off = ops_offsets(h.bw, h.ny);
  a.ny = h.ny;
  a.nxh = h.nxh;
  a.nz = h.nz;
  a.substep = substep;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.S = h.S;
  a.RK = h.RK;
  a.wbuf = h.wbuf;
  a.w00 = h.wbuf + 4 * h.ns;
  a.P = h.P;
  a.wband = h.wband;
  a.d0 = h.dops + off.d0;
  a.d1 = h.dops + off.d1;
  a.d2 = h.dops + off.d2;
  a.d0lu = h.dops + off.d0lu;
  a.integ = h.dops + off.integ;
  a.wlo = h.dops + off.wlo;
  a.whi = h.dops + off.whi;
  a.gains = h.gains;
  a.vwall = h.vwall;
  a.control_amp = h.cfg.control_amp;
  a.nu = h.cfg.nu;
  a.pr = h.cfg.pr;
  a.lmfxr = h.lmfxr;
  a.lmfzr = h.lmfzr;
  a.bulk_u = h.cfg.bulk_vel_u;
  a.bulk_w = h.cfg.bulk_vel_w;
  a.bulk_t = h.cfg.bulk_t;
  a.u_gal = h.cfg.u_gal;
  a.dsc = h.dsc;
  a.dt_ptr = dt_ptr ? dt_ptr : &h.dsc->dt;
  return a;
}

template <int BW>
cudaError_t wavespace_bw(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  WsArgs a = make_args(h, substep, dt_ptr);
  const int threads = 128;
  const unsigned blocks = (unsigned)((h.nmodes + threads - 1) / threads) + 1;  // +1: wave00 block
  if (h.cfg.control_amp != 0.0)
    k_control_probe<<<(unsigned)((h.nmodes + threads - 1) / threads), threads, 0, st>>>(a);
  if (h.mixed) k_wavespace<BW, float2><<<blocks, threads, 0, st>>>(a);
  else k_wavespace<BW, double2><<<blocks, threads, 0, st>>>(a);
  return cudaGetLastError();
}

template <int BW>
cudaError_t init_bw(Handle &h, cudaStream_t st) {
  WsArgs a = make_args(h, 1, nullptr);
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

template <int BW> struct WsRun {
  static cudaError_t run(Handle &h, int s, const double *dt, cudaStream_t st) { return wavespace_bw<BW>(h, s, dt, st); }
};
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

cudaError_t launch_control_probe(Handle &h, cudaStream_t st) {
  WsArgs a = make_args(h, 1, nullptr);
  const int threads = 128;
  k_control_probe<<<(unsigned)((h.nmodes + threads - 1) / threads), threads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_wavespace(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  return dispatch_bw<WsRun>(h.bw, h, substep, dt_ptr, st);
}
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
