// wavespace2.cu - per-(kx, kz) wall-normal solves of one substep with register-window sweeps.
//
// Same mathematics as wavespace.f90:22-113 and the routines it calls, reorganised into
// ascending / descending sweeps (sweeps.cuh) so that every recurrence runs out of registers:
//   hvhg (hvhg.f90:56-159)        4 D0 solves (a3, f8, f2, f4) + D1/D2 mat-vecs -> hg, hv, ht
//   solve_t (solve_t.f90:28-201)  LU(A_t) + solve -> theta, D2 theta -> store_t
//   solve_g + solve_v_f parts 1-4 LU(A_g) + solves of rhs_g, rhs_phi and the unit wall vector
//                                 -> g, store_g, phi_p, phi_h, store_phi (partial)
//   solve_v_f parts 5-8           LU(D2 - k2 D0) + solves -> v_p, v_h, dv_p, dv_h; C1, C2
//                                 from the mirror symmetry (solve_v_f.f90:293-298)
//   solve_u_w (solve_u_w.f90:27-38)
// phi_h, v_h and their derivatives have equal real and imaginary parts (the unit wall vector is
// (p0, p0), solve_v_f.f90:142), so they are carried as one real chain.  The mean mode
// (wave00.f90:41-714) runs on three threads of an extra block, one per mean line (U, W, Theta).
// One thread owns one mode; its lines are strided by the number of modes (coalesced per warp).
#include <cuda_runtime.h>

#include "kmm_internal.h"
#include "sweeps.cuh"

namespace kmm {

namespace {

__device__ __forceinline__ double rkc(int c, int s) {
  const double t[4][3] = {{29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0},
                          {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0},
                          {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0},
                          {0.0, -17.0 / 60.0, -5.0 / 12.0}};
  return t[c - 1][s - 1];
}

struct Ws2Args {
  int ny, nxh, nz, substep;
  int64_t nmodes, ns;
  double2 *S, *RK;
  const void *P;
  double2 *zc;   // [4][ny][nm] complex scratch lines
  double2 *ec;   // [3][ny][nm]
  double *xr;    // [6][ny][nm] real scratch lines
  double *ub;    // [2BW][ny][nm] per-mode U factor
  double *w00;   // mean-mode scratch, per line thread
  const double *tabs;  // t0, t1, t2, l0, u0 (global copy)
  const double *integ;
  const double2 *vwall;
  double control_amp;
  double nu, pr, lmfxr, lmfzr, bulk_u, bulk_w, bulk_t, u_gal;
  DevScalars *dsc;
  const double *dt_ptr;
};

template <int BW>
__device__ __forceinline__ Tabs<BW> tabs_at(const double *base, int ny) {
  const int64_t tw = (int64_t)ny * (4 * BW + 1);
  Tabs<BW> t;
  t.t0 = base;
  t.t1 = base + tw;
  t.t2 = base + 2 * tw;
  t.l0 = base + 3 * tw;
  t.u0 = t.l0 + (int64_t)ny * (2 * BW + 1);
  return t;
}

template <typename PT> __device__ __forceinline__ double2 ldp(const PT *p);
template <> __device__ __forceinline__ double2 ldp<double2>(const double2 *p) { return *p; }
template <> __device__ __forceinline__ double2 ldp<float2>(const float2 *p) {
  const float2 v = *p;
  return make_double2((double)v.x, (double)v.y);
}

// A = a D0 - b D2 (Dirichlet first / last rows) as offset rows.
template <int BW>
__device__ __forceinline__ void helm_row(const Tabs<BW> &tb, int r, int n, double ca, double cb, double *out) {
  const double *r0 = trow<BW>(tb.t0, r), *r2 = trow<BW>(tb.t2, r);
  if (r == 1 || r == n) {
#pragma unroll
    for (int e = -2 * BW; e <= 2 * BW; ++e) out[e + 2 * BW] = 0.0;
    out[2 * BW] = ca * r0[0] - cb * r2[0];
    return;
  }
#pragma unroll
  for (int e = -2 * BW; e <= 2 * BW; ++e) out[e + 2 * BW] = ca * r0[e] - cb * r2[e];
}

template <int BW, typename PT>
__device__ void mode_step2(const Ws2Args &a, const Tabs<BW> &tb, int64_t m) {
  const int n = a.ny, s = a.substep;
  const int64_t nm = a.nmodes, ns = a.ns;
  const double dt = *a.dt_ptr, nu = a.nu, pr = a.pr;
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;   // set_waveno
  const double kx = kxi * a.lmfxr, kz = kzint * a.lmfzr;     // wavespace.f90:69
  const double k2 = kx * kx + kz * kz;
  const PT *P = reinterpret_cast<const PT *>(a.P) + m;
  auto prod = [&](int slot, int r) { return ldp<PT>(P + slot * ns + (int64_t)(r - 1) * nm); };
  DLine Z[4], E[3];
#pragma unroll
  for (int i = 0; i < 4; ++i) Z[i] = DLine{a.zc + i * ns + m, nm};
#pragma unroll
  for (int i = 0; i < 3; ++i) E[i] = DLine{a.ec + i * ns + m, nm};
  RLine X[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) X[i] = RLine{a.xr + i * ns + m, nm};
  DLine Su{a.S + 0 * ns + m, nm}, Sv{a.S + 1 * ns + m, nm}, Sw{a.S + 2 * ns + m, nm}, St{a.S + 3 * ns + m, nm};
  DLine Rg{a.RK + 0 * ns + m, nm}, Rp{a.RK + 1 * ns + m, nm}, Rt{a.RK + 2 * ns + m, nm};
  UBand<BW> ub{a.ub + m, nm, ns};
  auto ufix = [&](int r, int e) { return tb.u0[(r - 1) * 2 * BW + e - 1]; };
  auto uper = [&](int r, int e) { return ub.get(r, e); };

  // ---- hvhg ----------------------------------------------------------------------------
  const double kxkz = kx * kz, kx2 = kx * kx, kz2 = kz * kz;
  const double c2i = kx * kx * kx + kx * (kz * kz), c4i = (kx * kx) * kz + kz * kz * kz;
  // ascending: a3 = -kx2 f1 - 2 kxkz f5 - kz2 f3 and f8 through D0^{-1}; a1 and t7 kept
  fwd_fixed<BW, 2>(tb, n,
      [&](int r, double2 *b) {
        const double2 f1 = prod(0, r), f3 = prod(2, r), f5 = prod(4, r);
        const double2 f7 = prod(5, r), f8 = prod(6, r), f9 = prod(7, r);
        b[0] = zsub(zsub(zscale(-kx2, f1), zscale(2.0 * kxkz, f5)), zscale(kz2, f3));
        b[1] = f8;
        E[0].st(r, zadd(zscale(kxkz, zsub(f1, f3)), zscale(kz2 - kx2, f5)));  // a1
        E[2].st(r, z2(-kx * f7.y - kz * f9.y, kx * f7.x + kz * f9.x));      // t7 = i kx f7 + i kz f9
      },
      [&](int r, const double2 *z) { Z[0].st(r, z[0]); Z[1].st(r, z[1]); });
  // ascending: f2 and f4 through D0^{-1}; e_hv = i(kx^3 + kx kz^2) f2 + i(kx^2 kz + kz^3) f4
  fwd_fixed<BW, 2>(tb, n,
      [&](int r, double2 *b) {
        const double2 f2 = prod(1, r), f4 = prod(3, r);
        b[0] = f2;
        b[1] = f4;
        E[1].st(r, z2(-c2i * f2.y - c4i * f4.y, c2i * f2.x + c4i * f4.x));
      },
      [&](int r, const double2 *z) { Z[2].st(r, z[0]); Z[3].st(r, z[1]); });
  // descending: hv += D1 c(a3); ht = -(t7 + D1 c(f8))
  bwd_emit<BW, 2, 0>(n, ufix,
      [&](int r, double2 *zc, double *) { zc[0] = Z[0].ld(r); zc[1] = Z[1].ld(r); },
      [&](int q, int r, const double2 (&wc)[2][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        const double2 d1a3 = mvc<BW>(tb.t1, q, r, wc[0]), d1f8 = mvc<BW>(tb.t1, q, r, wc[1]);
        E[1].st(q, zadd(E[1].ld(q), d1a3));
        const double2 t = zadd(E[2].ld(q), d1f8);
        E[2].st(q, z2(-t.x, -t.y));
      });
  // descending: hg = a1 + D1 (i kx c(f4) - i kz c(f2)); hv += D2 (i kz c(f4) + i kx c(f2))
  bwd_emit<BW, 2, 0>(n, ufix,
      [&](int r, double2 *zc, double *) { zc[0] = Z[2].ld(r); zc[1] = Z[3].ld(r); },
      [&](int q, int r, const double2 (&wc)[2][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        const double2 d1f2 = mvc<BW>(tb.t1, q, r, wc[0]), d1f4 = mvc<BW>(tb.t1, q, r, wc[1]);
        const double2 d2f2 = mvc<BW>(tb.t2, q, r, wc[0]), d2f4 = mvc<BW>(tb.t2, q, r, wc[1]);
        const double2 g1 = z2(-(kx * d1f4.y - kz * d1f2.y), kx * d1f4.x - kz * d1f2.x);
        const double2 v2 = z2(-(kz * d2f4.y + kx * d2f2.y), kz * d2f4.x + kx * d2f2.x);
        E[0].st(q, zadd(E[0].ld(q), g1));
        E[1].st(q, zadd(E[1].ld(q), v2));
      });
  // E0 = hg, E1 = hv, E2 = ht.  Substep 1 also needs D2 D0^{-1} of the three stores.
  if (s == 1) {
    fwd_fixed<BW, 2>(tb, n, [&](int r, double2 *b) { b[0] = Rg.ld(r); b[1] = Rp.ld(r); },
                     [&](int r, const double2 *z) { Z[0].st(r, z[0]); Z[1].st(r, z[1]); });
    bwd_emit<BW, 2, 0>(n, ufix,
        [&](int r, double2 *zc, double *) { zc[0] = Z[0].ld(r); zc[1] = Z[1].ld(r); },
        [&](int q, int r, const double2 (&wc)[2][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
          Z[0].st(q, mvc<BW>(tb.t2, q, r, wc[0]));
          Z[1].st(q, mvc<BW>(tb.t2, q, r, wc[1]));
        });
    fwd_fixed<BW, 1>(tb, n, [&](int r, double2 *b) { b[0] = Rt.ld(r); },
                     [&](int r, const double2 *z) { Z[2].st(r, z[0]); });
    bwd_emit<BW, 1, 0>(n, ufix, [&](int r, double2 *zc, double *) { zc[0] = Z[2].ld(r); },
        [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
          Z[2].st(q, mvc<BW>(tb.t2, q, r, wc[0]));
        });
  }
  // RK right-hand side (solve_g.f90:84-123): rows 1 and n are the Dirichlet rows (zero)
  auto rhs = [&](DLine store, DLine h, DLine d2, double visc, int r) {
    if (r == 1 || r == n) return z2(0.0, 0.0);
    if (s == 1) {
      const double alpha = dt * rkc(1, s) * visc, gamma = dt * rkc(3, s);
      return zadd(zadd(zscale(1.0 - alpha * k2, store.ld(r)), zscale(gamma, h.ld(r))), zscale(alpha, d2.ld(r)));
    }
    return zadd(store.ld(r), zscale(dt * rkc(3, s), h.ld(r)));
  };
  // new store (solve_g.f90:138-185): zeta' h + (1 - alpha' k2) f + alpha' D2 f, or f at s = 3
  auto store_new = [&](double2 h, double2 f, double2 d2f, double visc) {
    if (s == 3) return f;
    const double alpha = dt * rkc(1, s + 1) * visc, zeta = dt * rkc(4, s + 1);
    return zadd(zadd(zscale(zeta, h), zscale(1.0 - alpha * k2, f)), zscale(alpha, d2f));
  };

  // ---- solve_t ---------------------------------------------------------------------------
  {
    const double visc = nu / pr;
    const double beta = dt * rkc(2, s) * nu / pr;
    const double dummy = 1.0 + beta * k2;
    lu_fwd<BW, 1, 0>(n, [&](int r, double *row) { helm_row<BW>(tb, r, n, dummy, beta, row); },
        [&](int r, double2 *bc, double *) { bc[0] = rhs(Rt, E[2], Z[2], visc, r); },
        [&](int r, const double2 *zc, const double *) { Z[3].st(r, zc[0]); }, ub);
    bwd_emit<BW, 1, 0>(n, uper, [&](int r, double2 *zc, double *) { zc[0] = Z[3].ld(r); },
        [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
          const double2 th = mvc<BW>(tb.t0, q, r, wc[0]), d2th = mvc<BW>(tb.t2, q, r, wc[0]);
          St.st(q, th);
          Rt.st(q, store_new(E[2].ld(q), th, d2th, visc));
        });
  }
  // ---- solve_g and solve_v_f parts 1-4 --------------------------------------------------
  {
    const double beta = dt * rkc(2, s) * nu;
    const double dummy = 1.0 + beta * k2;
    const double p0 = dummy * trow<BW>(tb.t0, 1)[0] - beta * trow<BW>(tb.t2, 1)[0];  // A_g(1,1)
    lu_fwd<BW, 2, 1>(n, [&](int r, double *row) { helm_row<BW>(tb, r, n, dummy, beta, row); },
        [&](int r, double2 *bc, double *br) {
          bc[0] = rhs(Rg, E[0], Z[0], nu, r);
          bc[1] = rhs(Rp, E[1], Z[1], nu, r);
          br[0] = (r == 1) ? p0 : 0.0;  // the unit wall vector (solve_v_f.f90:142), real part
        },
        [&](int r, const double2 *zc, const double *zr) {
          Z[0].st(r, zc[0]);
          Z[1].st(r, zc[1]);
          X[0].st(r, zr[0]);
        }, ub);
    bwd_emit<BW, 2, 1>(n, uper,
        [&](int r, double2 *zc, double *zr) { zc[0] = Z[0].ld(r); zc[1] = Z[1].ld(r); zr[0] = X[0].ld(r); },
        [&](int q, int r, const double2 (&wc)[2][2 * BW + 1], const double (&wr)[1][2 * BW + 1]) {
          const double2 g = mvc<BW>(tb.t0, q, r, wc[0]), d2g = mvc<BW>(tb.t2, q, r, wc[0]);
          const double2 pp = mvc<BW>(tb.t0, q, r, wc[1]), d2pp = mvc<BW>(tb.t2, q, r, wc[1]);
          Su.st(q, g);
          Rg.st(q, store_new(E[0].ld(q), g, d2g, nu));
          Z[2].st(q, pp);
          Rp.st(q, store_new(E[1].ld(q), pp, d2pp, nu));
          X[1].st(q, mvr<BW>(tb.t0, q, r, wr[0]));  // phi_h (real part = imaginary part)
          X[2].st(q, mvr<BW>(tb.t2, q, r, wr[0]));  // D2 phi_h
        });
  }
  // ---- solve_v_f parts 5-8: (D2 - k2 D0) v = phi with v = wall value at rows 1, n ---------
  double2 vlo = z2(0.0, 0.0), vhi = z2(0.0, 0.0);
  if (a.control_amp != 0.0) {
    vlo = a.vwall[m];
    vhi = a.vwall[nm + m];
  }
  double dvp1x = 0, dvp1y = 0, dvpnx = 0, dvpny = 0, dvh1 = 0, dvhn = 0;
  lu_fwd<BW, 1, 1>(n,
      [&](int r, double *row) {
        const double *r0 = trow<BW>(tb.t0, r), *r2 = trow<BW>(tb.t2, r);
        if (r == 1 || r == n) {
#pragma unroll
          for (int e = -2 * BW; e <= 2 * BW; ++e) row[e + 2 * BW] = 0.0;
          row[2 * BW] = r0[0];
          return;
        }
#pragma unroll
        for (int e = -2 * BW; e <= 2 * BW; ++e) row[e + 2 * BW] = -k2 * r0[e] + r2[e];
      },
      [&](int r, double2 *bc, double *br) {
        bc[0] = (r == 1) ? vlo : (r == n) ? vhi : Z[2].ld(r);
        br[0] = (r == 1 || r == n) ? 0.0 : X[1].ld(r);
      },
      [&](int r, const double2 *zc, const double *zr) { Z[3].st(r, zc[0]); X[3].st(r, zr[0]); }, ub);
  bwd_emit<BW, 1, 1>(n, uper,
      [&](int r, double2 *zc, double *zr) { zc[0] = Z[3].ld(r); zr[0] = X[3].ld(r); },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&wr)[1][2 * BW + 1]) {
        const double2 vp = mvc<BW>(tb.t0, q, r, wc[0]), dvp = mvc<BW>(tb.t1, q, r, wc[0]);
        const double vh = mvr<BW>(tb.t0, q, r, wr[0]), dvh = mvr<BW>(tb.t1, q, r, wr[0]);
        Sv.st(q, vp);
        Sw.st(q, dvp);
        X[4].st(q, vh);
        X[5].st(q, dvh);
        if (q == 1) { dvp1x = dvp.x; dvp1y = dvp.y; dvh1 = dvh; }
        if (q == n) { dvpnx = dvp.x; dvpny = dvp.y; dvhn = dvh; }
      });
  // C1, C2 (solve_v_f.f90:293-294); the homogeneous derivative is dvh * (1 + i)
  const double2 h1 = z2(dvh1, dvh1), hn = z2(dvhn, dvhn);
  const double2 d1 = z2(dvp1x, dvp1y), dn = z2(dvpnx, dvpny);
  const double2 den = zsub(zmul(h1, h1), zmul(hn, hn));
  const double2 C1 = zdiv(zsub(zmul(hn, dn), zmul(h1, d1)), den);
  const double2 C2 = zdiv(zsub(zmul(h1, dn), zmul(hn, d1)), den);
  const double2 C1c = z2(C1.x - C1.y, C1.x + C1.y), C2c = z2(C2.x - C2.y, C2.x + C2.y);  // C * (1 + i)
  double cd = 1.0, ca = 0.0;
  if (s != 3) {
    const double alpha = dt * nu * rkc(1, s + 1);
    cd = 1.0 - alpha * k2;
    ca = alpha;
  }
  const double2 kxx = z2(0.0, kx / k2), kzz = z2(0.0, kz / k2);
  for (int r = 1; r <= n; ++r) {
    const int rr = n + 1 - r;
    const double2 v = zadd(zadd(Sv.ld(r), zscale(X[4].ld(r), C1c)), zscale(X[4].ld(rr), C2c));
    const double2 dv = zsub(zadd(Sw.ld(r), zscale(X[5].ld(r), C1c)), zscale(X[5].ld(rr), C2c));
    double2 sp = Rp.ld(r);
    sp = zadd(sp, zscale(cd * X[1].ld(r), C1c));
    sp = zadd(sp, zscale(cd * X[1].ld(rr), C2c));
    if (s != 3) {
      sp = zadd(sp, zscale(ca * X[2].ld(r), C1c));
      sp = zadd(sp, zscale(ca * X[2].ld(rr), C2c));
    }
    Rp.st(r, sp);
    const double2 g = Su.ld(r);
    Su.st(r, zsub(zmul(kxx, dv), zmul(kzz, g)));  // solve_u_w.f90:27-38
    Sv.st(r, v);
    Sw.st(r, zadd(zmul(kxx, g), zmul(kzz, dv)));
  }
}

// wave00.f90 for one mean line: U (line 0: forced, Galilean shift), W (line 1: phi = 0),
// Theta (line 2: nu/pr, forced to the bulk value).  FP64 scratch per line: 4 complex lines
// and a U factor band.
template <int BW, typename PT>
__device__ void mean_line2(const Ws2Args &a, const Tabs<BW> &tb, int line) {
  const int n = a.ny, s = a.substep;
  const int64_t ns = a.ns;
  const double dt = *a.dt_ptr;
  const double visc = (line == 2) ? a.nu / a.pr : a.nu;
  const double gal = (line == 0) ? a.u_gal : 0.0;
  const double bulk = (line == 0) ? a.bulk_u : (line == 1) ? a.bulk_w : a.bulk_t;
  const int pslot = (line == 0) ? 1 : (line == 1) ? 3 : 6;   // uv, vw, v theta
  const PT *P = reinterpret_cast<const PT *>(a.P) + pslot * ns;
  DLine store{a.RK + line * ns, a.nmodes};
  DLine out{a.S + (line == 0 ? 0 : line == 1 ? 2 : 3) * ns, a.nmodes};
  const int64_t per = 4 * (int64_t)n * 2 + 2 * BW * (int64_t)n;  // doubles per line thread
  double *base = a.w00 + line * per;
  DLine Zf{reinterpret_cast<double2 *>(base), 1}, Zs{reinterpret_cast<double2 *>(base) + n, 1};
  DLine R{reinterpret_cast<double2 *>(base) + 2 * n, 1}, DF{reinterpret_cast<double2 *>(base) + 3 * n, 1};
  UBand<BW> ub{base + 8 * (int64_t)n, 1, n};
  auto ufix = [&](int r, int e) { return tb.u0[(r - 1) * 2 * BW + e - 1]; };
  // D0 solves: the flux product (and the store at substep 1)
  fwd_fixed<BW, 2>(tb, n,
      [&](int r, double2 *b) {
        b[0] = ldp<PT>(P + (int64_t)(r - 1) * a.nmodes);
        b[1] = (s == 1) ? store.ld(r) : z2(0.0, 0.0);
      },
      [&](int r, const double2 *z) { Zf.st(r, z[0]); Zs.st(r, z[1]); });
  bwd_emit<BW, 2, 0>(n, ufix,
      [&](int r, double2 *zc, double *) { zc[0] = Zf.ld(r); zc[1] = Zs.ld(r); },
      [&](int q, int r, const double2 (&wc)[2][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        const double2 d = mvc<BW>(tb.t1, q, r, wc[0]);   // d/dy of the flux
        DF.st(q, d);
        double2 b;
        const double gamma = dt * rkc(3, s);
        if (s == 1) {
          const double alpha = dt * rkc(1, s) * visc;
          b = zsub(zadd(store.ld(q), zscale(alpha, mvc<BW>(tb.t2, q, r, wc[1]))), zscale(gamma, d));
        } else {
          b = zsub(store.ld(q), zscale(gamma, d));
        }
        // wave00.f90:169-173: zero wall rows, interior real part + u_gal, imaginary part 1
        R.st(q, (q == 1 || q == n) ? z2(0.0, 0.0) : z2(b.x + gal, 1.0));
      });
  // (D0 - beta D2) c = rhs, Dirichlet rows
  const double beta = dt * rkc(2, s) * visc;
  lu_fwd<BW, 1, 0>(n, [&](int r, double *row) { helm_row<BW>(tb, r, n, 1.0, beta, row); },
      [&](int r, double2 *bc, double *) { bc[0] = R.ld(r); },
      [&](int r, const double2 *zc, const double *) { R.st(r, zc[0]); }, ub);
  double2 integral = z2(0.0, 0.0);
  {  // backward substitution storing the coefficients (the integral needs all of them)
    double2 w[2 * BW + 1];
#pragma unroll
    for (int j = 0; j <= 2 * BW; ++j) w[j] = z2(0.0, 0.0);
    for (int r = n; r >= 1; --r) {
#pragma unroll
      for (int j = 2 * BW; j >= 1; --j) w[j] = w[j - 1];
      double2 acc = R.ld(r);
#pragma unroll
      for (int e = 1; e <= 2 * BW; ++e) {
        const double u = ub.get(r, e);
        acc.x -= u * w[e].x;
        acc.y -= u * w[e].y;
      }
      w[0] = acc;
      R.st(r, acc);
    }
  }
  for (int i = 1; i <= n; ++i) integral = zadd(integral, zscale(__ldg(a.integ + i - 1), R.ld(i)));  // LABS_integration
  double phi = (bulk - 0.5 * integral.x) / (0.5 * integral.y);  // calculate_phi
  if (line == 1) phi = 0.0;                                       // wave00.f90:396
  // c = Re c + phi Im c (real); mean profile D0 c, store alpha' D2 c + profile - zeta' d
  for (int r = 1; r <= n; ++r) {
    const double2 c = R.ld(r);
    Zf.st(r, z2(c.x + phi * c.y, 0.0));
  }
  if (s == 3) {
    const double *r1 = trow<BW>(tb.t1, 1), *rn = trow<BW>(tb.t1, n);
    const double wall = r1[0] * Zf.ld(1).x + r1[1] * Zf.ld(2).x - rn[-1] * Zf.ld(n - 1).x - rn[0] * Zf.ld(n).x;
    if (line == 0) a.dsc->wall_shear_stress = 0.5 * a.nu * wall;
    if (line == 2) a.dsc->wall_theta_stress = 0.5 * a.nu / a.pr * wall;
  }
  if (line == 0) a.dsc->phi_dpdx[s - 1] = phi;
  if (line == 2) a.dsc->phi_dtdx[s - 1] = phi;
  bwd_emit<BW, 1, 0>(n, [&](int, int) { return 0.0; },
      [&](int r, double2 *zc, double *) { zc[0] = Zf.ld(r); },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        double2 prof = mvc<BW>(tb.t0, q, r, wc[0]);
        prof.x -= gal;
        out.st(q, prof);
        if (s != 3) {
          const double alpha = dt * rkc(1, s + 1) * visc, zeta = dt * rkc(4, s + 1);
          store.st(q, zsub(zadd(zscale(alpha, mvc<BW>(tb.t2, q, r, wc[0])), prof), zscale(zeta, DF.ld(q))));
        } else {
          store.st(q, prof);
        }
      });
  if (line == 1) {  // v mean = 0 (wave00.f90:462)
    DLine Sv{a.S + ns, a.nmodes};
    for (int r = 1; r <= n; ++r) Sv.st(r, z2(0.0, 0.0));
  }
}

template <int BW, typename PT>
__global__ void __launch_bounds__(128) k_wavespace2(Ws2Args a, int use_smem) {
  extern __shared__ __align__(16) double stab[];
  const int n = a.ny;
  const int64_t tot = (int64_t)n * (3 * (4 * BW + 1) + (2 * BW + 1) + 2 * BW);
  const double *tb_base = a.tabs;
  if (use_smem) {
    for (int64_t i = threadIdx.x; i < tot; i += blockDim.x) stab[i] = a.tabs[i];
    __syncthreads();
    tb_base = stab;
  }
  if (a.dsc->err) return;  // a failed dt update leaves the state untouched
  const Tabs<BW> tb = tabs_at<BW>(tb_base, n);
  if (blockIdx.x == gridDim.x - 1) {
    if (threadIdx.x < 3) mean_line2<BW, PT>(a, tb, threadIdx.x);
    return;
  }
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0 || m >= a.nmodes) return;
  mode_step2<BW, PT>(a, tb, m);
}

template <int BW>
cudaError_t ws2_bw(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  OpsOffsets off = ops_offsets(h.bw, h.ny);
  Ws2Args a;
  a.ny = h.ny;
  a.nxh = h.nxh;
  a.nz = h.nz;
  a.substep = substep;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.S = h.S;
  a.RK = h.RK;
  a.P = h.P;
  a.zc = h.zc;
  a.ec = h.ec;
  a.xr = h.xr;
  a.ub = h.ub;
  a.w00 = h.w00;
  a.tabs = h.dops + off.t0;
  a.integ = h.dops + off.integ;
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
  const size_t tab_bytes = sizeof(double) * (size_t)h.ny * (3 * (4 * BW + 1) + (2 * BW + 1) + 2 * BW);
  const int use_smem = tab_bytes <= 200 * 1024;
  const int threads = 128;
  const unsigned blocks = (unsigned)((h.nmodes + threads - 1) / threads) + 1;  // +1: mean lines
  if (h.mixed)
    k_wavespace2<BW, float2><<<blocks, threads, use_smem ? tab_bytes : 0, st>>>(a, use_smem);
  else
    k_wavespace2<BW, double2><<<blocks, threads, use_smem ? tab_bytes : 0, st>>>(a, use_smem);
  return cudaGetLastError();
}

}  // namespace

void prepare_wavespace2() {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  auto set = [&](auto kern) {
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) return;
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  };
  set(k_wavespace2<2, float2>); set(k_wavespace2<2, double2>);
  set(k_wavespace2<3, float2>); set(k_wavespace2<3, double2>);
  set(k_wavespace2<4, float2>); set(k_wavespace2<4, double2>);
  set(k_wavespace2<5, float2>); set(k_wavespace2<5, double2>);
  set(k_wavespace2<6, float2>); set(k_wavespace2<6, double2>);
  set(k_wavespace2<7, float2>); set(k_wavespace2<7, double2>);
}

cudaError_t launch_wavespace2(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  if (h.cfg.control_amp != 0.0) {
    cudaError_t e = launch_control_probe(h, st);
    if (e != cudaSuccess) return e;
  }
  switch (h.bw) {
    case 2: return ws2_bw<2>(h, substep, dt_ptr, st);
    case 3: return ws2_bw<3>(h, substep, dt_ptr, st);
    case 4: return ws2_bw<4>(h, substep, dt_ptr, st);
    case 5: return ws2_bw<5>(h, substep, dt_ptr, st);
    case 6: return ws2_bw<6>(h, substep, dt_ptr, st);
    case 7: return ws2_bw<7>(h, substep, dt_ptr, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace kmm
