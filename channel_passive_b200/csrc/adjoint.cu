// adjoint.cu - discrete adjoint of the RK3 step for gradients of the opposition control.
//
// No counterpart in the reference (its control is commented out, solve_v_f.f90:253-257).  The
// control sets v at the wall rows of the v solve to v_wall(m) = A g(m) P(w . v_m), with A the
// amplitude, g(m) a gain per (kx, kz) mode, w the evaluation weights of the detection planes and P
// the projection the physical round trip applies to v (kz Nyquist row zeroed, Hermitian part on
// kx = 0).  The objective is J = (w_tau / N) sum_n tau_w(n) + (w_q / N) sum_n q_w(n) over N steps
// at a fixed time step, tau_w and q_w the substep-3 wall shear stress and wall scalar flux
// (wave00.f90:210-211, 621-622).  kmm_adjoint_forward runs the N steps keeping one checkpoint
// (state and RK stores) per step; kmm_adjoint_backward walks the steps backwards: it restores a
// step's checkpoint, recomputes substeps 1 and 2 to recover each substep's starting state, and
// applies the transposes of the three substeps in reverse order.
//
// The transpose of one substep, with <a, b> = Re sum conj(a) b over the stored coefficients:
//   wavespace^T   per (kx, kz) mode, three role warps per 32 modes (k_adj_modes): the routines of
//                 wavespace.f90 in reverse (solve_u_w, solve_t, solve_v_f, solve_g, hvhg), every
//                 band solve A^{-1} becoming A^{-T} and every band product M becoming M^T, both on
//                 the packed LU of fixed_bandec (module_labs.f90:3487-3636);
//                 the (0,0) lines of wave00 (k_adj_mean), the constant-flux phi entering through its
//                 affine dependence on the particular solution;
//                 the control probe and its projection (k_adj_probe), which also accumulates
//                 dJ/d(A g(m));
//   x_to_y^T      the z inverse transform (y_to_x) times rescale;
//   products^T    the x-pass transpose at the substep's starting state (k_xadj2, transforms2.cu);
//   y_to_x^T      the z forward transform (x_to_y) without rescale.
// Every piece is FP64; the adjoint needs an FP64 handle with a fixed time step.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "kmm_internal.h"
#include "labs.cuh"
#include "sweeps.cuh"

namespace kmm {

struct Adjoint {
  int nsteps = 0, capacity = 0;
  double w_tau = 1.0, w_q = 0.0;
  std::vector<double2 *> ck;  // per step: S [4 ns] then RK [3 ns]
  double2 *fin = nullptr;     // the state at the end of the trajectory [7 ns]
  double2 *sb = nullptr;      // substep starting states [3][4 ns]
  double2 *lS = nullptr, *lRK = nullptr, *lS0 = nullptr, *lRK0 = nullptr;  // [4 ns], [3 ns], [4 ns], [3 ns]
  double2 *lP = nullptr;      // [8 ns]
  double2 *lmid = nullptr;    // [8 nm]
  double2 *tmp = nullptr;     // [4 ns]
  double2 *X = nullptr;       // per-mode scratch lines [kAdjLines ns]
  // per substep, for the dt in cdt: the factored bands of theta's, g's (= phi's) and v's operators
  // [3][3][(2bw+1) ns] and the state-independent influence lines of solve_v_f [3][6 ns]
  double *B = nullptr;
  double2 *Xc = nullptr;
  double cdt[3] = {0.0, 0.0, 0.0};
  bool cvalid[3] = {false, false, false};
  double2 *ml = nullptr;      // mean-line scratch [3][8][ny] complex
  double *mb = nullptr;       // mean-line bands [3][(2bw+1) ny]
  double2 *lvw = nullptr;     // [2][nmodes] lambda of the wall values
  double *G = nullptr;        // [nmodes] sum of Re(conj(lambda v_wall) P(w . v)) per mode
  double *J = nullptr;        // [1] accumulated objective
};

namespace {

constexpr int kAdjLines = 18;

#define ADJ_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      set_error(std::string("adjoint: CUDA error: ") + cudaGetErrorString(e_) + " at " #call); \
      return KMM_ERR_CUDA;                                                                \
    }                                                                                     \
  } while (0)

// RK3 coefficients alpha, beta, gamma, zeta (module_runge_kutta.f90:34-45)
__constant__ double c_rka[4][3] = {{29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0},
                                   {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0},
                                   {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0},
                                   {0.0, -17.0 / 60.0, -5.0 / 12.0}};
__device__ __forceinline__ double rka(int c, int s) { return c_rka[c - 1][s - 1]; }

__device__ __forceinline__ double2 zcm(double2 a, double2 b) {  // conj(a) * b
  return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 zi(double c, double2 z) { return make_double2(-c * z.y, c * z.x); }  // (i c) z

// Packed-band row (1-based) holding matrix entry (j, c) in the near-boundary packing of
// LABS_full_to_band (module_labs.f90:301-328); c must lie in row j's profile row_lo..row_hi.
template <int BW>
__device__ __forceinline__ int ppos(int j, int c, int n) {
  if (j <= BW) return c <= BW + j ? BW + c - j + 1 : 2 * BW + 2 - c;
  if (j <= n - BW) return c - j + BW + 1;
  return c >= j - BW ? BW + c - j + 1 : n - c + 1;
}
template <int BW, typename B>
__device__ __forceinline__ double ent(const B &A, int j, int c, int n) {
  return A.g(ppos<BW>(j, c, n), j);
}

// y = s A^T x (+ y when acc): y_c = s sum_j A(j, c) x_j over the rows j whose profile holds c.
template <int BW, typename B, typename XT, typename YT>
__device__ void mm_t(const B &A, XT x, YT y, int n, double s = 1.0, bool acc = false) {
  for (int c = 1; c <= n; ++c) {
    double2 t = make_double2(0.0, 0.0);
    const int j0 = c - 2 * BW > 1 ? c - 2 * BW : 1, j1 = c + 2 * BW < n ? c + 2 * BW : n;
    for (int j = j0; j <= j1; ++j) {
      if (c < row_lo<BW>(j, n) || c > row_hi<BW>(j, n)) continue;
      t = zadd(t, zscale(ent<BW>(A, j, c, n), x.ld(j)));
    }
    t = zscale(s, t);
    y.st(c, acc ? zadd(y.ld(c), t) : t);
  }
}

// A^T x = b in place, A's packed Crout factors (L with the pivots, unit U): U^T z = b ascending,
// then L^T x = z descending.  The last 2BW results of each sweep stay in a register window (the
// recurrence would otherwise wait on its own stores), taken in the same order of j as a loop over
// the stored line, so the sums are the same.
template <int BW, typename B, typename LT>
__device__ void bs_t(const B &A, LT b, int n) {
  constexpr int W = 2 * BW;
  double2 win[W];  // ascending: win[k] = z_{c-W+k}; descending: win[k] = x_{c+1+k}
#pragma unroll
  for (int k = 0; k < W; ++k) win[k] = make_double2(0.0, 0.0);
  for (int c = 1; c <= n; ++c) {
    double2 t = b.ld(c);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const int j = c - W + k;
      if (j >= 1 && c <= row_hi<BW>(j, n)) t = zsub(t, zscale(ent<BW>(A, j, c, n), win[k]));
    }
#pragma unroll
    for (int k = 0; k < W - 1; ++k) win[k] = win[k + 1];
    win[W - 1] = t;
    b.st(c, t);
  }
#pragma unroll
  for (int k = 0; k < W; ++k) win[k] = make_double2(0.0, 0.0);
  for (int c = n; c >= 1; --c) {
    double2 t = b.ld(c);
#pragma unroll
    for (int k = 0; k < W; ++k) {
      const int j = c + 1 + k;
      if (j <= n && c >= row_lo<BW>(j, n)) t = zsub(t, zscale(ent<BW>(A, j, c, n), win[k]));
    }
    const double d = ent<BW>(A, c, c, n);
    t = make_double2(t.x / d, t.y / d);
#pragma unroll
    for (int k = W - 1; k >= 1; --k) win[k] = win[k - 1];
    win[0] = t;
    b.st(c, t);
  }
}

// ca P + cb Q with the first and last rows reduced to wa P + wb Q on the diagonal.
template <int BW>
__device__ void fill_rows(BandM<BW> D, BandS<BW> P, BandS<BW> Q, double ca, double cb, double wa, double wb,
                          int n) {
  for (int i = 1; i <= 2 * BW + 1; ++i) {
    D.set(i, 1, 0.0);
    D.set(i, n, 0.0);
  }
  D.set(BW + 1, 1, wa * P.g(BW + 1, 1) + wb * Q.g(BW + 1, 1));
  for (int j = 2; j <= n - 1; ++j)
    for (int i = 1; i <= 2 * BW + 1; ++i) D.set(i, j, ca * P.g(i, j) + cb * Q.g(i, j));
  D.set(BW + 1, n, wa * P.g(BW + 1, n) + wb * Q.g(BW + 1, n));
}

__device__ __forceinline__ void zero_walls(DLine l, int n) {
  l.st(1, make_double2(0.0, 0.0));
  l.st(n, make_double2(0.0, 0.0));
}

struct AdjArgs {
  int ny, nxh, nz, substep;
  int64_t nmodes, ns;
  double dt, nu, pr, lmfxr, lmfzr;
  const double *d0, *d1, *d2, *d0lu, *integ;
  const double2 *lS, *lRK;   // lambda of the substep's outputs (u, v, w, theta; the three stores)
  double2 *lP, *lRK0, *lvw;  // out: lambda of the products, of the starting stores, of the wall values
  double2 *X;
  double *B;                 // this substep's factored bands (k_adj_factor)
  double2 *Xc;               // this substep's influence lines c2, D0 c2, D2 c2, ch, D1 ch, D0 ch
  double2 *ml;
  double *mb;
  double w_tau, w_q;         // objective weights of this substep (zero unless substep 3)
};

// The transpose of solve_g.f90:28-201 (VT = nu) or solve_t.f90:28-201 (VT = nu / pr) for one
// mode: lf, lst = lambda of the new field and store; lh (out), lstore (out); A = the operator's
// factored band (k_adj_factor); t0, t1 scratch lines.
template <int BW>
__device__ void helm_t(const AdjArgs &a, double visc, double k2, DLine lf, DLine lst, DLine lh, DLine lstore,
                       BandM<BW> A, DLine t0, DLine t1) {
  const int n = a.ny, s = a.substep;
  const double dt = a.dt;
  const BandS<BW> D0{a.d0}, D2{a.d2}, D0lu{a.d0lu};
  const double alpha = dt * rka(1, s) * visc, gamma = dt * rka(3, s);
  if (s != 3) {
    const double a1 = dt * rka(1, s + 1) * visc, z1 = dt * rka(4, s + 1);
    for (int y = 1; y <= n; ++y) {
      lh.st(y, zscale(z1, lst.ld(y)));
      t0.st(y, zadd(lf.ld(y), zscale(1.0 - a1 * k2, lst.ld(y))));
    }
    mm_t<BW>(D0, t0, t1, n);
    mm_t<BW>(D2, lst, t1, n, a1, true);
  } else {
    for (int y = 1; y <= n; ++y) {
      lh.st(y, make_double2(0.0, 0.0));
      t0.st(y, zadd(lf.ld(y), lst.ld(y)));
    }
    mm_t<BW>(D0, t0, t1, n);
  }
  bs_t<BW>(A, t1, n);  // t1 = lambda of the right-hand side
  zero_walls(t1, n);
  if (s == 1) {
    mm_t<BW>(D2, t1, t0, n);
    bs_t<BW>(D0lu, t0, n);
    for (int y = 1; y <= n; ++y) lstore.st(y, zadd(zscale(1.0 - alpha * k2, t1.ld(y)), zscale(alpha, t0.ld(y))));
  } else {
    for (int y = 1; y <= n; ++y) lstore.st(y, t1.ld(y));
  }
  for (int y = 1; y <= n; ++y) lh.st(y, zadd(lh.ld(y), zscale(gamma, t1.ld(y))));
}

// The factored bands and state-independent lines of one substep, per mode (modes other than
// (0,0)): they depend on dt and k^2 alone, and the adjoint runs at a fixed time step, so the
// backward sweep makes them once per substep (Adjoint::cdt) instead of at every step.  Same
// routines as before in the same order, so the same numbers.
template <int BW>
__global__ void __launch_bounds__(64) k_adj_factor(AdjArgs a) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0 || m >= a.nmodes) return;
  const int n = a.ny, s = a.substep;
  const int64_t nm = a.nmodes, ns = a.ns;
  const double dt = a.dt;
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;
  const double kx = kxi * a.lmfxr, kz = kzint * a.lmfzr, k2 = kx * kx + kz * kz;
  const BandS<BW> D0{a.d0}, D1{a.d1}, D2{a.d2};
  const int64_t bsz = (int64_t)(2 * BW + 1) * n * nm;
  const BandM<BW> At{a.B + m, nm}, Ag{a.B + bsz + m, nm}, Vb{a.B + 2 * bsz + m, nm};
  {  // theta's operator (solve_t.f90:42-71)
    const double visc = a.nu / a.pr, beta = dt * rka(2, s) * visc;
    fill_rows<BW>(At, D0, D2, 1.0 + beta * k2, -beta, 1.0 + beta * k2, -beta, n);
    labs_lu<BW>(At, n);
  }
  const double beta = dt * rka(2, s) * a.nu;
  fill_rows<BW>(Ag, D0, D2, 1.0 + beta * k2, -beta, 1.0 + beta * k2, -beta, n);
  labs_lu<BW>(Ag, n);
  fill_rows<BW>(Vb, D2, D0, 1.0, -k2, 0.0, 1.0, n);  // D2 - k^2 D0, D0 at the walls
  labs_lu<BW>(Vb, n);
  // c2 = Ag^-1 (p0 + i p0) e_1, buf3 = D0 c2, d2h = D2 c2, ch = V^-1 buf3 (walls zero),
  // hh = D1 ch, hm = D0 ch
  auto C = [&](int i) { return DLine{a.Xc + i * ns + m, nm}; };
  const DLine c2 = C(0), buf3 = C(1), d2h = C(2), ch = C(3), hh = C(4), hm = C(5);
  const double p0 = Ag.g(BW + 1, 1);
  for (int y = 1; y <= n; ++y) c2.st(y, y == 1 ? make_double2(p0, p0) : make_double2(0.0, 0.0));
  labs_bs<BW>(Ag, c2, n);
  labs_mat_mul<BW>(D0, c2, buf3, n);
  labs_mat_mul<BW>(D2, c2, d2h, n);
  for (int y = 1; y <= n; ++y) ch.st(y, (y == 1 || y == n) ? make_double2(0.0, 0.0) : buf3.ld(y));
  labs_bs<BW>(Vb, ch, n);
  labs_mat_mul<BW>(D1, ch, hh, n);
  labs_mat_mul<BW>(D0, ch, hm, n);
}

// Per-mode transpose of wavespace (modes other than (0,0)), three warps per 32 modes.  Once the
// bands are factored (k_adj_factor), solve_t^T (role 0), solve_v_f^T (role 1) and solve_g^T
// (role 2) are independent; after a block barrier hvhg^T's four D0 solves are spread over the
// roles, and after a second one each role forms some of the products' lambda.  Each role runs
// the per-mode arithmetic of the single-thread order, so the results are the same numbers.
constexpr int kAdjRoles = 3;

template <int BW>
__global__ void __launch_bounds__(32 * kAdjRoles) k_adj_modes(AdjArgs a) {
  const int role = threadIdx.x / 32;
  const int64_t m = (int64_t)blockIdx.x * 32 + (threadIdx.x % 32);
  const bool live = m != 0 && m < a.nmodes;  // every thread reaches the barriers
  const int n = a.ny, s = a.substep;
  const int64_t nm = a.nmodes, ns = a.ns;
  const double dt = a.dt;
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;
  const double kx = kxi * a.lmfxr, kz = kzint * a.lmfzr, k2 = kx * kx + kz * kz;
  const BandS<BW> D0{a.d0}, D1{a.d1}, D2{a.d2}, D0lu{a.d0lu};
  auto X = [&](int i) { return DLine{a.X + i * ns + m, nm}; };
  auto in = [&](const double2 *p, int i) { return DLine{const_cast<double2 *>(p) + i * ns + m, nm}; };
  const int64_t bsz = (int64_t)(2 * BW + 1) * n * nm;
  const BandM<BW> At{a.B + m, nm}, Ag{a.B + bsz + m, nm}, Vb{a.B + 2 * bsz + m, nm};
  const DLine lu = in(a.lS, 0), lv = in(a.lS, 1), lw = in(a.lS, 2), lth = in(a.lS, 3);
  const DLine lsg = in(a.lRK, 0), lsp = in(a.lRK, 1), lst = in(a.lRK, 2);
  const DLine og = in(a.lRK0, 0), op = in(a.lRK0, 1), ot = in(a.lRK0, 2);

  if (live) {
    // solve_u_w^T: lambda g -> X0 (role 2), lambda dv -> X1 (role 1)
    const double kxx = kx / k2, kzz = kz / k2;
    if (role == 0) {
      // solve_t^T: lambda h_theta -> X2, lambda of the theta store -> ot
      helm_t<BW>(a, a.nu / a.pr, k2, lth, lst, X(2), ot, At, X(16), X(17));
    } else if (role == 1) {
      for (int y = 1; y <= n; ++y) X(1).st(y, zsub(zi(-kxx, lu.ld(y)), zi(kzz, lw.ld(y))));
      // solve_v_f^T (Ag, Vb and the state-independent lines from k_adj_factor)
      {
        const double nu = a.nu;
        const double alpha = dt * rka(1, s) * nu, gamma = dt * rka(3, s);
        auto C = [&](int i) { return DLine{a.Xc + i * ns + m, nm}; };
        const DLine buf3 = C(1), d2h = C(2), hh = C(4), hm = C(5);
        const double2 h1 = hh.ld(1), hn = hh.ld(n);
        const double2 den = zsub(zmul(h1, h1), zmul(hn, hn));
        const double q = s != 3 ? 1.0 - dt * rka(1, s + 1) * nu * k2 : 1.0;
        const double a1 = s != 3 ? dt * rka(1, s + 1) * nu : 0.0;
        const DLine ldv = X(1);
        double2 lC1 = make_double2(0.0, 0.0), lC2 = make_double2(0.0, 0.0);
        for (int y = 1; y <= n; ++y) {
          const int r = n + 1 - y;
          const double2 vy = lv.ld(y), py = lsp.ld(y), dy = ldv.ld(y);
          lC1 = zadd(lC1, zcm(hm.ld(y), vy));
          lC2 = zadd(lC2, zcm(hm.ld(r), vy));
          lC1 = zadd(lC1, zcm(zadd(zscale(q, buf3.ld(y)), zscale(a1, d2h.ld(y))), py));
          lC2 = zadd(lC2, zcm(zadd(zscale(q, buf3.ld(r)), zscale(a1, d2h.ld(r))), py));
          lC1 = zadd(lC1, zcm(hh.ld(y), dy));
          lC2 = zsub(lC2, zcm(hh.ld(r), dy));
        }
        // dv0 (the particular solution's dv/dy): its wall values set C1 and C2
        const DLine ldv0 = X(11);
        for (int y = 1; y <= n; ++y) ldv0.st(y, ldv.ld(y));
        const double2 hnd = zdiv(hn, den), h1d = zdiv(h1, den);
        ldv0.st(n, zadd(ldv0.ld(n), zadd(zcm(hnd, lC1), zcm(h1d, lC2))));
        ldv0.st(1, zsub(ldv0.ld(1), zadd(zcm(h1d, lC1), zcm(hnd, lC2))));
        // v0 = D0 cv, dv0 = D1 cv, cv = V^-1 r
        const DLine lr = X(12);
        mm_t<BW>(D0, lv, lr, n);
        mm_t<BW>(D1, ldv0, lr, n, 1.0, true);
        bs_t<BW>(Vb, lr, n);
        a.lvw[m] = lr.ld(1);
        a.lvw[nm + m] = lr.ld(n);
        // part 4: lambda of hv2 (= D0 c1) and of dv_a (= D2 c1)
        const DLine lhv2 = X(13), lc1 = X(14);
        for (int y = 1; y <= n; ++y) {
          const double2 w0 = (y == 1 || y == n) ? make_double2(0.0, 0.0) : lr.ld(y);
          lhv2.st(y, zadd(w0, zscale(q, lsp.ld(y))));
        }
        mm_t<BW>(D0, lhv2, lc1, n);
        if (s != 3) mm_t<BW>(D2, lsp, lc1, n, a1, true);
        bs_t<BW>(Ag, lc1, n);
        zero_walls(lc1, n);  // lambda of the right-hand side of phi
        // parts 2 and 1
        const DLine lhv = X(15);
        const double z1 = s != 3 ? dt * rka(4, s + 1) : 0.0;
        for (int y = 1; y <= n; ++y) lhv.st(y, zadd(zscale(z1, lsp.ld(y)), zscale(gamma, lc1.ld(y))));
        if (s == 1) {
          mm_t<BW>(D2, lc1, X(14 - 1), n);  // X13 is free again
          bs_t<BW>(D0lu, X(13), n);
          for (int y = 1; y <= n; ++y) op.st(y, zadd(zscale(1.0 - alpha * k2, lc1.ld(y)), zscale(alpha, X(13).ld(y))));
        } else {
          for (int y = 1; y <= n; ++y) op.st(y, lc1.ld(y));
        }
      }
    } else {
      for (int y = 1; y <= n; ++y) X(0).st(y, zsub(zi(kzz, lu.ld(y)), zi(kxx, lw.ld(y))));
      // solve_g^T: lambda h_g -> X3
      helm_t<BW>(a, a.nu, k2, X(0), lsg, X(3), og, Ag, X(4), X(5));
    }
  }
  __syncthreads();
  // hvhg^T with lambda h_g = X3, lambda h_v = X15, lambda h_theta = X2
  const DLine lhg = X(3), lhv = X(15), lht = X(2);
  const DLine e1hg = X(4), e1hv = X(5), e2hv = X(6), e1ht = X(7);
  if (live) {
    if (role == 0) {
      mm_t<BW>(D1, lhg, e1hg, n);
      bs_t<BW>(D0lu, e1hg, n);
      mm_t<BW>(D1, lht, e1ht, n);
      bs_t<BW>(D0lu, e1ht, n);
    } else if (role == 1) {
      mm_t<BW>(D1, lhv, e1hv, n);
      bs_t<BW>(D0lu, e1hv, n);
    } else {
      mm_t<BW>(D2, lhv, e2hv, n);
      bs_t<BW>(D0lu, e2hv, n);
    }
  }
  __syncthreads();
  if (live) {
    const double kx2 = kx * kx, kz2 = kz * kz, kxkz = kx * kz;
    const double c2 = kx * kx * kx + kx * (kz * kz), c4 = (kx * kx) * kz + kz * kz * kz;
    auto P = [&](int i) { return DLine{a.lP + i * ns + m, nm}; };
    for (int y = 1; y <= n; ++y) {
      if (role == 0) {
        const double2 g = lhg.ld(y), ev = e1hv.ld(y);
        P(0).st(y, zsub(zscale(kxkz, g), zscale(kx2, ev)));
        P(2).st(y, zsub(zscale(-kxkz, g), zscale(kz2, ev)));
        P(4).st(y, zsub(zscale(kz2 - kx2, g), zscale(2.0 * kxkz, ev)));
      } else if (role == 1) {
        const double2 v = lhv.ld(y), eg = e1hg.ld(y), e2 = e2hv.ld(y);
        P(1).st(y, zsub(zsub(zi(kz, eg), zi(c2, v)), zi(kx, e2)));
        P(3).st(y, zsub(zsub(zi(-kx, eg), zi(c4, v)), zi(kz, e2)));
      } else {
        const double2 t = lht.ld(y), et = e1ht.ld(y);
        P(5).st(y, zi(kx, t));
        P(7).st(y, zi(kz, t));
        P(6).st(y, make_double2(-et.x, -et.y));
      }
    }
  }
}

// The (0,0) lines of wave00 transposed, one thread per line (U, W, Theta); also clears the
// (0,0) entries of the products' lambda that the lines do not read.
template <int BW>
__global__ void k_adj_mean(AdjArgs a) {
  const int line = threadIdx.x;
  if (line >= 3) return;
  const int n = a.ny, s = a.substep;
  const int64_t nm = a.nmodes, ns = a.ns;
  const double dt = a.dt;
  const BandS<BW> D0{a.d0}, D1{a.d1}, D2{a.d2}, D0lu{a.d0lu};
  const double visc = line == 2 ? a.nu / a.pr : a.nu;
  const int uslot = line == 0 ? 0 : line == 1 ? 2 : 3;  // u, w, theta in the state planes
  const int pslot = line == 0 ? 1 : line == 1 ? 3 : 6;  // uv, vw, v theta among the products
  const DLine lprof{const_cast<double2 *>(a.lS) + uslot * ns, nm}, lsn{const_cast<double2 *>(a.lRK) + line * ns, nm};
  double2 *base = a.ml + (int64_t)line * 8 * n;
  auto L = [&](int i) { return DLine{base + i * n, 1}; };
  const BandM<BW> A0{a.mb + (int64_t)line * (2 * BW + 1) * n, 1};
  const double beta = dt * rka(2, s) * visc;
  fill_rows<BW>(A0, D0, D2, 1.0, -beta, 1.0, -beta, n);
  labs_lu<BW>(A0, n);
  // the unit-source solution c_im and its integral
  const DLine cim = L(0);
  for (int y = 1; y <= n; ++y) cim.st(y, make_double2((y == 1 || y == n) ? 0.0 : 1.0, 0.0));
  labs_bs<BW>(A0, cim, n);
  double iim = 0.0;
  for (int y = 1; y <= n; ++y) iim += a.integ[y - 1] * cim.ld(y).x;
  // lambda of b1 (real): from the profile D0 b1 (- u_gal), the store and the wall stress
  const DLine lpt = L(1), lb1 = L(2), ld = L(3);
  for (int y = 1; y <= n; ++y) lpt.st(y, make_double2(lprof.ld(y).x + lsn.ld(y).x, 0.0));
  mm_t<BW>(D0, lpt, lb1, n);
  if (s != 3) {
    const double a1 = dt * rka(1, s + 1) * visc, z1 = dt * rka(4, s + 1);
    for (int y = 1; y <= n; ++y) lpt.st(y, make_double2(lsn.ld(y).x, 0.0));
    mm_t<BW>(D2, lpt, lb1, n, a1, true);
    for (int y = 1; y <= n; ++y) ld.st(y, zscale(-z1, lsn.ld(y)));
  } else {
    for (int y = 1; y <= n; ++y) ld.st(y, make_double2(0.0, 0.0));
  }
  const double ltau = line == 0 ? a.w_tau : line == 2 ? a.w_q : 0.0;
  if (s == 3 && ltau != 0.0) {
    const double f = ltau * 0.5 * visc;
    lb1.st(1, zadd(lb1.ld(1), make_double2(f * ent<BW>(D1, 1, 1, n), 0.0)));
    lb1.st(2, zadd(lb1.ld(2), make_double2(f * ent<BW>(D1, 1, 2, n), 0.0)));
    lb1.st(n - 1, zadd(lb1.ld(n - 1), make_double2(-f * ent<BW>(D1, n, n - 1, n), 0.0)));
    lb1.st(n, zadd(lb1.ld(n), make_double2(-f * ent<BW>(D1, n, n, n), 0.0)));
  }
  // b1 = c_re + phi c_im, phi = (bulk - w . c_re / 2) / (I_im / 2) (calculate_phi)
  if (line != 1) {
    double cl = 0.0;
    for (int y = 1; y <= n; ++y) cl += cim.ld(y).x * lb1.ld(y).x;
    for (int y = 1; y <= n; ++y) lb1.st(y, make_double2(lb1.ld(y).x - a.integ[y - 1] * cl / iim, 0.0));
  }
  bs_t<BW>(A0, lb1, n);  // lambda of the real right-hand side
  const DLine lt = L(4);
  for (int y = 1; y <= n; ++y) lt.st(y, make_double2((y == 1 || y == n) ? 0.0 : lb1.ld(y).x, 0.0));
  const double gamma = dt * rka(3, s);
  const DLine lstore = L(5);
  if (s == 1) {
    const double alpha = dt * rka(1, s) * visc;
    mm_t<BW>(D2, lt, lstore, n);
    bs_t<BW>(D0lu, lstore, n);
    for (int y = 1; y <= n; ++y) lstore.st(y, zadd(lt.ld(y), zscale(alpha, lstore.ld(y))));
  } else {
    for (int y = 1; y <= n; ++y) lstore.st(y, lt.ld(y));
  }
  for (int y = 1; y <= n; ++y) ld.st(y, zsub(ld.ld(y), zscale(gamma, lt.ld(y))));
  const DLine lflux = L(6);
  mm_t<BW>(D1, ld, lflux, n);
  bs_t<BW>(D0lu, lflux, n);
  const DLine outp{a.lP + pslot * ns, nm}, outs{a.lRK0 + line * ns, nm};
  for (int y = 1; y <= n; ++y) {
    outp.st(y, lflux.ld(y));
    outs.st(y, lstore.ld(y));
  }
  if (line == 0) {
    const int other[5] = {0, 2, 4, 5, 7};
    for (int i = 0; i < 5; ++i) {
      const DLine o{a.lP + other[i] * ns, nm};
      for (int y = 1; y <= n; ++y) o.st(y, make_double2(0.0, 0.0));
    }
  }
}

// The control probe transposed, per mode: lambda of v_wall -> lambda of the starting v (written to
// lS0's v plane; the other planes cleared) and the gain sums G(m) += Re(conj(lambda v_wall) P(w.v)).
struct ProbeArgs {
  int ny, nxh, nz;
  int64_t nmodes, ns;
  double amp;
  const float *gains;
  const double *wlo, *whi;
  const double2 *vbase;  // the starting v planes
  const double2 *lvw;
  double2 *lS0;
  double *G;
};

__global__ void __launch_bounds__(128) k_adj_probe(ProbeArgs a) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes) return;
  const int n = a.ny;
  const int64_t nm = a.nmodes;
  const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
  const DLine v{const_cast<double2 *>(a.vbase) + m, nm};
  const DLine out{a.lS0 + a.ns + m, nm};
  for (int f = 0; f < 4; ++f)
    if (f != 1) {
      const DLine o{a.lS0 + f * a.ns + m, nm};
      for (int y = 1; y <= n; ++y) o.st(y, make_double2(0.0, 0.0));
    }
  const bool live = m != 0 && kzi != a.nz / 2;
  double2 plo = make_double2(0.0, 0.0), phi = make_double2(0.0, 0.0);  // lambda of the probes w . v_m
  if (live) {
    const double ag = a.amp * (double)a.gains[m];
    const double2 llo = a.lvw[m], lhi = a.lvw[nm + m];
    if (kxi != 0) {
      plo = zscale(ag, llo);
      phi = zscale(ag, lhi);
    } else {
      // v_wall(m) = A g(m) (probe_m + conj probe_mp) / 2; mode mp's wall value reads conj(probe_m)
      const int64_t mp = (int64_t)((a.nz - kzi) % a.nz) * a.nxh;
      const double agp = a.amp * (double)a.gains[mp];
      const double2 qlo = a.lvw[mp], qhi = a.lvw[nm + mp];
      plo = make_double2(0.5 * (ag * llo.x + agp * qlo.x), 0.5 * (ag * llo.y - agp * qlo.y));
      phi = make_double2(0.5 * (ag * lhi.x + agp * qhi.x), 0.5 * (ag * lhi.y - agp * qhi.y));
    }
    // the gain sums: Re(conj(lambda v_wall) P(w . v)) with the forward's projection
    double2 rlo = make_double2(0.0, 0.0), rhi = make_double2(0.0, 0.0);
    for (int y = 1; y <= n; ++y) {
      rlo = zadd(rlo, zscale(a.wlo[y - 1], v.ld(y)));
      rhi = zadd(rhi, zscale(a.whi[y - 1], v.ld(y)));
    }
    if (kxi == 0) {
      const int64_t mp = (int64_t)((a.nz - kzi) % a.nz) * a.nxh;
      const DLine vp{const_cast<double2 *>(a.vbase) + mp, nm};
      double2 qlo = make_double2(0.0, 0.0), qhi = make_double2(0.0, 0.0);
      for (int y = 1; y <= n; ++y) {
        qlo = zadd(qlo, zscale(a.wlo[y - 1], vp.ld(y)));
        qhi = zadd(qhi, zscale(a.whi[y - 1], vp.ld(y)));
      }
      rlo = make_double2(0.5 * (rlo.x + qlo.x), 0.5 * (rlo.y - qlo.y));
      rhi = make_double2(0.5 * (rhi.x + qhi.x), 0.5 * (rhi.y - qhi.y));
    }
    a.G[m] += zcm(llo, rlo).x + zcm(lhi, rhi).x;
  }
  for (int y = 1; y <= n; ++y)
    out.st(y, live ? zadd(zscale(a.wlo[y - 1], plo), zscale(a.whi[y - 1], phi)) : make_double2(0.0, 0.0));
}

__global__ void k_axpy(double2 *y, const double2 *x, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = zadd(y[i], x[i]);
}

__global__ void k_accumulate_J(double *J, const DevScalars *dsc, double w_tau, double w_q) {
  if (threadIdx.x == 0 && blockIdx.x == 0) J[0] += w_tau * dsc->wall_shear_stress + w_q * dsc->wall_theta_stress;
}

template <typename T>
int adj_alloc(Handle &h, T **p, size_t count) {
  const size_t bytes = sizeof(T) * (count ? count : 1);
  const cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e != cudaSuccess) {
    set_error("adjoint: cudaMalloc of " + std::to_string(bytes) + " bytes failed: " + cudaGetErrorString(e));
    return KMM_ERR_CUDA;
  }
  return KMM_OK;
}

int adjoint_buffers(Handle &h) {
  if (h.adj) return KMM_OK;
  h.adj = new Adjoint();
  Adjoint &A = *h.adj;
  const size_t ns = (size_t)h.ns, nm = (size_t)h.nm, ny = (size_t)h.ny;
  const size_t band = (size_t)(2 * h.bw + 1) * ns;
  int rc;
  if ((rc = adj_alloc(h, &A.fin, 7 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.sb, 12 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.lS, 4 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.lRK, 3 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.lS0, 4 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.lRK0, 3 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.lP, 8 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.lmid, 8 * nm))) return rc;
  if ((rc = adj_alloc(h, &A.tmp, 4 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.X, (size_t)kAdjLines * ns))) return rc;
  if ((rc = adj_alloc(h, &A.B, 9 * band))) return rc;
  if ((rc = adj_alloc(h, &A.Xc, 18 * ns))) return rc;
  if ((rc = adj_alloc(h, &A.ml, 3 * 8 * ny))) return rc;
  if ((rc = adj_alloc(h, &A.mb, 3 * (size_t)(2 * h.bw + 1) * ny))) return rc;
  if ((rc = adj_alloc(h, &A.lvw, 2 * (size_t)h.nmodes))) return rc;
  if ((rc = adj_alloc(h, &A.G, (size_t)h.nmodes))) return rc;
  if ((rc = adj_alloc(h, &A.J, 1))) return rc;
  return KMM_OK;
}

template <int BW>
cudaError_t adj_substep_bw(Handle &h, int s, const double2 *sbase, double dt, double w_tau, double w_q,
                           cudaStream_t st) {
  Adjoint &A = *h.adj;
  const OpsOffsets off = ops_offsets(h.bw, h.ny);
  AdjArgs a{};
  a.ny = h.ny;
  a.nxh = h.nxh;
  a.nz = h.nz;
  a.substep = s;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.dt = dt;
  a.nu = h.cfg.nu;
  a.pr = h.cfg.pr;
  a.lmfxr = h.lmfxr;
  a.lmfzr = h.lmfzr;
  a.d0 = h.dops + off.d0;
  a.d1 = h.dops + off.d1;
  a.d2 = h.dops + off.d2;
  a.d0lu = h.dops + off.d0lu;
  a.integ = h.dops + off.integ;
  a.lS = A.lS;
  a.lRK = A.lRK;
  a.lP = A.lP;
  a.lRK0 = A.lRK0;
  a.lvw = A.lvw;
  a.X = A.X;
  a.B = A.B + (int64_t)(s - 1) * 3 * (2 * h.bw + 1) * h.ns;
  a.Xc = A.Xc + (int64_t)(s - 1) * 6 * h.ns;
  a.ml = A.ml;
  a.mb = A.mb;
  a.w_tau = w_tau;
  a.w_q = w_q;
  cudaError_t e;
  if (!A.cvalid[s - 1] || A.cdt[s - 1] != dt) {
    k_adj_factor<BW><<<(unsigned)((h.nmodes + 63) / 64), 64, 0, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    A.cdt[s - 1] = dt;
    A.cvalid[s - 1] = true;
  }
  // the (0,0) lines on the side stream beside the other modes (disjoint entries of every line)
  if ((e = cudaEventRecord(h.ev_fork, st)) != cudaSuccess) return e;
  if ((e = cudaStreamWaitEvent(h.side, h.ev_fork, 0)) != cudaSuccess) return e;
  k_adj_mean<BW><<<1, 32, 0, h.side>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaEventRecord(h.ev_join, h.side)) != cudaSuccess) return e;
  // three role warps per 32 modes
  k_adj_modes<BW><<<(unsigned)((h.nmodes + 31) / 32), 32 * kAdjRoles, 0, st>>>(a);
  if ((e = cudaStreamWaitEvent(st, h.ev_join, 0)) != cudaSuccess) return e;
  const unsigned blocks = (unsigned)((h.nmodes + 127) / 128);
  ProbeArgs pa{};
  pa.ny = h.ny;
  pa.nxh = h.nxh;
  pa.nz = h.nz;
  pa.nmodes = h.nmodes;
  pa.ns = h.ns;
  pa.amp = h.cfg.control_amp;
  pa.gains = h.gains;
  pa.wlo = h.dops + off.wlo;
  pa.whi = h.dops + off.whi;
  pa.vbase = sbase + h.ns;
  pa.lvw = A.lvw;
  pa.lS0 = A.lS0;
  pa.G = A.G;
  k_adj_probe<<<blocks, 128, 0, st>>>(pa);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  // x_to_y^T, products^T at the starting state, y_to_x^T
  if ((e = launch_zinv(h, sbase, h.MID, 4, st)) != cudaSuccess) return e;
  if ((e = launch_zinv(h, A.lP, A.lmid, 8, st)) != cudaSuccess) return e;
  if ((e = launch_xadj2(h, reinterpret_cast<const double2 *>(h.MID), A.lmid, h.rescale, st)) != cudaSuccess) return e;
  if ((e = launch_zfwd(h, A.lmid, A.tmp, 4, 1.0, true, st)) != cudaSuccess) return e;
  const int64_t n4 = 4 * h.ns;
  k_axpy<<<(unsigned)((n4 + 255) / 256), 256, 0, st>>>(A.lS0, A.tmp, n4);
  return cudaGetLastError();
}

cudaError_t adj_substep(Handle &h, int s, const double2 *sbase, double dt, double w_tau, double w_q,
                        cudaStream_t st) {
  switch (h.bw) {
    case 2: return adj_substep_bw<2>(h, s, sbase, dt, w_tau, w_q, st);
    case 3: return adj_substep_bw<3>(h, s, sbase, dt, w_tau, w_q, st);
    case 4: return adj_substep_bw<4>(h, s, sbase, dt, w_tau, w_q, st);
    case 5: return adj_substep_bw<5>(h, s, sbase, dt, w_tau, w_q, st);
    case 6: return adj_substep_bw<6>(h, s, sbase, dt, w_tau, w_q, st);
    case 7: return adj_substep_bw<7>(h, s, sbase, dt, w_tau, w_q, st);
    default: return cudaErrorInvalidValue;
  }
}

int adjoint_checks(Handle &h, const char *name) {
  if (h.mixed) {
    set_error(std::string(name) + ": the adjoint runs in FP64; create the handle with KMM_PREC_FP64");
    return KMM_ERR_CONFIG;
  }
  if (!h.cfg.fixed_dt) {
    set_error(std::string(name) + ": the adjoint needs a fixed time step (fixed_dt = 1)");
    return KMM_ERR_CONFIG;
  }
  if (h.nsc != 1) {
    set_error(std::string(name) + ": the adjoint covers one passive scalar");
    return KMM_ERR_CONFIG;
  }
  return KMM_OK;
}

}  // namespace

void adjoint_free(Handle &h) {
  if (!h.adj) return;
  Adjoint &A = *h.adj;
  for (double2 *p : A.ck) cudaFree(p);
  void *ptrs[] = {A.fin, A.sb, A.lS, A.lRK, A.lS0, A.lRK0, A.lP, A.lmid, A.tmp, A.X, A.B, A.Xc, A.ml, A.mb, A.lvw, A.G, A.J};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  delete h.adj;
  h.adj = nullptr;
}

}  // namespace kmm

using namespace kmm;

extern "C" {

int kmm_adjoint_forward(kmm_handle *hh, int nsteps, double w_tau, double w_q, double *J) {
  if (!hh || nsteps <= 0) {
    set_error("kmm_adjoint_forward: null handle or nsteps <= 0");
    return KMM_ERR_ARG;
  }
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  int rc = adjoint_checks(h, "kmm_adjoint_forward");
  if (rc) return rc;
  if ((rc = adjoint_buffers(h))) return rc;
  Adjoint &A = *h.adj;
  const size_t ck_bytes = sizeof(double2) * 7 * (size_t)h.ns;
  while ((int)A.ck.size() < nsteps) {
    double2 *p = nullptr;
    if ((rc = adj_alloc(h, &p, 7 * (size_t)h.ns))) return rc;
    A.ck.push_back(p);
  }
  if (h.ops.wlo.empty()) {
    // the probe weights of the configured detection plane, also when the amplitude is zero
    std::string err;
    if ((rc = build_control_weights(h.ops, h.cfg.control_yd, err))) {
      set_error("kmm_adjoint_forward: " + err);
      return rc;
    }
    const OpsOffsets off = ops_offsets(h.bw, h.ny);
    ADJ_CUDA(cudaMemcpy(h.dops + off.wlo, h.ops.wlo.data(), sizeof(double) * (size_t)h.ny, cudaMemcpyHostToDevice));
    ADJ_CUDA(cudaMemcpy(h.dops + off.whi, h.ops.whi.data(), sizeof(double) * (size_t)h.ny, cudaMemcpyHostToDevice));
  }
  if ((rc = capture_step_graph(h))) return rc;
  cudaStream_t st = h.stream;
  ADJ_CUDA(cudaMemsetAsync(A.J, 0, sizeof(double), st));
  const double wt = w_tau / nsteps, wq = w_q / nsteps;
  for (int n = 0; n < nsteps; ++n) {
    ADJ_CUDA(cudaMemcpyAsync(A.ck[n], h.S, sizeof(double2) * 4 * (size_t)h.ns, cudaMemcpyDeviceToDevice, st));
    ADJ_CUDA(cudaMemcpyAsync(A.ck[n] + 4 * h.ns, h.RK, sizeof(double2) * 3 * (size_t)h.ns, cudaMemcpyDeviceToDevice, st));
    ADJ_CUDA(cudaGraphLaunch(h.gexec, st));
    k_accumulate_J<<<1, 32, 0, st>>>(A.J, h.dsc, wt, wq);
  }
  (void)ck_bytes;
  ADJ_CUDA(cudaGetLastError());
  ADJ_CUDA(cudaStreamSynchronize(st));
  int err = 0;
  if ((rc = read_device_scalars(h, nullptr, &err))) return rc;
  if (err) {
    set_error("kmm_adjoint_forward: the step failed on the device (status " + std::to_string(err) + ")");
    return err;
  }
  A.nsteps = nsteps;
  A.w_tau = w_tau;
  A.w_q = w_q;
  if (J) ADJ_CUDA(cudaMemcpy(J, A.J, sizeof(double), cudaMemcpyDeviceToHost));
  return KMM_OK;
}

int kmm_adjoint_backward(kmm_handle *hh, double *dJ_dA, double *dJ_dgains) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  int rc = adjoint_checks(h, "kmm_adjoint_backward");
  if (rc) return rc;
  if (!h.adj || h.adj->nsteps <= 0) {
    set_error("kmm_adjoint_backward: no recorded trajectory (call kmm_adjoint_forward first)");
    return KMM_ERR_ARG;
  }
  Adjoint &A = *h.adj;
  cudaStream_t st = h.stream;
  const size_t ns = (size_t)h.ns;
  double dt = 0.0;
  ADJ_CUDA(cudaStreamSynchronize(st));
  ADJ_CUDA(cudaMemcpy(&dt, &h.dsc->dt, sizeof(double), cudaMemcpyDeviceToHost));
  ADJ_CUDA(cudaMemcpyAsync(A.fin, h.S, sizeof(double2) * 4 * ns, cudaMemcpyDeviceToDevice, st));
  ADJ_CUDA(cudaMemcpyAsync(A.fin + 4 * ns, h.RK, sizeof(double2) * 3 * ns, cudaMemcpyDeviceToDevice, st));
  ADJ_CUDA(cudaMemsetAsync(A.lS, 0, sizeof(double2) * 4 * ns, st));
  ADJ_CUDA(cudaMemsetAsync(A.lRK, 0, sizeof(double2) * 3 * ns, st));
  ADJ_CUDA(cudaMemsetAsync(A.G, 0, sizeof(double) * (size_t)h.nmodes, st));
  const int N = A.nsteps;
  for (int n = N - 1; n >= 0; --n) {
    ADJ_CUDA(cudaMemcpyAsync(h.S, A.ck[n], sizeof(double2) * 4 * ns, cudaMemcpyDeviceToDevice, st));
    ADJ_CUDA(cudaMemcpyAsync(h.RK, A.ck[n] + 4 * ns, sizeof(double2) * 3 * ns, cudaMemcpyDeviceToDevice, st));
    for (int s = 1; s <= 3; ++s) {
      ADJ_CUDA(cudaMemcpyAsync(A.sb + (s - 1) * 4 * ns, h.S, sizeof(double2) * 4 * ns, cudaMemcpyDeviceToDevice, st));
      if (s < 3 && (rc = run_substep(h, s, st))) return rc;
    }
    for (int s = 3; s >= 1; --s) {
      const double wt = s == 3 ? A.w_tau / N : 0.0, wq = s == 3 ? A.w_q / N : 0.0;
      ADJ_CUDA(adj_substep(h, s, A.sb + (s - 1) * 4 * ns, dt, wt, wq, st));
      std::swap(A.lS, A.lS0);
      std::swap(A.lRK, A.lRK0);
    }
  }
  ADJ_CUDA(cudaMemcpyAsync(h.S, A.fin, sizeof(double2) * 4 * ns, cudaMemcpyDeviceToDevice, st));
  ADJ_CUDA(cudaMemcpyAsync(h.RK, A.fin + 4 * ns, sizeof(double2) * 3 * ns, cudaMemcpyDeviceToDevice, st));
  std::vector<double> G((size_t)h.nmodes);
  std::vector<float> g((size_t)h.nmodes);
  ADJ_CUDA(cudaMemcpyAsync(G.data(), A.G, sizeof(double) * G.size(), cudaMemcpyDeviceToHost, st));
  ADJ_CUDA(cudaMemcpyAsync(g.data(), h.gains, sizeof(float) * g.size(), cudaMemcpyDeviceToHost, st));
  ADJ_CUDA(cudaStreamSynchronize(st));
  int err = 0;
  if ((rc = read_device_scalars(h, nullptr, &err))) return rc;
  if (err) {
    set_error("kmm_adjoint_backward: a recomputed step failed on the device (status " + std::to_string(err) + ")");
    return err;
  }
  double da = 0.0;
  for (size_t m = 0; m < G.size(); ++m) da += (double)g[m] * G[m];
  if (dJ_dA) *dJ_dA = da;
  if (dJ_dgains)
    for (size_t m = 0; m < G.size(); ++m) dJ_dgains[m] = h.cfg.control_amp * G[m];
  return KMM_OK;
}

int kmm_adjoint_release(kmm_handle *hh) {
  if (!hh) return KMM_ERR_ARG;
  Handle &h = *reinterpret_cast<Handle *>(hh);
  DeviceGuard dg(h.cfg.device);
  cudaStreamSynchronize(h.stream);
  adjoint_free(h);
  return KMM_OK;
}

}  // extern "C"
