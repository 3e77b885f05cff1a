// wavespace_split.cu - the per-(kx, kz) wall-normal solves of one substep (wavespace.f90:22-113)
// as three kernels with several threads per mode.
//
// One thread per mode leaves about four warps on each SM (nxh * nz modes), too few to cover the
// memory latency of the row recurrences.  The solves of one mode are independent chains, so each
// kernel gives every chain its own warp ("role"); lane t of a warp owns mode 32 * block + t, so
// every line access of a warp stays one contiguous run.
//
// k_hvhg (hvhg.f90:56-159), one D0 solve per role, ascending then descending:
//   role 0  a3 = -kx^2 f1 - 2 kx kz f5 - kz^2 f3   -> HV0 = i(kx^3+kx kz^2) f2 + i(kx^2 kz+kz^3) f4 + D1 c(a3)
//   role 1  f8                                      -> HT  = -(i kx f7 + i kz f9 + D1 c(f8))
//   role 2  f2                                      -> G2  = a1 - i kz D1 c(f2),  V2 = i kx D2 c(f2)
//   role 3  f4                                      -> G3  = i kx D1 c(f4),       V3 = i kz D2 c(f4)
//           and, with opposition control, the probes v(+-y_d) of the starting v
//   so hg = G2 + G3, hv = HV0 + (V2 + V3), ht = HT.  At substep 1 roles 0-2 also solve D0 for the
//   store they feed (RK_STORE 2, 3, 1) and emit D2 of it (DP, DT, DG; solve_g.f90:84-111).
// k_helmholtz, one profile LU per role (solve_t.f90:28-201, solve_g.f90, solve_v_f.f90:95-298):
//   role 0  (alpha D0 - beta_t D2) theta = rhs_t      -> St, new RK_STORE 3
//   role 1  (alpha D0 - beta D2) g = rhs_g             -> Su (g), new RK_STORE 1
//   role 2  (alpha D0 - beta D2) phi_p = rhs_phi       -> new RK_STORE 2 (partial), then
//           (D2 - k^2 D0) v_p = phi_p, v_p = vwall     -> Sv = v_p, Sw = D1 v_p
//   role 3  (alpha D0 - beta D2) phi_h = (p0, 0, ..)   -> phi_h, D2 phi_h, then
//           (D2 - k^2 D0) v_h = phi_h, v_h = 0 at walls -> v_h, D1 v_h
//   phi_h and v_h have equal real and imaginary parts (the unit wall vector is (p0, p0),
//   solve_v_f.f90:142), so role 3 carries one real chain.
// k_assemble, one thread per (y, mode): C1, C2 from the wall derivatives (solve_v_f.f90:293-298),
//   v, dv/dy, RK_STORE 2 completion, then u and w (solve_u_w.f90:27-38).
// k_mean, three threads on a forked stream: wave00.f90:41-714 for U, W and Theta.
#include <cuda_runtime.h>

#include "kmm_internal.h"
#include "sweeps.cuh"

namespace kmm {

namespace {

constexpr int kLanes = 32;  // modes per block; one warp per role
constexpr int kRoles = 4;

// Lines k_hvhg hands to k_helmholtz.  The six nonlinear-term lines H_HV0..H_V3 are combinations
// of the products and are stored at the products' precision PT (float2 in the mixed path, packed
// at (PT *)hl + i * ns); the substep-1 lines H_DP, H_DT, H_DG (D2 D0^{-1} of the FP64 RK stores)
// stay double2 at hl + i * ns.
// A second passive scalar adds H_HT2 (its nonlinear term, at PT like H_HT) and H_DT2 (substep 1,
// double2 like H_DT).
enum HLine { H_HV0 = 0, H_HT, H_G2, H_V2, H_G3, H_V3, H_DP, H_DT, H_DG, H_HT2, H_DT2, H_COUNT };

// Low-storage RK3 coefficients alpha, beta, gamma, zeta of substeps 1-3
// (RK3_initialize, module_runge_kutta.f90:34-45).
__constant__ double c_rk[4][3] = {{29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0},
                                  {37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0},
                                  {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0},
                                  {0.0, -17.0 / 60.0, -5.0 / 12.0}};
__device__ __forceinline__ double rkc(int c, int s) { return c_rk[c - 1][s - 1]; }

struct SplitArgs {
  int ny, nxh, nz, substep;
  int64_t nmodes, ns;
  double2 *S, *RK;
  const void *P;
  double2 *zl;       // [8][ny][nm] role-private forward lines
  double2 *hl;       // [H_COUNT][ny][nm] hvhg outputs
  double *xr;        // [6][ny][nm] real lines of role 3
  double *ub;        // [3][ub_role] per-role U factors
  int64_t ub_role;   // doubles per role
  double2 *dv;       // [3][nm] dv_p(1), dv_p(n), (dv_h(1), dv_h(n))
  const double *tabs;   // t0, t1, t2, l0, u0
  double2 *vwall;          // [2][nm] control probes v(y_d), v(-y_d) of each mode
  const double *wlo, *whi;  // control weights: v(y_d) = w . v
  const float *gains;       // control gain per mode
  double control_amp;
  double nu, pr, pr2, lmfxr, lmfzr;
  DevScalars *dsc;
  const double *dt_ptr;
  double *vf;        // the v operator's profile LU per mode: LBand, then UBand at vf + vf_l
  int64_t vf_l;
  int groups;        // 32-mode groups per block of k_hvhg (Tuning::groups)
  int hgroups;       // 32-mode groups per block of k_helmholtz (Tuning::hgroups)
  int ulayout;       // U factor layout of the per-role regions (Tuning::ulayout)
  int stab;          // 1: k_hvhg copies the operator tables it reads to shared memory
  int hstab;         // 1: k_helmholtz does (Tuning::hstab)
  // this substep's influence lines phi_h, D2 phi_h, v_h, dv_h / dy [4][ny][nm] and v_h's wall
  // derivatives [nm] (the factor cache's slots with Tuning::fcache, else xr lines 1..4, dv line 2)
  double *xinf;
  double2 *dvh;
  // Tuning::fcache: this substep's cached LU of theta's operator (fth) and of the one g and phi
  // share (fgp), each an LBand with its UBand vf_l doubles on, and the dt they hold (fcdt)
  double *fth, *fgp;
  double *fcdt;
};

// Operator tables in shared memory (SplitArgs::stab).  Every lane of a warp reads the same table
// entry at the same row (the modes of a warp sweep in lockstep), yet beside the streamed lines
// L1 kept only about a third of those reads.  The block copies the 3 tables a kernel reads,
// 3 * ny * (4BW+1) doubles starting at table `first` of T0, T1, T2, L0 + U0, before any sweep.
template <int BW>
__device__ __forceinline__ const double *tabs_to_shared(const SplitArgs &a, int first, double *smem) {
  const int tw = a.ny * (4 * BW + 1);
  const double *src = a.tabs + first * tw;
  for (int i = threadIdx.x; i < 3 * tw; i += blockDim.x) smem[i] = src[i];
  __syncthreads();
  return smem;
}

// A solver role's U factors for mode m: [offset][y][mode] (layout 0) or [y][offset][mode]
// (layout 1, the BW offsets of one row next to each other); the first rows' extra entries follow
// at BW * ns in both.
template <int BW>
__device__ __forceinline__ UBand<BW> role_uband(const SplitArgs &a, int role, int64_t m) {
  double *base = a.ub + role * a.ub_role + m;
  return a.ulayout == 0 ? make_uband<BW>(base, a.nmodes, a.ns)
                        : make_uband<BW>(base, BW * a.nmodes, a.nmodes, BW * a.ns, a.nmodes);
}

template <typename PT> __device__ __forceinline__ double2 ldp(const PT *p);
template <> __device__ __forceinline__ double2 ldp<double2>(const double2 *p) { return *p; }
template <> __device__ __forceinline__ double2 ldp<float2>(const float2 *p) {
  const float2 v = *p;
  return make_double2((double)v.x, (double)v.y);
}

struct ModeK {
  double kx, kz, k2;
};
__device__ __forceinline__ ModeK mode_k(const SplitArgs &a, int64_t m) {
  const int mi = (int)m, kzi = mi / a.nxh, kxi = mi - kzi * a.nxh;
  const int kzint = (kzi <= a.nz / 2) ? kzi : kzi - a.nz;  // set_waveno
  ModeK k;
  k.kx = kxi * a.lmfxr;                                   // wavespace.f90:69
  k.kz = kzint * a.lmfzr;
  k.k2 = k.kx * k.kx + k.kz * k.kz;
  return k;
}

// A = ca D0 - cb D2 with the Dirichlet first / last rows, as an offset row (|e| <= BW only
// for a centre row, which is never a wall row).
template <int BW>
__device__ __forceinline__ void helm_row(const Tabs<BW> &tb, int r, int n, double ca, double cb, double *out,
                                         bool centre) {
  const double *r0 = trow<BW>(tb.t0, r), *r2 = trow<BW>(tb.t2, r);
  if (centre) {
#pragma unroll
    for (int e = -BW; e <= BW; ++e) out[e + 2 * BW] = ca * r0[e] - cb * r2[e];
    return;
  }
  if (r == 1 || r == n) {
#pragma unroll
    for (int e = -2 * BW; e <= 2 * BW; ++e) out[e + 2 * BW] = 0.0;
    out[2 * BW] = ca * r0[0] - cb * r2[0];
    return;
  }
#pragma unroll
  for (int e = -2 * BW; e <= 2 * BW; ++e) out[e + 2 * BW] = ca * r0[e] - cb * r2[e];
}

// (D2 - k^2 D0) with the wall rows replaced by D0 (v given there), solve_v_f.f90:95-140.
template <int BW>
__device__ __forceinline__ void vrow(const Tabs<BW> &tb, int r, int n, double k2, double *row, bool centre) {
  const double *r0 = trow<BW>(tb.t0, r), *r2 = trow<BW>(tb.t2, r);
  if (centre) {
#pragma unroll
    for (int e = -BW; e <= BW; ++e) row[e + 2 * BW] = -k2 * r0[e] + r2[e];
    return;
  }
  if (r == 1 || r == n) {
#pragma unroll
    for (int e = -2 * BW; e <= 2 * BW; ++e) row[e + 2 * BW] = 0.0;
    row[2 * BW] = r0[0];
    return;
  }
#pragma unroll
  for (int e = -2 * BW; e <= 2 * BW; ++e) row[e + 2 * BW] = -k2 * r0[e] + r2[e];
}

// A staged nonlinear-term unit, widened to double2.
template <typename PT, int K, int S>
__device__ __forceinline__ double2 ring_hv(const Ring<K, S> &ring, int step, int k) {
  if constexpr (sizeof(PT) == sizeof(float2)) return ring.f(step, k);
  else return ring.c(step, k);
}

// ------------------------------------------------------------------------------------------
// k_hvhg: role ROLE of mode m; NC = 2 adds the store's D0 solve at substep 1.
// SA = 0: the sweeps prefetch their rows into L1 (kPrefetchRows ahead).  SA = 1, 2: they stage
// them through a thread-private shared-memory ring, cp.async SA rows ahead (Ring; as in
// k_helmholtz), kHvUnits 16-byte units per row:
//   forward   0..2 the role's products, 3 the RK store (substep 1), 4 v (the control probe);
//   backward  0 the product chain, 1 the store chain, 2..4 the products the emission of row
//             q = r + BW reads.
constexpr int kHvUnits = 5;

template <int BW, typename PT, int ROLE, int NC, int SA>
__device__ __forceinline__ void hvhg_role(const SplitArgs &a, const Tabs<BW> &tb, int64_t m,
                                          const Ring<kHvUnits, SA + 1> &ring) {
  const int n = a.ny;
  const int64_t nm = a.nmodes, ns = a.ns;
  const ModeK k = mode_k(a, m);
  const double kx = k.kx, kz = k.kz;
  const double kxkz = kx * kz, kx2 = kx * kx, kz2 = kz * kz;
  const PT *P = reinterpret_cast<const PT *>(a.P) + m;
  auto prod = [&](int slot, int r) { return ldp<PT>(P + slot * ns + (r - 1) * (int)nm); };
  auto pfp = [&](int slot, int r) { pf_l1(P + slot * ns + (r - 1) * (int)nm); };
  auto pat = [&](int slot, int r) { return P + slot * ns + (r - 1) * (int)nm; };
  // a product of row r: staged (unit u of step `step`) or straight from global memory
  auto rp = [&](int step, int u) { return ring_hv<PT>(ring, step, u); };
  // the product chain's forward results at the products' precision (PT), the store chain's
  // (substep 1, FP64 state) in double2
  const Line<PT> Z0{reinterpret_cast<PT *>(a.zl + (2 * ROLE) * ns) + m, nm};
  const DLine Z1{a.zl + (2 * ROLE + 1) * ns + m, nm};
  // role 4 is a second scalar: products u, v, w theta2 in P slots 8, 9, 10, store 4
  constexpr bool SCAL = ROLE == 1 || ROLE == 4;
  constexpr int s7 = ROLE == 4 ? 8 : 5, s8 = ROLE == 4 ? 9 : 6, s9 = ROLE == 4 ? 10 : 7;
  constexpr int store_slot = ROLE == 0 ? 1 : ROLE == 1 ? 2 : ROLE == 4 ? 3 : 0;  // RK_STORE 2, 3, (4), 1
  constexpr int d2_line = ROLE == 0 ? H_DP : ROLE == 1 ? H_DT : ROLE == 4 ? H_DT2 : H_DG;
  const DLine Rs{a.RK + store_slot * ns + m, nm};
  auto hl = [&](int i) { return DLine{a.hl + i * ns + m, nm}; };
  auto hv = [&](int i) { return Line<PT>{reinterpret_cast<PT *>(a.hl) + i * ns + m, nm}; };
  auto ufix = [&](int r, int e) { return tb.u0[(r - 1) * 2 * BW + e - 1]; };
  // Role 3 also probes the wall-normal velocity at the detection planes for opposition
  // control: v(+-y_d) = w . v over the substep's starting v, with the precomputed weights
  // w = D0^{-T} B(+-y_d).
  const bool probe = ROLE == 3 && a.control_amp != 0.0;
  const DLine Sv{a.S + ns + m, nm};
  double2 plo = z2(0.0, 0.0), phi = z2(0.0, 0.0);

  constexpr int PF = SA > 0 ? SA : kPrefetchRows;
  constexpr bool RING = SA > 0;
  fwd_fixed<BW, NC, PF, RING>(tb, n,
      [&](int r, double2 *b) {
        if constexpr (ROLE == 0) {
          const double2 f1 = RING ? rp(r, 0) : prod(0, r), f3 = RING ? rp(r, 1) : prod(2, r);
          const double2 f5 = RING ? rp(r, 2) : prod(4, r);
          b[0] = zsub(zsub(zscale(-kx2, f1), zscale(2.0 * kxkz, f5)), zscale(kz2, f3));
        } else if constexpr (SCAL) {
          b[0] = RING ? rp(r, 0) : prod(s8, r);
        } else if constexpr (ROLE == 2) {
          b[0] = RING ? rp(r, 0) : prod(1, r);
        } else {
          b[0] = RING ? rp(r, 0) : prod(3, r);
          if (probe) {
            const double2 v = RING ? ring.c(r, 4) : Sv.ld(r);
            plo = zadd(plo, zscale(__ldg(a.wlo + r - 1), v));
            phi = zadd(phi, zscale(__ldg(a.whi + r - 1), v));
          }
        }
        if constexpr (NC == 2) b[1] = RING ? ring.c(r, 3) : Rs.ld(r);
      },
      [&](int r, const double2 *z) {
        Z0.st(r, z[0]);
        if constexpr (NC == 2) Z1.st(r, z[1]);
      },
      [&](int r) {
        if constexpr (RING) {
          if constexpr (ROLE == 0) {
            ring.get(r, 0, pat(0, r));
            ring.get(r, 1, pat(2, r));
            ring.get(r, 2, pat(4, r));
          } else {
            ring.get(r, 0, pat(SCAL ? s8 : ROLE == 2 ? 1 : 3, r));
          }
          if constexpr (NC == 2) ring.get(r, 3, Rs.p + (r - 1) * (int)nm);
          if (probe) ring.get(r, 4, Sv.p + (r - 1) * (int)nm);
        } else {
          if constexpr (ROLE == 0) { pfp(0, r); pfp(2, r); pfp(4, r); }
          else pfp(SCAL ? s8 : ROLE == 2 ? 1 : 3, r);
          if constexpr (NC == 2) pf_l1(Rs.p + (r - 1) * (int)nm);
          if (probe) pf_l1(Sv.p + (r - 1) * (int)nm);
        }
      });
  if (probe) {
    a.vwall[m] = plo;
    a.vwall[nm + m] = phi;
  }

  bwd_emit<BW, NC, 0, PF, RING>(n, ufix,
      [&](int r, double2 *zc, double *) {
        zc[0] = RING ? rp(r, 0) : Z0.ld(r);
        if constexpr (NC == 2) zc[1] = RING ? ring.c(r, 1) : Z1.ld(r);
      },
      [&](int q, int r, const double2 (&wc)[NC][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        // the products of row q: staged with step r when q = r + BW, else from global memory
        const bool st = RING && q == r + BW;
        auto pq = [&](int slot, int u) { return st ? rp(r, u) : prod(slot, q); };
        if constexpr (ROLE == 0) {
          const double c2i = kx * kx * kx + kx * (kz * kz), c4i = (kx * kx) * kz + kz * kz * kz;
          const double2 f2 = pq(1, 2), f4 = pq(3, 3);
          const double2 ehv = z2(-c2i * f2.y - c4i * f4.y, c2i * f2.x + c4i * f4.x);
          hv(H_HV0).st(q, zadd(ehv, mvc<BW>(tb.t1, q, r, wc[0])));
        } else if constexpr (SCAL) {
          const double2 f7 = pq(s7, 2), f9 = pq(s9, 3);
          const double2 t7 = z2(-kx * f7.y - kz * f9.y, kx * f7.x + kz * f9.x);
          const double2 t = zadd(t7, mvc<BW>(tb.t1, q, r, wc[0]));
          hv(ROLE == 4 ? H_HT2 : H_HT).st(q, z2(-t.x, -t.y));
        } else if constexpr (ROLE == 2) {
          const double2 f1 = pq(0, 2), f3 = pq(2, 3), f5 = pq(4, 4);
          const double2 a1 = zadd(zscale(kxkz, zsub(f1, f3)), zscale(kz2 - kx2, f5));
          const double2 d1 = mvc<BW>(tb.t1, q, r, wc[0]), d2 = mvc<BW>(tb.t2, q, r, wc[0]);
          hv(H_G2).st(q, zadd(a1, z2(kz * d1.y, -kz * d1.x)));
          hv(H_V2).st(q, z2(-kx * d2.y, kx * d2.x));
        } else {
          const double2 d1 = mvc<BW>(tb.t1, q, r, wc[0]), d2 = mvc<BW>(tb.t2, q, r, wc[0]);
          hv(H_G3).st(q, z2(-kx * d1.y, kx * d1.x));
          hv(H_V3).st(q, z2(-kz * d2.y, kz * d2.x));
        }
        if constexpr (NC == 2) hl(d2_line).st(q, mvc<BW>(tb.t2, q, r, wc[NC - 1]));
      },
      [&](int r) {
        if constexpr (RING) {
          ring.get(r, 0, Z0.p + (r - 1) * (int)nm);
          if constexpr (NC == 2) ring.get(r, 1, Z1.p + (r - 1) * (int)nm);
          if (r <= n - 2 * BW) {
            const int q = r + BW;
            if constexpr (ROLE == 0) {
              ring.get(r, 2, pat(1, q));
              ring.get(r, 3, pat(3, q));
            } else if constexpr (SCAL) {
              ring.get(r, 2, pat(s7, q));
              ring.get(r, 3, pat(s9, q));
            } else if constexpr (ROLE == 2) {
              ring.get(r, 2, pat(0, q));
              ring.get(r, 3, pat(2, q));
              ring.get(r, 4, pat(4, q));
            }
          }
        } else {
          pf_l1(Z0.p + (r - 1) * (int)nm);
          if constexpr (NC == 2) pf_l1(Z1.p + (r - 1) * (int)nm);
          if (r <= n - 2 * BW) {
            const int q = r + BW;
            if constexpr (ROLE == 0) { pfp(1, q); pfp(3, q); }
            else if constexpr (SCAL) { pfp(s7, q); pfp(s9, q); }
            else if constexpr (ROLE == 2) { pfp(0, q); pfp(2, q); pfp(4, q); }
          }
        }
      });
}

// NS passive scalars: roles 0..3 as above, role 4 the second scalar's h_theta2.  Four resident
// blocks of one scalar's 128 threads keep 128 registers a thread; with a fifth role three blocks
// keep 136 (four would cap it at 96 and spill about 1 KB a thread).
// One scalar: up to two 32-mode groups per block (Tuning::groups); the bound keeps 128 registers.
// SA > 0 (one scalar): the staging ring of SA + 1 slots, the tables (with stab) after it.
template <int BW, typename PT, int NS, int SA = 0>
__global__ void __launch_bounds__(NS == 1 ? 2 * kLanes * kRoles : kLanes * (kRoles + 1), NS == 1 ? 2 : 3)
k_hvhg(SplitArgs a) {
  extern __shared__ double2 hvhg_smem[];
  if (a.dsc->err) return;  // uniform over the block, like a.stab
  constexpr int R = kRoles + NS - 1;
  const int role = (threadIdx.x / kLanes) % R, grp = threadIdx.x / (kLanes * R);
  const int64_t m = ((int64_t)blockIdx.x * a.groups + grp) * kLanes + (threadIdx.x % kLanes);
  const int ring_units = SA > 0 ? (SA + 1) * kHvUnits * (int)blockDim.x : 0;
  // T1, T2 and the D0 factor (L0, U0) are what the hvhg roles read: from T1 on
  const double *t1 = a.tabs + a.ny * (4 * BW + 1);
  if (a.stab) t1 = tabs_to_shared<BW>(a, 1, reinterpret_cast<double *>(hvhg_smem + ring_units));
  if (m == 0 || m >= a.nmodes) return;
  const Tabs<BW> tb = tabs_from_t1<BW>(t1, a.ny);
  const Ring<kHvUnits, SA + 1> ring{hvhg_smem + threadIdx.x, (int)blockDim.x};
  const bool s1 = a.substep == 1;
  switch (role) {
    case 0: s1 ? hvhg_role<BW, PT, 0, 2, SA>(a, tb, m, ring) : hvhg_role<BW, PT, 0, 1, SA>(a, tb, m, ring); break;
    case 1: s1 ? hvhg_role<BW, PT, 1, 2, SA>(a, tb, m, ring) : hvhg_role<BW, PT, 1, 1, SA>(a, tb, m, ring); break;
    case 2: s1 ? hvhg_role<BW, PT, 2, 2, SA>(a, tb, m, ring) : hvhg_role<BW, PT, 2, 1, SA>(a, tb, m, ring); break;
    case 3: hvhg_role<BW, PT, 3, 1, SA>(a, tb, m, ring); break;
    default:
      if constexpr (NS == 2)
        s1 ? hvhg_role<BW, PT, 4, 2, SA>(a, tb, m, ring) : hvhg_role<BW, PT, 4, 1, SA>(a, tb, m, ring);
      break;
  }
}

// ------------------------------------------------------------------------------------------
// k_helmholtz.  Every sweep stages the rows it reads through a thread-private shared-memory ring
// (Ring, cp.async SA steps ahead): the kernel's 12 warps per SM would need more L1 than there is
// to keep prefetched lines until use.  Units per step: kHelmUnits<BW>.
template <int BW>
constexpr int kHelmUnits = 5 + BW;

// FC: the operator's LU comes from the factor cache (Tuning::fcache), so the forward sweep is a
// substitution with the cached L (fwd_lband, the arithmetic of the LuSweep chains it replaces)
// and the backward sweep reads the cached U.
template <int BW, int ROLE, typename PT, int SA, bool FC = false>
__device__ __forceinline__ void helmholtz_role(const SplitArgs &a, const Tabs<BW> &tb, int64_t m,
                                               const Ring<kHelmUnits<BW>, SA + 1> &ring) {
  const int n = a.ny, s = a.substep;
  const int64_t nm = a.nmodes, ns = a.ns;
  const double dt = *a.dt_ptr, nu = a.nu;
  const double k2 = mode_k(a, m).k2;
  auto hl = [&](int i) { return DLine{a.hl + i * ns + m, nm}; };
  auto row = [&](const auto *base, int r) { return base + (r - 1) * (int)nm; };
  double *const fset = ROLE == 0 ? a.fth : a.fgp;  // (FC; roles 0 and 1 only)
  const UBand<BW> ub = FC ? make_uband<BW>(fset + a.vf_l + m, nm, ns) : role_uband<BW>(a, ROLE, m);
  const DLine Zr{a.zl + ROLE * ns + m, nm};

  // RK right-hand side (solve_g.f90:84-123): rows 1 and n are the Dirichlet rows (zero)
  auto rhs = [&](double2 store, double2 h, double2 d2, double visc, int r) {
    if (r == 1 || r == n) return z2(0.0, 0.0);
    if (s == 1) {
      const double alpha = dt * rkc(1, s) * visc, gamma = dt * rkc(3, s);
      return zadd(zadd(zscale(1.0 - alpha * k2, store), zscale(gamma, h)), zscale(alpha, d2));
    }
    return zadd(store, zscale(dt * rkc(3, s), h));
  };
  // new store (solve_g.f90:138-185): zeta' h + (1 - alpha' k2) f + alpha' D2 f, or f at s = 3
  auto store_new = [&](double2 h, double2 f, double2 d2f, double visc) {
    if (s == 3) return f;
    const double alpha = dt * rkc(1, s + 1) * visc, zeta = dt * rkc(4, s + 1);
    return zadd(zadd(zscale(zeta, h), zscale(1.0 - alpha * k2, f)), zscale(alpha, d2f));
  };

  // one complex Helmholtz solve: theta (role 0, h = HT), g (role 1, h = G2 + G3), and a second
  // scalar theta2 (role 3, h = HT2, nu / pr2)
  constexpr bool SCAL = ROLE == 0 || ROLE == 3;
  const double visc = ROLE == 0 ? nu / a.pr : ROLE == 3 ? nu / a.pr2 : nu;
  const double beta = dt * rkc(2, s) * visc;
  const double dummy = 1.0 + beta * k2;
  const int sslot = ROLE == 0 ? 2 : ROLE == 3 ? 3 : 0;
  const DLine store{a.RK + sslot * ns + m, nm};
  const DLine d2l = hl(ROLE == 0 ? H_DT : ROLE == 3 ? H_DT2 : H_DG);
  auto hv = [&](int i) { return Line<PT>{reinterpret_cast<PT *>(a.hl) + i * ns + m, nm}; };
  constexpr int hline = ROLE == 0 ? H_HT : ROLE == 3 ? H_HT2 : H_G2;
  const PT *hA = hv(hline).p, *hB = hv(H_G3).p;
  auto hsum = [&](int r) {
    if constexpr (SCAL) return hv(hline).ld(r);
    else return zadd(hv(H_G2).ld(r), hv(H_G3).ld(r));
  };
  auto rh = [&](int step, int k) { return ring_hv<PT>(ring, step, k); };
  // forward units: 0 store, 1 hA, 2 hB, 3 D2 store (substep 1); FC: 4..4+BW L(r, r-d)
  auto fin = [&](int r, double2 *bc, double *) {
    const double2 h = SCAL ? rh(r, 1) : zadd(rh(r, 1), rh(r, 2));
    bc[0] = rhs(ring.c(r, 0), h, s == 1 ? ring.c(r, 3) : z2(0.0, 0.0), visc, r);
  };
  auto fout = [&](int r, const double2 *zc, const double *) { Zr.st(r, zc[0]); };
  auto fpf = [&](int r) {
    ring.get(r, 0, row(store.p, r));
    ring.get(r, 1, row(hA, r));
    if (ROLE == 1) ring.get(r, 2, row(hB, r));
    if (s == 1) ring.get(r, 3, row(d2l.p, r));
    if constexpr (FC) {
#pragma unroll
      for (int d = 0; d <= BW; ++d) ring.get(r, 4 + d, fset + m + d * (int)ns + (r - 1) * (int)nm);
    }
  };
  if constexpr (FC) {
    const LBand<BW> fl = make_lband<BW>(fset + m, nm, ns, n);
    fwd_lband<BW, 1, 0, SA, true>([&](int r, int d) { return d <= BW ? ring.d(r, 4 + d) : fl.get(r, d); }, n, fin,
                                  fout, fpf);
  } else {
    lu_fwd<BW, 1, 0, SA, true>(n, [&](int r, double *rw, bool c) { helm_row<BW>(tb, r, n, dummy, beta, rw, c); },
                               fin, fout, ub, fpf);
  }
  // backward units: 0 Z(r), 1..BW U(r, e), BW+1 hA(q), BW+2 hB(q) with q = r + BW
  const DLine out{ROLE == 0 ? a.S + 3 * ns + m : ROLE == 3 ? a.S + 4 * ns + m : a.S + m, nm};
  bwd_emit<BW, 1, 0, SA, true>(n, [&](int r, int e) { return e <= BW ? ring.d(r, e) : ub.get(r, e); },
      [&](int r, double2 *zc, double *) { zc[0] = ring.c(r, 0); },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        const double2 f = mvc<BW>(tb.t0, q, r, wc[0]), d2f = mvc<BW>(tb.t2, q, r, wc[0]);
        out.st(q, f);
        double2 h;
        if (q == r + BW) h = SCAL ? rh(r, BW + 1) : zadd(rh(r, BW + 1), rh(r, BW + 2));
        else h = hsum(q);
        store.st(q, store_new(h, f, d2f, visc));
      },
      [&](int r) {
        ring.get(r, 0, row(Zr.p, r));
#pragma unroll
        for (int e = 1; e <= BW; ++e) ring.get(r, e, ub.p + (e - 1) * (int)ub.es + (r - 1) * (int)ub.s);
        if (r <= n - 2 * BW) {
          ring.get(r, BW + 1, row(hA, r + BW));
          if (ROLE == 1) ring.get(r, BW + 2, row(hB, r + BW));
        }
      });
}

// Role 2 of k_helmholtz: phi_p together with the unit-wall solution phi_h, then v_p together with
// v_h.  The two pairs share their operators, so each pair runs as one profile LU (lu_fwd) with a
// complex chain (the particular solution) and a real chain (the influence solution: phi_h and
// v_h have equal real and imaginary parts), and one backward sweep.
//   (alpha D0 - beta D2) phi_p = RK right-hand side,  same operator phi_h = p0 e_1
//     (solve_v_f.f90:140-153, the LU of solve_g.f90:42-71);
//   (D2 - k^2 D0) v_p = phi_p with the wall velocities at rows 1 and n, and v_h = phi_h with zero
//     walls (solve_v_f.f90:202-272).
// FC: both operators' factors are cached, and so are the influence solutions (k_helm_factor):
// each sweep carries the complex chain alone.
template <int BW, typename PT, int SA, bool FC = false>
__device__ __forceinline__ void helmholtz_phi_v(const SplitArgs &a, const Tabs<BW> &tb, int64_t m,
                                                const Ring<kHelmUnits<BW>, SA + 1> &ring) {
  const int n = a.ny, s = a.substep;
  const int64_t nm = a.nmodes, ns = a.ns;
  const double dt = *a.dt_ptr, nu = a.nu;
  const double k2 = mode_k(a, m).k2;
  auto hl = [&](int i) { return DLine{a.hl + i * ns + m, nm}; };
  auto row = [&](const auto *base, int r) { return base + (r - 1) * (int)nm; };
  const UBand<BW> ub = FC ? make_uband<BW>(a.fgp + a.vf_l + m, nm, ns) : role_uband<BW>(a, 2, m);
  const DLine Zr{a.zl + 2 * ns + m, nm};
  const RLine Xz{a.xr + m, nm}, X1{a.xinf + m, nm}, X2{a.xinf + ns + m, nm};
  const RLine X4{a.xinf + 2 * ns + m, nm}, X5{a.xinf + 3 * ns + m, nm};
  constexpr int XO = FC ? 0 : 1;  // units the influence chains take in a sweep

  const double beta = dt * rkc(2, s) * nu;
  const double dummy = 1.0 + beta * k2;
  const double p0 = dummy * trow<BW>(tb.t0, 1)[0] - beta * trow<BW>(tb.t2, 1)[0];  // A_g(1,1)
  const DLine store{a.RK + ns + m, nm};
  const DLine d2l = hl(H_DP);
  auto hv = [&](int i) { return Line<PT>{reinterpret_cast<PT *>(a.hl) + i * ns + m, nm}; };
  const PT *h0 = hv(H_HV0).p, *h1 = hv(H_V2).p, *h2 = hv(H_V3).p;
  auto hsum = [&](int r) { return zadd(hv(H_HV0).ld(r), zadd(hv(H_V2).ld(r), hv(H_V3).ld(r))); };
  auto rh = [&](int step, int k) { return ring_hv<PT>(ring, step, k); };
  // RK right-hand side of phi (solve_v_f.f90:54-97 with solve_g.f90:84-123's form); walls zero
  auto rhs = [&](double2 st, double2 h, double2 d2, int r) {
    if (r == 1 || r == n) return z2(0.0, 0.0);
    if (s == 1) {
      const double alpha = dt * rkc(1, s) * nu, gamma = dt * rkc(3, s);
      return zadd(zadd(zscale(1.0 - alpha * k2, st), zscale(gamma, h)), zscale(alpha, d2));
    }
    return zadd(st, zscale(dt * rkc(3, s), h));
  };
  auto store_new = [&](double2 h, double2 f, double2 d2f) {
    if (s == 3) return f;
    const double alpha = dt * rkc(1, s + 1) * nu, zeta = dt * rkc(4, s + 1);
    return zadd(zadd(zscale(zeta, h), zscale(1.0 - alpha * k2, f)), zscale(alpha, d2f));
  };
  // phi forward units: 0 store, 1..3 HV0, V2, V3, 4 D2 store (substep 1).  FC: 4..4+BW
  // L(r, r-d) of the cached factor instead, and the D2 store (substep 1) prefetched into L1
  if constexpr (FC) {
    const LBand<BW> fl = make_lband<BW>(a.fgp + m, nm, ns, n);
    fwd_lband<BW, 1, 0, SA, true>([&](int r, int d) { return d <= BW ? ring.d(r, 4 + d) : fl.get(r, d); }, n,
        [&](int r, double2 *bc, double *) {
          const double2 h = zadd(rh(r, 1), zadd(rh(r, 2), rh(r, 3)));
          bc[0] = rhs(ring.c(r, 0), h, s == 1 ? d2l.ld(r) : z2(0.0, 0.0), r);
        },
        [&](int r, const double2 *zc, const double *) { Zr.st(r, zc[0]); },
        [&](int r) {
          ring.get(r, 0, row(store.p, r));
          ring.get(r, 1, row(h0, r));
          ring.get(r, 2, row(h1, r));
          ring.get(r, 3, row(h2, r));
          if (s == 1) pf_l1(row(d2l.p, r));
#pragma unroll
          for (int d = 0; d <= BW; ++d) ring.get(r, 4 + d, a.fgp + m + d * (int)ns + (r - 1) * (int)nm);
        });
  } else {
    lu_fwd<BW, 1, 1, SA, true>(n, [&](int r, double *rw, bool c) { helm_row<BW>(tb, r, n, dummy, beta, rw, c); },
        [&](int r, double2 *bc, double *br) {
          const double2 h = zadd(rh(r, 1), zadd(rh(r, 2), rh(r, 3)));
          bc[0] = rhs(ring.c(r, 0), h, s == 1 ? ring.c(r, 4) : z2(0.0, 0.0), r);
          br[0] = (r == 1) ? p0 : 0.0;
        },
        [&](int r, const double2 *zc, const double *zr) {
          Zr.st(r, zc[0]);
          Xz.st(r, zr[0]);
        },
        ub,
        [&](int r) {
          ring.get(r, 0, row(store.p, r));
          ring.get(r, 1, row(h0, r));
          ring.get(r, 2, row(h1, r));
          ring.get(r, 3, row(h2, r));
          if (s == 1) ring.get(r, 4, row(d2l.p, r));
        });
  }
  // phi backward units: 0 Z(r), 1 Xz(r), 2..BW+1 U(r, e), BW+2..BW+4 HV0, V2, V3 at q = r + BW
  // (FC: no Xz, the others one unit lower)
  const DLine out{a.zl + 4 * ns + m, nm};
  bwd_emit<BW, 1, FC ? 0 : 1, SA, true>(n, [&](int r, int e) { return e <= BW ? ring.d(r, XO + e) : ub.get(r, e); },
      [&](int r, double2 *zc, double *zr) {
        zc[0] = ring.c(r, 0);
        if constexpr (!FC) zr[0] = ring.d(r, 1);
      },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&wr)[1][2 * BW + 1]) {
        const double2 f = mvc<BW>(tb.t0, q, r, wc[0]), d2f = mvc<BW>(tb.t2, q, r, wc[0]);
        out.st(q, f);
        const double2 h = (q == r + BW) ? zadd(rh(r, BW + 1 + XO), zadd(rh(r, BW + 2 + XO), rh(r, BW + 3 + XO)))
                                        : hsum(q);
        store.st(q, store_new(h, f, d2f));
        if constexpr (!FC) {
          X1.st(q, mvr<BW>(tb.t0, q, r, wr[0]));  // phi_h (real part = imaginary part)
          X2.st(q, mvr<BW>(tb.t2, q, r, wr[0]));  // D2 phi_h
        }
      },
      [&](int r) {
        ring.get(r, 0, row(Zr.p, r));
        if constexpr (!FC) ring.get(r, 1, row(Xz.p, r));
#pragma unroll
        for (int e = 1; e <= BW; ++e) ring.get(r, XO + e, ub.p + (e - 1) * (int)ub.es + (r - 1) * (int)ub.s);
        if (r <= n - 2 * BW) {
          ring.get(r, BW + 1 + XO, row(h0, r + BW));
          ring.get(r, BW + 2 + XO, row(h1, r + BW));
          ring.get(r, BW + 3 + XO, row(h2, r + BW));
        }
      });
  // (D2 - k^2 D0) v = phi with v_p = the wall velocity at rows 1 and n, v_h = 0 there.
  // Opposition control, the extension at the wall rows of the v solve (solve_v_f.f90:251-257,
  // whose commented lines read vold): v at the walls = A * gain * v(+-y_d).  vold is field 10,
  // v after the physical round trip (dft_x_realspace.f90:123), which has no kz Nyquist mode
  // and, at kx = 0, only the Hermitian part (v(kz) + conj v(-kz)) / 2.
  double2 vlo = z2(0.0, 0.0), vhi = z2(0.0, 0.0);
  if (a.control_amp != 0.0) {
    const int kzi = (int)(m / a.nxh), kxi = (int)(m - (int64_t)kzi * a.nxh);
    if (kzi != a.nz / 2) {
      vlo = a.vwall[m];
      vhi = a.vwall[nm + m];
      if (kxi == 0) {
        const int64_t mp = (int64_t)((a.nz - kzi) % a.nz) * a.nxh;
        const double2 pl = a.vwall[mp], ph = a.vwall[nm + mp];
        vlo = z2(0.5 * (vlo.x + pl.x), 0.5 * (vlo.y - pl.y));
        vhi = z2(0.5 * (vhi.x + ph.x), 0.5 * (vhi.y - ph.y));
      }
      const double gmul = a.control_amp * (double)__ldg(a.gains + m);
      vlo = zscale(gmul, vlo);
      vhi = zscale(gmul, vhi);
    }
  }
  // the v operator does not change during a run: its factors come from k_vop_factor
  const LBand<BW> vl = make_lband<BW>(a.vf + m, nm, ns, n);
  const UBand<BW> vu = make_uband<BW>(a.vf + a.vf_l + m, nm, ns);
  // v forward units: 0 phi_p(r), 1 phi_h(r), 2..BW+2 L(r, r-d) for d = 0..BW (FC: no phi_h)
  fwd_lband<BW, 1, FC ? 0 : 1, SA, true>(
      [&](int r, int d) { return d <= BW ? ring.d(r, 1 + XO + d) : vl.get(r, d); }, n,
      [&](int r, double2 *bc, double *br) {
        const bool wall = (r == 1 || r == n);
        bc[0] = (r == 1) ? vlo : (r == n) ? vhi : ring.c(r, 0);
        if constexpr (!FC) br[0] = wall ? 0.0 : ring.d(r, 1);
      },
      [&](int r, const double2 *zc, const double *zr) {
        Zr.st(r, zc[0]);
        if constexpr (!FC) Xz.st(r, zr[0]);
      },
      [&](int r) {
        ring.get(r, 0, row(out.p, r));
        if constexpr (!FC) ring.get(r, 1, row(X1.p, r));
#pragma unroll
        for (int d = 0; d <= BW; ++d) ring.get(r, 1 + XO + d, vl.p + d * (int)ns + (r - 1) * (int)nm);
      });
  // v backward units: 0 Z(r), 1 Xz(r), 2..BW+1 U(r, e) (FC: no Xz)
  const DLine Sv{a.S + ns + m, nm}, Sw{a.S + 2 * ns + m, nm};
  double dh1 = 0.0, dhn = 0.0;
  bwd_emit<BW, 1, FC ? 0 : 1, SA, true>(n, [&](int r, int e) { return e <= BW ? ring.d(r, XO + e) : vu.get(r, e); },
      [&](int r, double2 *zc, double *zr) {
        zc[0] = ring.c(r, 0);
        if constexpr (!FC) zr[0] = ring.d(r, 1);
      },
      [&](int q, int r, const double2 (&wc)[1][2 * BW + 1], const double (&wr)[1][2 * BW + 1]) {
        const double2 vp = mvc<BW>(tb.t0, q, r, wc[0]), dvp = mvc<BW>(tb.t1, q, r, wc[0]);
        Sv.st(q, vp);
        Sw.st(q, dvp);
        if (q == 1) a.dv[m] = dvp;
        if (q == n) a.dv[nm + m] = dvp;
        if constexpr (!FC) {
          const double vh = mvr<BW>(tb.t0, q, r, wr[0]), dvh = mvr<BW>(tb.t1, q, r, wr[0]);
          X4.st(q, vh);
          X5.st(q, dvh);
          if (q == 1) dh1 = dvh;
          if (q == n) dhn = dvh;
        }
      },
      [&](int r) {
        ring.get(r, 0, row(Zr.p, r));
        if constexpr (!FC) ring.get(r, 1, row(Xz.p, r));
#pragma unroll
        for (int e = 1; e <= BW; ++e) ring.get(r, XO + e, vu.p + (e - 1) * (int)vu.es + (r - 1) * (int)vu.s);
      });
  if constexpr (!FC) a.dvh[m] = z2(dh1, dhn);
}

// The profile LU of the v operator (D2 - k^2 D0 with Dirichlet first and last rows, the matrix
// of solve_v_f.f90:202-231) of every mode, once per handle: it depends on k^2 alone.  Same
// LuSweep arithmetic as a per-substep factorisation, so the factors are the same numbers.
template <int BW>
__global__ void __launch_bounds__(128) k_vop_factor(SplitArgs a) {
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= a.nmodes) return;
  const int n = a.ny;
  const Tabs<BW> tb = tabs_at<BW>(a.tabs, n);
  const double k2 = mode_k(a, m).k2;
  const LBand<BW> lb = make_lband<BW>(a.vf + m, a.nmodes, a.ns, n);
  LuSweep<BW, 0, 0, true> lu;
  lu.init(n, make_uband<BW>(a.vf + a.vf_l + m, a.nmodes, a.ns));
  for (int r = 1; r <= n; ++r) {
    double2 bc[1] = {z2(0.0, 0.0)}, zc[1];
    double br[1] = {0.0}, zr[1];
    lu.step(r, [&](int rr, double *row, bool c) { vrow<BW>(tb, rr, n, k2, row, c); }, bc, br, zc, zr);
#pragma unroll
    for (int d = 0; d <= 2 * BW; ++d) lb.set(r, d, lu.Lk[d]);
  }
}

// Three roles per mode: theta, g, and phi with v (helmholtz_phi_v); a fourth for a second scalar.
constexpr int kHelmRoles = 3;

// Staging ring bytes of one 32-mode group (NS scalars, SA steps of look-ahead).
template <int BW, int NS = 1, int SA = 1>
constexpr size_t helm_smem() {
  return sizeof(double2) * (size_t)(SA + 1) * kHelmUnits<BW> * kLanes * (kHelmRoles + NS - 1);
}

// With a fourth role (a second scalar) three resident blocks keep the 168 registers of one
// scalar's kernel; four would cap it at 128 and spill.
// One scalar: 1, 2 or 4 32-mode groups per block (Tuning::hgroups) and 1 or 2 steps of staging
// look-ahead (Tuning::stage); the bound (384 threads) keeps 168 registers.  Four groups with the
// tables in shared memory and two steps of look-ahead hold 218 KB at ny = 129, one block (12
// warps) per SM.
// FC (one scalar): the sweeps read the factor cache that k_helm_factor filled for this dt, and
// the kernel records that dt as the one the cache holds.
template <int BW, typename PT, int NS, int SA, bool FC = false>
__global__ void __launch_bounds__(4 * kLanes * kHelmRoles, 1) k_helmholtz(SplitArgs a) {
  extern __shared__ double2 helm_ring[];
  if (a.dsc->err) return;  // a failed dt update leaves the state untouched (uniform over the block)
  if constexpr (FC) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.fcdt = *a.dt_ptr;  // read by the next k_helm_factor only
  }
  constexpr int R = kHelmRoles + NS - 1;
  const int role = (threadIdx.x / kLanes) % R, grp = threadIdx.x / (kLanes * R);
  const int64_t m = ((int64_t)blockIdx.x * a.hgroups + grp) * kLanes + (threadIdx.x % kLanes);
  // T0, T1, T2 (after the staging ring when in shared memory)
  const double *t0 = a.tabs;
  if (a.hstab)
    t0 = tabs_to_shared<BW>(a, 0, reinterpret_cast<double *>(helm_ring + (SA + 1) * kHelmUnits<BW> * blockDim.x));
  if (m == 0 || m >= a.nmodes) return;
  const Tabs<BW> tb = tabs_at<BW>(t0, a.ny);  // (its L0 and U0 are not read here)
  const Ring<kHelmUnits<BW>, SA + 1> ring{helm_ring + threadIdx.x, (int)blockDim.x};
  switch (role) {
    case 0: helmholtz_role<BW, 0, PT, SA, FC>(a, tb, m, ring); break;
    case 1: helmholtz_role<BW, 1, PT, SA, FC>(a, tb, m, ring); break;
    case 2: helmholtz_phi_v<BW, PT, SA, FC>(a, tb, m, ring); break;
    default:
      if constexpr (NS == 2 && !FC) helmholtz_role<BW, 3, PT, SA>(a, tb, m, ring);
      break;
  }
}

// The factor cache of a substep with a fixed time step (Tuning::fcache), for every mode: the
// profile LU of theta's operator and of the one g and phi share (alpha D0 - beta D2 with the
// Dirichlet rows), and the influence solutions phi_h (through that LU) and v_h (through the v
// operator's factors) with their emitted lines, as k_helmholtz computes them otherwise: the same
// LuSweep arithmetic, so the same numbers.  A no-op while the cache holds this dt; with a
// fixed time step it runs once per substep of the run (and again after a change of dt).
template <int BW>
__global__ void __launch_bounds__(128) k_helm_factor(SplitArgs a) {
  if (a.dsc->err || *a.fcdt == *a.dt_ptr) return;
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0 || m >= a.nmodes) return;
  const int n = a.ny, s = a.substep;
  const int64_t nm = a.nmodes, ns = a.ns;
  const Tabs<BW> tb = tabs_at<BW>(a.tabs, n);
  const double dt = *a.dt_ptr, k2 = mode_k(a, m).k2;
  const double2 zero[1] = {z2(0.0, 0.0)};
  double2 zc[1];
  double zr[1];
  {  // theta: nu / pr (solve_t.f90:42-71)
    const double beta = dt * rkc(2, s) * (a.nu / a.pr), dummy = 1.0 + beta * k2;
    const LBand<BW> lb = make_lband<BW>(a.fth + m, nm, ns, n);
    LuSweep<BW, 0, 0, true> lu;
    lu.init(n, make_uband<BW>(a.fth + a.vf_l + m, nm, ns));
    for (int r = 1; r <= n; ++r) {
      const double br[1] = {0.0};
      lu.step(r, [&](int rr, double *row, bool c) { helm_row<BW>(tb, rr, n, dummy, beta, row, c); }, zero, br, zc, zr);
#pragma unroll
      for (int d = 0; d <= 2 * BW; ++d) lb.set(r, d, lu.Lk[d]);
    }
  }
  // g and phi: nu (solve_g.f90:42-71, solve_v_f.f90:140-153), with phi_h = p0 e_1 through it
  const RLine Xz{a.xr + m, nm};
  const RLine X1{a.xinf + m, nm}, X2{a.xinf + ns + m, nm}, X4{a.xinf + 2 * ns + m, nm}, X5{a.xinf + 3 * ns + m, nm};
  {
    const double beta = dt * rkc(2, s) * a.nu, dummy = 1.0 + beta * k2;
    const double p0 = dummy * trow<BW>(tb.t0, 1)[0] - beta * trow<BW>(tb.t2, 1)[0];  // A_g(1,1)
    const LBand<BW> lb = make_lband<BW>(a.fgp + m, nm, ns, n);
    LuSweep<BW, 0, 1, true> lu;
    lu.init(n, make_uband<BW>(a.fgp + a.vf_l + m, nm, ns));
    for (int r = 1; r <= n; ++r) {
      const double br[1] = {(r == 1) ? p0 : 0.0};
      lu.step(r, [&](int rr, double *row, bool c) { helm_row<BW>(tb, rr, n, dummy, beta, row, c); }, zero, br, zc, zr);
#pragma unroll
      for (int d = 0; d <= 2 * BW; ++d) lb.set(r, d, lu.Lk[d]);
      Xz.st(r, zr[0]);
    }
  }
  const UBand<BW> ug = make_uband<BW>(a.fgp + a.vf_l + m, nm, ns);
  bwd_emit<BW, 0, 1>(n, [&](int r, int e) { return ug.get(r, e); },
      [&](int r, double2 *, double *z) { z[0] = Xz.ld(r); },
      [&](int q, int r, const double2 (&)[1][2 * BW + 1], const double (&wr)[1][2 * BW + 1]) {
        X1.st(q, mvr<BW>(tb.t0, q, r, wr[0]));  // phi_h
        X2.st(q, mvr<BW>(tb.t2, q, r, wr[0]));  // D2 phi_h
      });
  // v_h: (D2 - k^2 D0) v_h = phi_h with v_h = 0 at the walls (solve_v_f.f90:202-272)
  const LBand<BW> vl = make_lband<BW>(a.vf + m, nm, ns, n);
  const UBand<BW> vu = make_uband<BW>(a.vf + a.vf_l + m, nm, ns);
  fwd_lband<BW, 0, 1>([&](int r, int d) { return vl.get(r, d); }, n,
      [&](int r, double2 *, double *b) { b[0] = (r == 1 || r == n) ? 0.0 : X1.ld(r); },
      [&](int r, const double2 *, const double *z) { Xz.st(r, z[0]); });
  double dh1 = 0.0, dhn = 0.0;
  bwd_emit<BW, 0, 1>(n, [&](int r, int e) { return vu.get(r, e); },
      [&](int r, double2 *, double *z) { z[0] = Xz.ld(r); },
      [&](int q, int r, const double2 (&)[1][2 * BW + 1], const double (&wr)[1][2 * BW + 1]) {
        const double vh = mvr<BW>(tb.t0, q, r, wr[0]), dvh = mvr<BW>(tb.t1, q, r, wr[0]);
        X4.st(q, vh);
        X5.st(q, dvh);
        if (q == 1) dh1 = dvh;
        if (q == n) dhn = dvh;
      });
  a.dvh[m] = z2(dh1, dhn);
}

// ------------------------------------------------------------------------------------------
// k_assemble: one thread per (y, mode); grid (modes / 256, ny).
__global__ void __launch_bounds__(512) k_assemble(SplitArgs a) {
  if (a.dsc->err) return;
  const int64_t nm = a.nmodes, ns = a.ns;
  const int r = blockIdx.y + 1;
  const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (m == 0 || m >= nm) return;
  const int n = a.ny, s = a.substep, rr = n + 1 - r;
  const ModeK k = mode_k(a, m);
  // C1, C2 (solve_v_f.f90:293-294); the homogeneous derivative is dvh * (1 + i)
  const double2 dvh = a.dvh[m];
  const double2 h1 = z2(dvh.x, dvh.x), hn = z2(dvh.y, dvh.y);
  const double2 d1 = a.dv[m], dn = a.dv[nm + m];
  const double2 den = zsub(zmul(h1, h1), zmul(hn, hn));
  const double2 C1 = zdiv(zsub(zmul(hn, dn), zmul(h1, d1)), den);
  const double2 C2 = zdiv(zsub(zmul(h1, dn), zmul(hn, d1)), den);
  const double2 C1c = z2(C1.x - C1.y, C1.x + C1.y), C2c = z2(C2.x - C2.y, C2.x + C2.y);  // C * (1 + i)
  double cd = 1.0, ca = 0.0;
  if (s != 3) {
    const double alpha = *a.dt_ptr * a.nu * rkc(1, s + 1);
    cd = 1.0 - alpha * k.k2;
    ca = alpha;
  }
  const double *xr = a.xinf + m;  // phi_h, D2 phi_h, v_h, dv_h / dy
  auto X = [&](int i, int row) { return xr[(i - 1) * ns + (row - 1) * (int)nm]; };
  const int64_t o = (r - 1) * (int)nm + m;
  double2 *S = a.S, *Rp = a.RK + ns;
  const double2 v = zadd(zadd(S[ns + o], zscale(X(3, r), C1c)), zscale(X(3, rr), C2c));
  const double2 dv = zsub(zadd(S[2 * ns + o], zscale(X(4, r), C1c)), zscale(X(4, rr), C2c));
  double2 sp = Rp[o];
  sp = zadd(sp, zscale(cd * X(1, r), C1c));
  sp = zadd(sp, zscale(cd * X(1, rr), C2c));
  if (s != 3) {
    sp = zadd(sp, zscale(ca * X(2, r), C1c));
    sp = zadd(sp, zscale(ca * X(2, rr), C2c));
  }
  Rp[o] = sp;
  const double2 kxx = z2(0.0, k.kx / k.k2), kzz = z2(0.0, k.kz / k.k2);
  const double2 g = S[o];
  S[o] = zsub(zmul(kxx, dv), zmul(kzz, g));  // solve_u_w.f90:27-38
  S[ns + o] = v;
  S[2 * ns + o] = zadd(zmul(kxx, g), zmul(kzz, dv));
}

// ------------------------------------------------------------------------------------------
// k_mean: wave00.f90 for one mean line per thread: U (line 0: forced, Galilean shift),
// W (line 1: phi = 0), Theta (line 2: nu/pr, forced to the bulk value).
struct MeanArgs {
  int ny, substep, nsc;
  int64_t nmodes, ns;
  double2 *S, *RK;
  const void *P;
  double *w00;
  const double *tabs, *integ;
  double nu, pr, bulk_u, bulk_w, bulk_t, u_gal;
  double pr2, bulk_t2;  // a second passive scalar (line 3)
  DevScalars *dsc;
  const double *dt_ptr;
};

template <int BW, typename PT>
__global__ void k_mean(MeanArgs a) {
  const int line = threadIdx.x;
  if (line >= 2 + a.nsc || a.dsc->err) return;
  const Tabs<BW> tb = tabs_at<BW>(a.tabs, a.ny);
  const int n = a.ny, s = a.substep;
  const int64_t ns = a.ns;
  const double dt = *a.dt_ptr;
  // line 3: a second passive scalar, the theta block with its own Prandtl number and bulk value
  const double visc = (line == 2) ? a.nu / a.pr : (line == 3) ? a.nu / a.pr2 : a.nu;
  const double gal = (line == 0) ? a.u_gal : 0.0;
  const double bulk = (line == 0) ? a.bulk_u : (line == 1) ? a.bulk_w : (line == 2) ? a.bulk_t : a.bulk_t2;
  const int pslot = (line == 0) ? 1 : (line == 1) ? 3 : (line == 2) ? 6 : 9;  // uv, vw, v theta, v theta2
  const PT *P = reinterpret_cast<const PT *>(a.P) + pslot * ns;
  const DLine store{a.RK + line * ns, a.nmodes};
  const DLine out{a.S + (line == 0 ? 0 : line == 1 ? 2 : line == 2 ? 3 : 4) * ns, a.nmodes};
  const int64_t per = 8 * (int64_t)n + 2 * BW * (int64_t)n;  // doubles per line thread
  double *base = a.w00 + line * per;
  const DLine Zf{reinterpret_cast<double2 *>(base), 1}, Zs{reinterpret_cast<double2 *>(base) + n, 1};
  const DLine R{reinterpret_cast<double2 *>(base) + 2 * n, 1}, DF{reinterpret_cast<double2 *>(base) + 3 * n, 1};
  const UBand<BW> ub = make_uband<BW>(base + 8 * (int64_t)n, 1, n);
  auto ufix = [&](int r, int e) { return tb.u0[(r - 1) * 2 * BW + e - 1]; };
  // D0 solves: the flux product (and the store at substep 1)
  fwd_fixed<BW, 2>(tb, n,
      [&](int r, double2 *b) {
        b[0] = ldp<PT>(P + (r - 1) * (int)a.nmodes);
        b[1] = (s == 1) ? store.ld(r) : z2(0.0, 0.0);
      },
      [&](int r, const double2 *z) { Zf.st(r, z[0]); Zs.st(r, z[1]); },
      [&](int r) {
        pf_l1(P + (r - 1) * (int)a.nmodes);
        pf_l1(store.p + (r - 1) * (int)a.nmodes);
      });
  auto pfw = [&](const DLine &l, int r) { pf_l1(l.p + (r - 1)); };
  bwd_emit<BW, 2, 0>(n, ufix,
      [&](int r, double2 *zc, double *) { zc[0] = Zf.ld(r); zc[1] = Zs.ld(r); },
      [&](int q, int r, const double2 (&wc)[2][2 * BW + 1], const double (&)[1][2 * BW + 1]) {
        const double2 d = mvc<BW>(tb.t1, q, r, wc[0]);  // d/dy of the flux
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
      },
      [&](int r) {
        pfw(Zf, r);
        pfw(Zs, r);
        if (r <= n - 2 * BW) pf_l1(store.p + (r + BW - 1) * (int)a.nmodes);
      });
  // (D0 - beta D2) c = rhs, Dirichlet rows
  const double beta = dt * rkc(2, s) * visc;
  lu_fwd<BW, 1, 0>(n, [&](int r, double *row, bool c) { helm_row<BW>(tb, r, n, 1.0, beta, row, c); },
      [&](int r, double2 *bc, double *) { bc[0] = R.ld(r); },
      [&](int r, const double2 *zc, const double *) { R.st(r, zc[0]); }, ub, [&](int r) { pfw(R, r); });
  // backward substitution storing the coefficients; the integral (LABS_integration) runs along,
  // summed from row n down
  double2 integral = z2(0.0, 0.0);
  {
    double2 w[2 * BW + 1];
#pragma unroll
    for (int j = 0; j <= 2 * BW; ++j) w[j] = z2(0.0, 0.0);
    for (int r = n; r >= 1; --r) {
      if (r > kPrefetchRows) {
        pfw(R, r - kPrefetchRows);
#pragma unroll
        for (int e = 1; e <= BW; ++e) pf_l1(ub.p + (e - 1) * (int)n + (r - kPrefetchRows - 1));
      }
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
      integral = zadd(integral, zscale(__ldg(a.integ + r - 1), acc));
    }
  }
  double phi = (bulk - 0.5 * integral.x) / (0.5 * integral.y);  // calculate_phi
  if (line == 1) phi = 0.0;                                       // wave00.f90:396
  // c = Re c + phi Im c (real), formed where it is read: the wall stresses and the last sweep
  auto creal = [&](int r) {
    const double2 c = R.ld(r);
    return c.x + phi * c.y;
  };
  if (s == 3) {
    const double *r1 = trow<BW>(tb.t1, 1), *rn = trow<BW>(tb.t1, n);
    const double wall = r1[0] * creal(1) + r1[1] * creal(2) - rn[-1] * creal(n - 1) - rn[0] * creal(n);
    if (line == 0) a.dsc->wall_shear_stress = 0.5 * a.nu * wall;
    if (line == 2) a.dsc->wall_theta_stress = 0.5 * a.nu / a.pr * wall;
    if (line == 3) a.dsc->wall_theta_stress2 = 0.5 * a.nu / a.pr2 * wall;
  }
  if (line == 0) a.dsc->phi_dpdx[s - 1] = phi;
  if (line == 2) a.dsc->phi_dtdx[s - 1] = phi;
  if (line == 3) a.dsc->phi_dtdx2[s - 1] = phi;
  bwd_emit<BW, 1, 0>(n, [&](int, int) { return 0.0; },
      [&](int r, double2 *zc, double *) { zc[0] = z2(creal(r), 0.0); },
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
      },
      [&](int r) {
        pfw(R, r);
        if (r <= n - 2 * BW) pfw(DF, r + BW);
      });
  if (line == 1) {  // v mean = 0 (wave00.f90:462)
    const DLine Sv{a.S + ns, a.nmodes};
    for (int r = 1; r <= n; ++r) Sv.st(r, z2(0.0, 0.0));
  }
}

// part 0: fork the mean lines to h.side, then k_hvhg; part 1: k_helmholtz; part 2: k_assemble,
// then join h.side back to st.
template <int BW>
cudaError_t split_bw(Handle &h, int part, int substep, const double *dt_ptr, cudaStream_t st) {
  const OpsOffsets off = ops_offsets(h.bw, h.ny);
  const double *dtp = dt_ptr ? dt_ptr : &h.dsc->dt;
  SplitArgs a;
  a.ny = h.ny;
  a.nxh = h.nxh;
  a.nz = h.nz;
  a.substep = substep;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.S = h.S;
  a.RK = h.RK;
  a.P = h.P;
  a.zl = h.zc;
  a.hl = h.ec;
  a.xr = h.xr;
  a.ub = h.ub;
  a.ub_role = split_ub_role(h);
  a.dv = h.dvw;
  a.tabs = h.dops + off.t0;
  a.vwall = h.vwall;
  a.wlo = h.dops + off.wlo;
  a.whi = h.dops + off.whi;
  a.gains = h.gains;
  a.control_amp = h.cfg.control_amp;
  a.nu = h.cfg.nu;
  a.pr = h.cfg.pr;
  a.pr2 = h.cfg.pr2;
  a.lmfxr = h.lmfxr;
  a.lmfzr = h.lmfzr;
  a.dsc = h.dsc;
  a.dt_ptr = dtp;
  a.vf = h.vf;
  a.vf_l = vop_lband_doubles(h);
  a.groups = h.nsc == 1 ? h.tune.groups : 1;
  a.hgroups = h.tune.hgroups;
  a.ulayout = h.tune.ulayout;
  a.stab = h.tune.stab;
  a.hstab = h.tune.hstab;
  const bool fc = h.tune.fcache && h.hf;
  const int64_t fset = vop_factor_doubles(h);
  a.fth = fc ? h.hf + 2 * (int64_t)(substep - 1) * fset : nullptr;
  a.fgp = fc ? a.fth + fset : nullptr;
  a.fcdt = fc ? h.fcdt + (substep - 1) : nullptr;
  a.xinf = fc ? h.hinf + 4 * (int64_t)(substep - 1) * h.ns : h.xr + h.ns;
  a.dvh = fc ? h.hdvh + (int64_t)(substep - 1) * h.nmodes : h.dvw + 2 * h.nmodes;

  MeanArgs ma;
  ma.ny = h.ny;
  ma.substep = substep;
  ma.nsc = h.nsc;
  ma.pr2 = h.cfg.pr2;
  ma.bulk_t2 = h.cfg.bulk_t2;
  ma.nmodes = h.nmodes;
  ma.ns = h.ns;
  ma.S = h.S;
  ma.RK = h.RK;
  ma.P = h.P;
  ma.w00 = h.w00;
  ma.tabs = a.tabs;
  ma.integ = h.dops + off.integ;
  ma.nu = h.cfg.nu;
  ma.pr = h.cfg.pr;
  ma.bulk_u = h.cfg.bulk_vel_u;
  ma.bulk_w = h.cfg.bulk_vel_w;
  ma.bulk_t = h.cfg.bulk_t;
  ma.u_gal = h.cfg.u_gal;
  ma.dsc = h.dsc;
  ma.dt_ptr = dtp;

  cudaError_t e;
  const int G = a.groups;
  const unsigned blocks = (unsigned)((h.nmodes + (int64_t)kLanes * G - 1) / ((int64_t)kLanes * G));
  const size_t tsm = a.stab ? solver_tables_bytes(h) : 0, htsm = a.hstab ? solver_tables_bytes(h) : 0;
  if (part == 0) {
    // the mean lines touch only mode 0, which the split kernels skip: run them beside those
    if ((e = cudaEventRecord(h.ev_fork, st)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(h.side, h.ev_fork, 0)) != cudaSuccess) return e;
    if (h.mixed) k_mean<BW, float2><<<1, 32, 0, h.side>>>(ma);
    else k_mean<BW, double2><<<1, 32, 0, h.side>>>(ma);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaEventRecord(h.ev_join, h.side)) != cudaSuccess) return e;
    if (h.nsc == 2) {
      if (h.mixed) k_hvhg<BW, float2, 2><<<blocks, kLanes * (kRoles + 1), tsm, st>>>(a);
      else k_hvhg<BW, double2, 2><<<blocks, kLanes * (kRoles + 1), tsm, st>>>(a);
    } else {
      const int nt = kLanes * kRoles * G, sa = h.tune.hvstage;
      const size_t sm = (sa > 0 ? sizeof(double2) * (size_t)(sa + 1) * kHvUnits * nt : 0) + tsm;
      if (sa == 2) {
        if (h.mixed) k_hvhg<BW, float2, 1, 2><<<blocks, nt, sm, st>>>(a);
        else k_hvhg<BW, double2, 1, 2><<<blocks, nt, sm, st>>>(a);
      } else if (sa == 1) {
        if (h.mixed) k_hvhg<BW, float2, 1, 1><<<blocks, nt, sm, st>>>(a);
        else k_hvhg<BW, double2, 1, 1><<<blocks, nt, sm, st>>>(a);
      } else {
        if (h.mixed) k_hvhg<BW, float2, 1><<<blocks, nt, sm, st>>>(a);
        else k_hvhg<BW, double2, 1><<<blocks, nt, sm, st>>>(a);
      }
    }
    return cudaGetLastError();
  }
  if (part == 1) {
    if (h.nsc == 2) {
      const int HG = a.hgroups;
      const unsigned hb = (unsigned)((h.nmodes + (int64_t)kLanes * HG - 1) / ((int64_t)kLanes * HG));
      const int nt = kLanes * (kHelmRoles + 1) * HG;
      const size_t sm = HG * helm_smem<BW, 2>() + htsm;
      if (h.mixed) k_helmholtz<BW, float2, 2, 1><<<hb, nt, sm, st>>>(a);
      else k_helmholtz<BW, double2, 2, 1><<<hb, nt, sm, st>>>(a);
    } else {
      const int HG = a.hgroups;
      const unsigned hb = (unsigned)((h.nmodes + (int64_t)kLanes * HG - 1) / ((int64_t)kLanes * HG));
      const int nt = kLanes * kHelmRoles * HG;
      if (fc) {
        k_helm_factor<BW><<<(unsigned)((h.nmodes + 127) / 128), 128, 0, st>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
      }
      if (h.tune.stage == 2) {
        const size_t sm = HG * helm_smem<BW, 1, 2>() + htsm;
        if (fc) {
          if (h.mixed) k_helmholtz<BW, float2, 1, 2, true><<<hb, nt, sm, st>>>(a);
          else k_helmholtz<BW, double2, 1, 2, true><<<hb, nt, sm, st>>>(a);
        } else {
          if (h.mixed) k_helmholtz<BW, float2, 1, 2><<<hb, nt, sm, st>>>(a);
          else k_helmholtz<BW, double2, 1, 2><<<hb, nt, sm, st>>>(a);
        }
      } else {
        const size_t sm = HG * helm_smem<BW>() + htsm;
        if (fc) {
          if (h.mixed) k_helmholtz<BW, float2, 1, 1, true><<<hb, nt, sm, st>>>(a);
          else k_helmholtz<BW, double2, 1, 1, true><<<hb, nt, sm, st>>>(a);
        } else {
          if (h.mixed) k_helmholtz<BW, float2, 1, 1><<<hb, nt, sm, st>>>(a);
          else k_helmholtz<BW, double2, 1, 1><<<hb, nt, sm, st>>>(a);
        }
      }
    }
    return cudaGetLastError();
  }
  const int at = h.tune.asm_threads;
  const dim3 agrid((unsigned)((h.nmodes + at - 1) / at), (unsigned)h.ny);
  k_assemble<<<agrid, at, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t split_part(Handle &h, int part, int substep, const double *dt_ptr, cudaStream_t st) {
  switch (h.bw) {
    case 2: return split_bw<2>(h, part, substep, dt_ptr, st);
    case 3: return split_bw<3>(h, part, substep, dt_ptr, st);
    case 4: return split_bw<4>(h, part, substep, dt_ptr, st);
    case 5: return split_bw<5>(h, part, substep, dt_ptr, st);
    case 6: return split_bw<6>(h, part, substep, dt_ptr, st);
    case 7: return split_bw<7>(h, part, substep, dt_ptr, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

int64_t split_ub_role(const Handle &h) {
  return (int64_t)h.bw * h.ns + (int64_t)h.bw * h.bw * h.nmodes;
}

int64_t vop_lband_doubles(const Handle &h) {
  return (int64_t)(h.bw + 1) * h.ns + (int64_t)h.bw * h.bw * h.nmodes;
}

int64_t vop_factor_doubles(const Handle &h) { return vop_lband_doubles(h) + split_ub_role(h); }

bool factor_cache_possible(const Handle &h) { return h.cfg.fixed_dt != 0 && h.nsc == 1; }

namespace {

template <int BW>
cudaError_t set_smem_limit_bw(int bytes) {
  auto lim = [bytes](auto kern) { return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes); };
  cudaError_t e = lim(k_helmholtz<BW, float2, 1, 1>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, double2, 1, 1>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, float2, 1, 2>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, double2, 1, 2>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, float2, 1, 1, true>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, double2, 1, 1, true>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, float2, 1, 2, true>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, double2, 1, 2, true>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, float2, 2, 1>);
  if (e == cudaSuccess) e = lim(k_helmholtz<BW, double2, 2, 1>);
  if (e == cudaSuccess) e = lim(k_hvhg<BW, float2, 1>);
  if (e == cudaSuccess) e = lim(k_hvhg<BW, double2, 1>);
  if (e == cudaSuccess) e = lim(k_hvhg<BW, float2, 1, 1>);
  if (e == cudaSuccess) e = lim(k_hvhg<BW, double2, 1, 1>);
  if (e == cudaSuccess) e = lim(k_hvhg<BW, float2, 1, 2>);
  if (e == cudaSuccess) e = lim(k_hvhg<BW, double2, 1, 2>);
  if (e == cudaSuccess) e = lim(k_hvhg<BW, float2, 2>);
  if (e == cudaSuccess) e = lim(k_hvhg<BW, double2, 2>);
  return e;
}

cudaError_t set_solver_smem_limits(const Handle &h) {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (e != cudaSuccess) return e;
  switch (h.bw) {
    case 2: return set_smem_limit_bw<2>(optin);
    case 3: return set_smem_limit_bw<3>(optin);
    case 4: return set_smem_limit_bw<4>(optin);
    case 5: return set_smem_limit_bw<5>(optin);
    case 6: return set_smem_limit_bw<6>(optin);
    case 7: return set_smem_limit_bw<7>(optin);
    default: return cudaErrorInvalidValue;
  }
}

size_t helm_ring_bytes(const Handle &h, int hgroups, int stage) {
  const size_t per = sizeof(double2) * (size_t)(stage + 1) * (5 + h.bw) * kLanes;  // kHelmUnits<BW>
  return per * (size_t)(kHelmRoles + h.nsc - 1) * hgroups;
}

int device_attr(cudaDeviceAttr attr) {
  int dev = 0, v = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&v, attr, dev) != cudaSuccess) return 0;
  return v;
}

}  // namespace

size_t solver_tables_bytes(const Handle &h) { return sizeof(double) * 3 * (size_t)h.ny * (4 * h.bw + 1); }

bool hvhg_tables_fit(const Handle &h) {
  return solver_tables_bytes(h) <= (size_t)device_attr(cudaDevAttrMaxSharedMemoryPerBlockOptin);
}

bool hvhg_shape_fits(const Handle &h, int groups, int stab, int stage) {
  if (h.nsc == 2 && (groups != 1 || stage != 0)) return false;
  const size_t nt = (size_t)kLanes * kRoles * groups;
  const size_t bytes = (stage > 0 ? sizeof(double2) * (size_t)(stage + 1) * kHvUnits * nt : 0) +
                       (stab ? solver_tables_bytes(h) : 0);
  return bytes <= (size_t)device_attr(cudaDevAttrMaxSharedMemoryPerBlockOptin);
}

bool helm_shape_fits(const Handle &h, int hgroups, int hstab, int stage) {
  // at most 384 threads (the kernel's launch bound); two scalars take one row of look-ahead
  if (hgroups < 1 || kLanes * (kHelmRoles + h.nsc - 1) * hgroups > 4 * kLanes * kHelmRoles) return false;
  if (h.nsc == 2 && stage != 1) return false;
  const size_t bytes = helm_ring_bytes(h, hgroups, stage) + (hstab ? solver_tables_bytes(h) : 0);
  return bytes <= (size_t)device_attr(cudaDevAttrMaxSharedMemoryPerBlockOptin);
}

void default_solver_shapes(Handle &h) {
  // k_hvhg: 32-mode blocks reading the tables through L1 and staging their rows two ahead
  // through shared memory (0.218 -> 0.212 ms against L1 prefetches at 192x129x192; one row
  // ahead spills and is slower, and the tables in shared memory beside the ring cost more).  k_helmholtz: the largest blocks that still
  // put a block on nearly every SM, with the tables in shared memory and two steps of staging
  // look-ahead where a block holds them; else 64-mode blocks with the tables where two fit on
  // an SM; else 32-mode blocks reading the tables through L1.
  h.tune.groups = 1;
  h.tune.stab = 0;
  h.tune.hgroups = 1;
  h.tune.hstab = 0;
  h.tune.stage = 1;
  h.tune.hvstage = 0;
  const int sms = device_attr(cudaDevAttrMultiProcessorCount);
  // the most 32-mode groups a 384-thread block holds: 4 with one scalar, 3 with two
  const int hgmax = (4 * kHelmRoles) / (kHelmRoles + h.nsc - 1);
  const bool full = h.nmodes >= (int64_t)kLanes * hgmax * sms * 9 / 10;
  if (h.nsc != 1) {
    // two scalars: the largest blocks with the tables in shared memory where they still put a
    // block on nearly every SM (one row of look-ahead)
    if (full && helm_shape_fits(h, hgmax, 1, 1)) {
      h.tune.hgroups = hgmax;
      h.tune.hstab = 1;
    }
    return;
  }
  if (hvhg_shape_fits(h, 1, 0, 2)) h.tune.hvstage = 2;  // k_hvhg: a two-row staging ring
  const size_t per_sm = (size_t)device_attr(cudaDevAttrMaxSharedMemoryPerMultiprocessor);
  if (full && helm_shape_fits(h, 4, 1, 2)) {
    h.tune.hgroups = 4;
    h.tune.hstab = 1;
    h.tune.stage = 2;
  } else if (full && helm_shape_fits(h, 4, 1, 1)) {
    // a larger ny: the tables and a one-row ring still fit beside each other
    h.tune.hgroups = 4;
    h.tune.hstab = 1;
  } else if (2 * (helm_ring_bytes(h, 2, 1) + solver_tables_bytes(h) + 1024) <= per_sm) {
    h.tune.hgroups = 2;
    h.tune.hstab = 1;
  }
}

cudaError_t launch_vop_factor(Handle &h, cudaStream_t st) {
  SplitArgs a{};
  a.ny = h.ny;
  a.nxh = h.nxh;
  a.nz = h.nz;
  a.nmodes = h.nmodes;
  a.ns = h.ns;
  a.tabs = h.dops + ops_offsets(h.bw, h.ny).t0;
  a.lmfxr = h.lmfxr;
  a.lmfzr = h.lmfzr;
  a.vf = h.vf;
  a.vf_l = vop_lband_doubles(h);
  const unsigned blocks = (unsigned)((h.nmodes + 127) / 128);
  // the solver kernels' staging ring and operator tables may exceed the default 48 KB of dynamic
  // shared memory: allow every instantiation of this BW the device's opt-in maximum (the
  // attribute only bounds a launch; each launch asks for what it uses)
  cudaError_t e = set_solver_smem_limits(h);
  if (e != cudaSuccess) return e;
  switch (h.bw) {
    case 2: k_vop_factor<2><<<blocks, 128, 0, st>>>(a); break;
    case 3: k_vop_factor<3><<<blocks, 128, 0, st>>>(a); break;
    case 4: k_vop_factor<4><<<blocks, 128, 0, st>>>(a); break;
    case 5: k_vop_factor<5><<<blocks, 128, 0, st>>>(a); break;
    case 6: k_vop_factor<6><<<blocks, 128, 0, st>>>(a); break;
    case 7: k_vop_factor<7><<<blocks, 128, 0, st>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

cudaError_t launch_ws_hvhg(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  return split_part(h, 0, substep, dt_ptr, st);
}

cudaError_t launch_ws_helmholtz(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  return split_part(h, 1, substep, dt_ptr, st);
}

cudaError_t launch_ws_assemble_only(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  return split_part(h, 2, substep, dt_ptr, st);
}

cudaError_t launch_ws_join(Handle &h, cudaStream_t st) { return cudaStreamWaitEvent(st, h.ev_join, 0); }

cudaError_t launch_ws_assemble(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  cudaError_t e = launch_ws_assemble_only(h, substep, dt_ptr, st);
  return e == cudaSuccess ? launch_ws_join(h, st) : e;
}

cudaError_t launch_wavespace_split(Handle &h, int substep, const double *dt_ptr, cudaStream_t st) {
  cudaError_t e = launch_ws_hvhg(h, substep, dt_ptr, st);
  if (e == cudaSuccess) e = launch_ws_helmholtz(h, substep, dt_ptr, st);
  if (e == cudaSuccess) e = launch_ws_assemble(h, substep, dt_ptr, st);
  return e;
}

}  // namespace kmm
