// sweeps.cuh - register-window sweeps for one (kx, kz) system per thread.
//
// The wall-normal operators are held in "offset rows": T(r, e) = D(r, r+e) for e in [-2BW, 2BW]
// (zero outside the matrix).  A collocation matrix row r spans columns lo(r)..hi(r):
//   lo = max(1, r-BW) for r <= n-BW, n-2BW for the last BW rows,
//   hi = min(r+BW, n) for r > BW,    2BW+1 for the first BW rows,
// which is the near-boundary packing of LABS_full_to_band (module_labs.f90:301-328).  An LU
// without pivoting keeps L and U inside that profile, so the Crout factorisation of
// fixed_bandec (module_labs.f90:3487-3636: L carries the pivots, U has a unit diagonal) is
// computed here row by row:
//   L(r, c) = A(r, c) - sum_{p=lo..c-1} L(r, p) U(p, c),     c = lo..r
//   U(r, c) = (A(r, c) - sum_{p=lo..r-1} L(r, p) U(p, c)) / L(r, r),   c = r+1..hi
// and fused with the forward substitution of every right-hand side that is ready, so L is
// never stored.  The solution windows live in registers:
//   forward  z_r = (b_r - sum_e L(r, r-e) z_{r-e}) / L(r, r)        window z_{r-2BW..r-1}
//   backward x_r = z_r - sum_e U(r, r+e) x_{r+e}                     window x_{r..r+2BW}
// and a band mat-vec (M x)_q = sum_e M(q, q+e) x_{q+e} of the solution is emitted from the
// backward window as soon as its inputs exist: row q = r+BW at step r (r <= n-2BW), the last
// BW rows at step n-2BW and the first BW rows at step 1, in descending order of q.  All loops over e have compile-time
// trip counts, so the windows stay in registers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "labs.cuh"

namespace kmm {

// Rows of look-ahead for the prefetches issued by the sweeps: the per-row loads of a thread are
// independent of its recurrence, so fetching them a few rows early hides the memory latency that
// would otherwise stall every row (a few warps per scheduler have little else to run).
// KMM_PREFETCH_ROWS (0 = none) and KMM_PREFETCH_L2 (prefetch into L2 instead of L1) are build
// tuning macros.
#ifndef KMM_PREFETCH_ROWS
#define KMM_PREFETCH_ROWS 4
#endif
constexpr int kPrefetchRows = KMM_PREFETCH_ROWS;

// cp.async copies global -> shared that bypass registers, tracked in per-thread commit groups.
__device__ __forceinline__ void cp_async16(void *sdst, const void *gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async8(void *sdst, const void *gsrc) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Steps of look-ahead of an asynchronously staged sweep (by default; the Helmholtz kernel takes
// its own as a template parameter), and its ring slots.
constexpr int kStageAhead = 1;
constexpr int kStageSlots = kStageAhead + 1;

// A thread-private ring in shared memory of S slots x K 16-byte units, interleaved across the
// block's nt threads (unit (slot, k) of thread t at smem[(slot * K + k) * nt + t]): the rows one
// sweep step reads, copied in by cp.async S - 1 steps before that step.  Slots are indexed by the
// sweep step (the row being eliminated), so a step's inputs may come from other rows (the
// emission rows q = r + BW of a backward sweep).
template <int K, int S = kStageSlots>
struct Ring {
  double2 *base;  // this thread's column: smem + threadIdx.x
  int nt;
  __device__ __forceinline__ double2 *at(int step, int k) const { return base + ((step % S) * K + k) * nt; }
  __device__ __forceinline__ void get(int step, int k, const double2 *g) const { cp_async16(at(step, k), g); }
  __device__ __forceinline__ void get(int step, int k, const float2 *g) const { cp_async8(at(step, k), g); }
  __device__ __forceinline__ void get(int step, int k, const double *g) const { cp_async8(at(step, k), g); }
  __device__ __forceinline__ double2 c(int step, int k) const { return *at(step, k); }
  __device__ __forceinline__ double d(int step, int k) const { return *reinterpret_cast<const double *>(at(step, k)); }
  __device__ __forceinline__ double2 f(int step, int k) const {  // a float2 unit, widened
    const float2 v = *reinterpret_cast<const float2 *>(at(step, k));
    return make_double2((double)v.x, (double)v.y);
  }
};

__device__ __forceinline__ void pf_l1(const void *p) {
  if constexpr (kPrefetchRows > 0) {
#ifdef KMM_PREFETCH_L2
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
#else
    asm volatile("prefetch.global.L1 [%0];" ::"l"(p));
#endif
  }
}

struct RLine {
  double *p;
  int64_t s;
  __device__ __forceinline__ double ld(int i) const { return p[(i - 1) * (int)s]; }
  __device__ __forceinline__ void st(int i, double v) const { p[(i - 1) * (int)s] = v; }
};

// Per-mode unit-upper factor U(r, r+e), e = 1..2BW.  Inside the profile only the first BW rows
// reach past e = BW (their last column is 2BW+1), so U is kept as [e = 1..BW][y][mode] plus
// [r = 1..BW][e = BW+1..2BW][mode] for those rows; every other entry is zero and not stored.
// A region for one mode set holds BW * es + BW * BW * s doubles.
template <int BW>
struct UBand {
  double *p;   // [BW][ny][s]
  double *px;  // [BW][BW][xs]
  int64_t s;   // stride between rows (number of modes)
  int64_t es;  // stride between offsets (ny * number of modes)
  int64_t xs;  // stride between the extra entries of the first rows (number of modes)
  __device__ __forceinline__ double get(int r, int e) const {
    if (e <= BW) return p[(e - 1) * (int)es + (r - 1) * (int)s];
    return r <= BW ? px[((r - 1) * BW + e - BW - 1) * (int)xs] : 0.0;
  }
  __device__ __forceinline__ void set(int r, int e, double v) const {
    if (e <= BW) p[(e - 1) * (int)es + (r - 1) * (int)s] = v;
    else if (r <= BW) px[((r - 1) * BW + e - BW - 1) * (int)xs] = v;
  }
  __device__ __forceinline__ const double *row_ptr(int r) const { return p + (r - 1) * (int)s; }
};
template <int BW>
__device__ __forceinline__ UBand<BW> make_uband(double *base, int64_t s, int64_t es) {
  return UBand<BW>{base, base + BW * es, s, es, s};
}
// The same for layouts whose row and offset strides are not (modes, ny * modes): the first rows'
// extra entries sit at base + px_off, xs apart ([BW][BW][mode] for xs = number of modes).
template <int BW>
__device__ __forceinline__ UBand<BW> make_uband(double *base, int64_t s, int64_t es, int64_t px_off, int64_t xs) {
  return UBand<BW>{base, base + px_off, s, es, xs};
}

// Per-mode L factor of a profile LU kept for later forward sweeps, the UBand idea for L:
// L(r, r-d) for d = 0..BW (d = 0 holds 1 / L(r, r)) as [BW+1][ny][mode], plus d = BW+1..2BW of
// the last BW rows (the only rows that reach below r - BW) as [BW][BW][mode].
// A region for one mode set holds (BW + 1) * es + BW * BW * s doubles.
template <int BW>
struct LBand {
  double *p;   // [BW+1][ny][s]
  double *px;  // [BW][BW][s], rows n-BW+1..n
  int64_t s, es;
  int n;
  __device__ __forceinline__ double get(int r, int d) const {
    if (d <= BW) return p[d * (int)es + (r - 1) * (int)s];
    return r > n - BW ? px[((r - (n - BW) - 1) * BW + d - BW - 1) * (int)s] : 0.0;
  }
  __device__ __forceinline__ void set(int r, int d, double v) const {
    if (d <= BW) p[d * (int)es + (r - 1) * (int)s] = v;
    else if (r > n - BW) px[((r - (n - BW) - 1) * BW + d - BW - 1) * (int)s] = v;
  }
};
template <int BW>
__device__ __forceinline__ LBand<BW> make_lband(double *base, int64_t s, int64_t es, int n) {
  return LBand<BW>{base, base + (BW + 1) * es, s, es, n};
}

template <int BW>
__device__ __forceinline__ int row_lo(int r, int n) { return (r <= n - BW) ? (r - BW > 1 ? r - BW : 1) : n - 2 * BW; }
template <int BW>
__device__ __forceinline__ int row_hi(int r, int n) { return (r <= BW) ? 2 * BW + 1 : (r + BW < n ? r + BW : n); }

// Offset-row tables shared by all modes.
template <int BW>
struct Tabs {
  const double *t0, *t1, *t2;  // [(r-1)*(4BW+1) + e + 2BW]
  const double *l0;            // D0 profile LU: [(r-1)*(2BW+1) + e] = L(r, r-e), e=0 -> 1/L(r,r)
  const double *u0;            // [(r-1)*2BW + e-1] = U(r, r+e)
};

template <int BW>
__device__ __forceinline__ const double *trow(const double *t, int r) { return t + (r - 1) * (4 * BW + 1) + 2 * BW; }

// The tables as laid out in the operator buffer: T0, T1, T2 [ny][4BW+1], L0 [ny][2BW+1], U0 [ny][2BW].
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

// The same from T1 on (T1, T2, L0, U0 contiguous as above); T0 is left unset.
template <int BW>
__device__ __forceinline__ Tabs<BW> tabs_from_t1(const double *t1, int ny) {
  const int64_t tw = (int64_t)ny * (4 * BW + 1);
  Tabs<BW> t;
  t.t0 = nullptr;
  t.t1 = t1;
  t.t2 = t1 + tw;
  t.l0 = t1 + 2 * tw;
  t.u0 = t.l0 + (int64_t)ny * (2 * BW + 1);
  return t;
}

// (M x)_q from the backward window w[j] = x_{r+j}: sum_j M(q, r+j-q) w[j].
template <int BW, typename WT>
__device__ __forceinline__ double2 mvc(const double *t, int q, int r, const WT &w) {
  const double *row = trow<BW>(t, q) + (r - q);
  double2 acc = z2(0.0, 0.0);
#pragma unroll
  for (int j = 0; j <= 2 * BW; ++j) {
    const double m = row[j];
    acc.x += m * w[j].x;
    acc.y += m * w[j].y;
  }
  return acc;
}
template <int BW, typename WT>
__device__ __forceinline__ double mvr(const double *t, int q, int r, const WT &w) {
  const double *row = trow<BW>(t, q) + (r - q);
  double acc = 0.0;
#pragma unroll
  for (int j = 0; j <= 2 * BW; ++j) acc += row[j] * w[j];
  return acc;
}

// Forward substitution with the fixed D0 factor for NC complex chains, ascending.
// in(r, b[NC]) supplies the right-hand sides of row r; out(r, z[NC]) receives the results.
struct NoPf {
  __device__ __forceinline__ void operator()(int) const {}
};

// Every sweep runs pf(r) PF steps before step r reads row r's inputs.  With ASYNC, pf issues
// cp.async copies: each step commits one group (possibly empty) and waits for the group of the
// current step, so PF groups stay in flight.
template <int BW, int NC, int PF = kPrefetchRows, bool ASYNC = false, typename In, typename Out, typename Pf = NoPf>
__device__ __forceinline__ void fwd_fixed(const Tabs<BW> &tb, int n, In in, Out out, Pf pf = Pf()) {
  constexpr int W = 2 * BW;
  double2 w[NC][W];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int k = 0; k < W; ++k) w[c][k] = z2(0.0, 0.0);
  for (int r = 1; r <= PF; ++r) {
    if (r <= n) pf(r);
    if constexpr (ASYNC) cp_async_commit();
  }
  for (int r = 1; r <= n; ++r) {
    if (r + PF <= n) pf(r + PF);
    if constexpr (ASYNC) {
      cp_async_commit();
      cp_async_wait<PF>();
    }
    double2 b[NC];
    in(r, b);
    const double *L = tb.l0 + (r - 1) * (W + 1);
    const double rp = L[0];
    double2 z[NC];
    // L(r, r-e) vanishes for e > BW above the last BW rows
    auto chain = [&]<int E>() {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double2 acc = b[c];
#pragma unroll
        for (int e = 1; e <= E; ++e) {
          const double l = L[e];
          acc.x -= l * w[c][W - e].x;
          acc.y -= l * w[c][W - e].y;
        }
        z[c] = z2(acc.x * rp, acc.y * rp);
      }
    };
    if (r <= n - BW) chain.template operator()<BW>();
    else chain.template operator()<W>();
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
      for (int k = 0; k < W - 1; ++k) w[c][k] = w[c][k + 1];
      w[c][W - 1] = z[c];
    }
    out(r, z);
  }
}

// Backward substitution (unit U given by ufn(r, e)) for NC complex and NR real chains,
// descending, with mat-vec emission: emit(q, r, wc, wr) where wc[c][j] = x_{r+j}.
template <int BW, int NC, int NR, int PF = kPrefetchRows, bool ASYNC = false, typename UF, typename Zin,
          typename Emit, typename Pf = NoPf>
__device__ __forceinline__ void bwd_emit(int n, UF ufn, Zin zin, Emit emit, Pf pf = Pf()) {
  constexpr int W = 2 * BW + 1;
  constexpr int NCc = NC > 0 ? NC : 1, NRr = NR > 0 ? NR : 1;
  double2 wc[NCc][W];
  double wr[NRr][W];
#pragma unroll
  for (int j = 0; j < W; ++j) {
#pragma unroll
    for (int c = 0; c < NCc; ++c) wc[c][j] = z2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < NRr; ++c) wr[c][j] = 0.0;
  }
  for (int r = n; r > n - PF; --r) {
    if (r >= 1) pf(r);
    if constexpr (ASYNC) cp_async_commit();
  }
  for (int r = n; r >= 1; --r) {
    if (r - PF >= 1) pf(r - PF);
    if constexpr (ASYNC) {
      cp_async_commit();
      cp_async_wait<PF>();
    }
#pragma unroll
    for (int j = W - 1; j >= 1; --j) {
#pragma unroll
      for (int c = 0; c < NCc; ++c) wc[c][j] = wc[c][j - 1];
#pragma unroll
      for (int c = 0; c < NRr; ++c) wr[c][j] = wr[c][j - 1];
    }
    double2 zc[NCc];
    double zr[NRr];
    zin(r, zc, zr);
    // U(r, r+e) vanishes for e > BW below the first BW rows
    auto chain = [&]<int E>() {
      double u[E];
#pragma unroll
      for (int e = 1; e <= E; ++e) u[e - 1] = ufn(r, e);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double2 acc = zc[c];
#pragma unroll
        for (int e = 1; e <= E; ++e) {
          acc.x -= u[e - 1] * wc[c][e].x;
          acc.y -= u[e - 1] * wc[c][e].y;
        }
        wc[c][0] = acc;
      }
#pragma unroll
      for (int c = 0; c < NR; ++c) {
        double acc = zr[c];
#pragma unroll
        for (int e = 1; e <= E; ++e) acc -= u[e - 1] * wr[c][e];
        wr[c][0] = acc;
      }
    };
    if (r > BW) chain.template operator()<BW>();
    else chain.template operator()<2 * BW>();
    if (r == n - 2 * BW)
      for (int q = n; q > n - BW; --q) emit(q, r, wc, wr);
    if (r <= n - 2 * BW) emit(r + BW, r, wc, wr);
    if (r == 1)
      for (int q = BW; q >= 1; --q) emit(q, r, wc, wr);
  }
}

// Profile Crout LU of a per-mode matrix fused with the forward substitution of NC complex and
// NR real chains, one row per step(), ascending.  rowA(r, a, centre) fills a[e + 2BW] = A(r, r+e)
// (for centre rows only |e| <= BW, the entries they use); bc / br are the right-hand sides of
// row r and zc / zr receive the forward results; U goes to ust for the backward sweep.  Rows
// 2BW+1..n-BW only touch U(p, p+e) with e <= BW of the last BW rows, which stay in a register
// window; the first 2BW and last BW rows read U back from ust.
// With KEEP_L, step() leaves row r's L (Lk[d] = L(r, r-d), Lk[0] = 1 / L(r, r)) in Lk.
template <int BW, int NC, int NR, bool KEEP_L = false>
struct LuSweep {
  static constexpr int W = 2 * BW;
  static constexpr int NCc = NC > 0 ? NC : 1, NRr = NR > 0 ? NR : 1;
  double2 wc[NCc][W];
  double wr[NRr][W];
  double Uw[BW][BW];  // Uw[dp-1][e-1] = U(r-dp, r-dp+e)
  double Lk[KEEP_L ? W + 1 : 1];
  UBand<BW> ust;
  int n;

  __device__ __forceinline__ void init(int n_, UBand<BW> u) {
    n = n_;
    ust = u;
#pragma unroll
    for (int k = 0; k < W; ++k) {
#pragma unroll
      for (int c = 0; c < NCc; ++c) wc[c][k] = z2(0.0, 0.0);
#pragma unroll
      for (int c = 0; c < NRr; ++c) wr[c][k] = 0.0;
    }
#pragma unroll
    for (int i = 0; i < BW; ++i)
#pragma unroll
      for (int e = 0; e < BW; ++e) Uw[i][e] = 0.0;
  }

  template <typename RowA>
  __device__ __forceinline__ void step(int r, RowA rowA, const double2 *bc, const double *br, double2 *zc,
                                       double *zr) {
    double a[4 * BW + 1];
    double L[W + 1];  // L[d] = L(r, r-d)
    double Ur[W];     // U(r, r+e), e = 1..W
    if (r > 2 * BW && r <= n - BW) {
      rowA(r, a, true);
      // centre row: lo = r - BW, hi = r + BW; U of rows r-BW..r-1 from the register window
#pragma unroll
      for (int d = W; d > BW; --d) L[d] = 0.0;
#pragma unroll
      for (int d = BW; d >= 0; --d) {
        double acc = a[2 * BW - d];
#pragma unroll
        for (int dp = BW; dp > d; --dp) acc -= L[dp] * Uw[dp - 1][dp - d - 1];
        L[d] = acc;
      }
      const double rp = 1.0 / L[0];
#pragma unroll
      for (int e = 1; e <= W; ++e) {
        double v = 0.0;
        if (e <= BW) {
          double acc = a[2 * BW + e];
#pragma unroll
          for (int dp = BW; dp >= 1; --dp)
            if (e + dp <= BW) acc -= L[dp] * Uw[dp - 1][e + dp - 1];
          v = acc * rp;
        }
        Ur[e - 1] = v;
      }
      L[0] = rp;  // from here on L[0] holds the reciprocal pivot
    } else {
      rowA(r, a, false);
      const int lo = row_lo<BW>(r, n), hi = row_hi<BW>(r, n);
#pragma unroll
      for (int d = W; d >= 0; --d) {
        double acc = 0.0;
        if (r - d >= lo) {
          acc = a[2 * BW - d];
#pragma unroll
          for (int dp = W; dp > d; --dp)
            if (r - dp >= lo) acc -= L[dp] * ust.get(r - dp, dp - d);
        }
        L[d] = acc;
      }
      const double rp = 1.0 / L[0];
#pragma unroll
      for (int e = 1; e <= W; ++e) {
        double v = 0.0;
        if (r + e <= hi) {
          double acc = a[2 * BW + e];
#pragma unroll
          for (int dp = W; dp >= 1; --dp)
            if (r - dp >= lo && e + dp <= W) acc -= L[dp] * ust.get(r - dp, e + dp);
          v = acc * rp;
        }
        Ur[e - 1] = v;
      }
      L[0] = rp;
    }
#pragma unroll
    for (int e = 1; e <= W; ++e) ust.set(r, e, Ur[e - 1]);
#pragma unroll
    for (int i = BW - 1; i >= 1; --i)
#pragma unroll
      for (int e = 0; e < BW; ++e) Uw[i][e] = Uw[i - 1][e];
#pragma unroll
    for (int e = 0; e < BW; ++e) Uw[0][e] = Ur[e];
    const double rp = L[0];
    if constexpr (KEEP_L) {
#pragma unroll
      for (int d = 0; d <= W; ++d) Lk[d] = L[d];
    }
    // L(r, r-d) vanishes for d > BW above the last BW rows
    auto chain = [&]<int D>() {
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double2 acc = bc[c];
#pragma unroll
        for (int d = 1; d <= D; ++d) {
          acc.x -= L[d] * wc[c][W - d].x;
          acc.y -= L[d] * wc[c][W - d].y;
        }
        zc[c] = z2(acc.x * rp, acc.y * rp);
      }
#pragma unroll
      for (int c = 0; c < NR; ++c) {
        double acc = br[c];
#pragma unroll
        for (int d = 1; d <= D; ++d) acc -= L[d] * wr[c][W - d];
        zr[c] = acc * rp;
      }
    };
    if (r <= n - BW) chain.template operator()<BW>();
    else chain.template operator()<W>();
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
      for (int k = 0; k < W - 1; ++k) wc[c][k] = wc[c][k + 1];
      wc[c][W - 1] = zc[c];
    }
#pragma unroll
    for (int c = 0; c < NR; ++c) {
#pragma unroll
      for (int k = 0; k < W - 1; ++k) wr[c][k] = wr[c][k + 1];
      wr[c][W - 1] = zr[c];
    }
  }
};

// The LuSweep over rows 1..n: in(r, bc, br) supplies row r's right-hand sides, out(r, zc, zr)
// receives the forward results.
template <int BW, int NC, int NR, int PF = kPrefetchRows, bool ASYNC = false, typename RowA, typename In,
          typename Out, typename Pf = NoPf>
__device__ __forceinline__ void lu_fwd(int n, RowA rowA, In in, Out out, UBand<BW> ust, Pf pf = Pf()) {
  constexpr int NCc = NC > 0 ? NC : 1, NRr = NR > 0 ? NR : 1;
  LuSweep<BW, NC, NR> lu;
  lu.init(n, ust);
  for (int r = 1; r <= PF; ++r) {
    if (r <= n) pf(r);
    if constexpr (ASYNC) cp_async_commit();
  }
  for (int r = 1; r <= n; ++r) {
    if (r + PF <= n) pf(r + PF);
    if constexpr (ASYNC) {
      cp_async_commit();
      cp_async_wait<PF>();
    }
    double2 bc[NCc];
    double br[NRr];
    in(r, bc, br);
    double2 zc[NCc];
    double zr[NRr];
    lu.step(r, rowA, bc, br, zc, zr);
    out(r, zc, zr);
  }
}

// Forward substitution with a per-mode L kept by a KEEP_L LuSweep, for NC complex and NR real
// chains, ascending (the arithmetic of LuSweep::step's chains); lget(r, d) = L(r, r-d), d = 0
// giving 1 / L(r, r).
template <int BW, int NC, int NR, int PF = kPrefetchRows, bool ASYNC = false, typename LGet, typename In,
          typename Out, typename Pf = NoPf>
__device__ __forceinline__ void fwd_lband(LGet lget, int n, In in, Out out, Pf pf = Pf()) {
  constexpr int W = 2 * BW;
  constexpr int NCc = NC > 0 ? NC : 1, NRr = NR > 0 ? NR : 1;
  double2 wc[NCc][W];
  double wr[NRr][W];
#pragma unroll
  for (int k = 0; k < W; ++k) {
#pragma unroll
    for (int c = 0; c < NCc; ++c) wc[c][k] = z2(0.0, 0.0);
#pragma unroll
    for (int c = 0; c < NRr; ++c) wr[c][k] = 0.0;
  }
  for (int r = 1; r <= PF; ++r) {
    if (r <= n) pf(r);
    if constexpr (ASYNC) cp_async_commit();
  }
  for (int r = 1; r <= n; ++r) {
    if (r + PF <= n) pf(r + PF);
    if constexpr (ASYNC) {
      cp_async_commit();
      cp_async_wait<PF>();
    }
    double2 bc[NCc];
    double br[NRr];
    in(r, bc, br);
    double2 zc[NCc];
    double zr[NRr];
    const double rp = lget(r, 0);
    auto chain = [&]<int D>() {
      double L[D + 1];
#pragma unroll
      for (int d = 1; d <= D; ++d) L[d] = lget(r, d);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        double2 acc = bc[c];
#pragma unroll
        for (int d = 1; d <= D; ++d) {
          acc.x -= L[d] * wc[c][W - d].x;
          acc.y -= L[d] * wc[c][W - d].y;
        }
        zc[c] = z2(acc.x * rp, acc.y * rp);
      }
#pragma unroll
      for (int c = 0; c < NR; ++c) {
        double acc = br[c];
#pragma unroll
        for (int d = 1; d <= D; ++d) acc -= L[d] * wr[c][W - d];
        zr[c] = acc * rp;
      }
    };
    if (r <= n - BW) chain.template operator()<BW>();
    else chain.template operator()<W>();
#pragma unroll
    for (int c = 0; c < NC; ++c) {
#pragma unroll
      for (int k = 0; k < W - 1; ++k) wc[c][k] = wc[c][k + 1];
      wc[c][W - 1] = zc[c];
    }
#pragma unroll
    for (int c = 0; c < NR; ++c) {
#pragma unroll
      for (int k = 0; k < W - 1; ++k) wr[c][k] = wr[c][k + 1];
      wr[c][W - 1] = zr[c];
    }
    out(r, zc, zr);
  }
}

}  // namespace kmm
