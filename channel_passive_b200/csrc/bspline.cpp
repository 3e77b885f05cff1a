// bspline.cpp - wall-normal B-spline collocation operators without GSL.
//
// Replaces labs_fill_full.cpp:35-256 (which calls GSL's gsl_bspline_* and
// gsl_integration_glfixed_*) and the set-up half of LABS_initialize
// (module_labs.f90:77-238: LABS_eval_bw, LABS_full_to_band, LABS_lu of D0).
//
// Conventions restated from GSL's documented behaviour:
//   knots    t[0..k-1] = y_0, t[k..n-1] = interior breakpoints, t[n..n+k-1] = y_end
//   Greville abscissa i = running mean of t[i+1..i+k-1] (GSL's gsl_stats_mean recurrence)
//   span     t[s] <= x < t[s+1], the last non-empty span at the right end point
//   Gauss-Legendre rule of (k - nderiv + 1)/2 points per breakpoint interval
// Basis values and derivatives use the Cox-de Boor triangle followed by the derivative
// recurrence on coefficient differences (de Boor, "A Practical Guide to Splines", ch. X).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "kmm_internal.h"

namespace kmm {
namespace {

constexpr double kPi = 3.141592653589793238462643;  // labs_fill_full.cpp:24

void breakpoints(int nbreak, double stretch, double ly, int grid, std::vector<double> &y) {
  y.resize(nbreak);
  if (grid == KMM_GRID_TANH) {
    // labs_fill_full.cpp:89 (commented alternative in the reference)
    for (int i = 0; i < nbreak; ++i)
      y[i] = 0.5 * ly * std::tanh(stretch * (-1.0 + (2.0 * i) / (nbreak - 1))) / std::tanh(stretch);
    return;
  }
  if (std::fabs(stretch) <= 0.0000000000000001) {  // labs_fill_full.cpp:80-85
    for (int i = 0; i < nbreak; ++i) y[i] = -1.0 + 2.0 / (nbreak - 1) * i;
  } else {  // Jimenez sine map, labs_fill_full.cpp:92
    for (int i = 0; i < nbreak; ++i)
      y[i] = std::sin(stretch * kPi / 2.0 * (-1.0 + (2.0 * i) / (nbreak - 1))) /
             std::sin(stretch * kPi / 2.0);
  }
}

int find_span(const std::vector<double> &t, int k, int n, double x) {
  for (int s = k - 1; s < n; ++s) {
    if (t[s] <= x && x < t[s + 1]) return s;
    if (t[s] < x && x == t[s + 1] && t[s + 1] == t[n]) return s;
  }
  return -1;
}

// ders[d*k + r] = d-th derivative of basis s-k+1+r at x, d = 0..nder (nder <= k-1).
void basis_derivs(const std::vector<double> &t, int k, int s, double x, int nder,
                  std::vector<double> &ders) {
  const int p = k - 1;
  std::vector<double> ndu(k * k, 0.0), left(k, 0.0), right(k, 0.0), a(2 * k, 0.0);
  auto N = [&](int i, int j) -> double & { return ndu[i * k + j]; };
  N(0, 0) = 1.0;
  for (int j = 1; j < k; ++j) {
    left[j] = x - t[s + 1 - j];
    right[j] = t[s + j] - x;
    double saved = 0.0;
    for (int r = 0; r < j; ++r) {
      N(j, r) = right[r + 1] + left[j - r];
      double temp = N(r, j - 1) / N(j, r);
      N(r, j) = saved + right[r + 1] * temp;
      saved = left[j - r] * temp;
    }
    N(j, j) = saved;
  }
  ders.assign((nder + 1) * k, 0.0);
  for (int r = 0; r < k; ++r) ders[r] = N(r, p);
  for (int r = 0; r < k; ++r) {
    int s1 = 0, s2 = 1;
    a[0] = 1.0;
    for (int d = 1; d <= nder; ++d) {
      double acc = 0.0;
      int rk = r - d, pk = p - d;
      if (r >= d) {
        a[s2 * k + 0] = a[s1 * k + 0] / N(pk + 1, rk);
        acc = a[s2 * k + 0] * N(rk, pk);
      }
      int j1 = (rk >= -1) ? 1 : -rk;
      int j2 = (r - 1 <= pk) ? d - 1 : p - r;
      for (int j = j1; j <= j2; ++j) {
        a[s2 * k + j] = (a[s1 * k + j] - a[s1 * k + j - 1]) / N(pk + 1, rk + j);
        acc += a[s2 * k + j] * N(rk + j, pk);
      }
      if (r <= pk) {
        a[s2 * k + d] = -a[s1 * k + d - 1] / N(pk + 1, r);
        acc += a[s2 * k + d] * N(r, pk);
      }
      ders[d * k + r] = acc;
      std::swap(s1, s2);
    }
  }
  double fac = p;
  for (int d = 1; d <= nder; ++d) {
    for (int r = 0; r < k; ++r) ders[d * k + r] *= fac;
    fac *= (p - d);
  }
}

// Values of all n bases (derivative nder) at x into out[n].
void eval_all(const std::vector<double> &t, int k, int n, double x, int nder, double *out) {
  std::fill(out, out + n, 0.0);
  int s = find_span(t, k, n, x);
  if (s < 0) return;
  std::vector<double> d;
  int nd = std::min(nder, k - 1);
  basis_derivs(t, k, s, x, nd, d);
  if (nder > k - 1) return;
  for (int r = 0; r < k; ++r) out[s - k + 1 + r] = d[nder * k + r];
}

// Gauss-Legendre nodes/weights on [-1, 1] by Newton iteration on P_m.
void gauss_legendre(int m, std::vector<double> &x, std::vector<double> &w) {
  x.assign(m, 0.0);
  w.assign(m, 0.0);
  for (int i = 0; i < (m + 1) / 2; ++i) {
    double z = std::cos(kPi * (i + 0.75) / (m + 0.5)), pp = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= m; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = m * (z * p1 - p2) / (z * z - 1.0);
      double z1 = z;
      z = z1 - p1 / pp;
      if (std::fabs(z - z1) <= 1e-16) break;
    }
    x[i] = -z;
    x[m - 1 - i] = z;
    w[i] = w[m - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

}  // namespace

// LABS_fill_full restated (labs_fill_full.cpp:35-195).  full[d] is [point][basis].
static void fill_full(int k, int n, double stretch, double ly, int grid, HostOps &ops) {
  const int nbreak = n - k + 2;
  breakpoints(nbreak, stretch, ly, grid, ops.brk);
  ops.knots.clear();
  for (int i = 0; i < k; ++i) ops.knots.push_back(ops.brk[0]);
  for (int i = 1; i < nbreak - 1; ++i) ops.knots.push_back(ops.brk[i]);
  for (int i = 0; i < k; ++i) ops.knots.push_back(ops.brk[nbreak - 1]);
  const std::vector<double> &t = ops.knots;
  ops.y.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {  // Greville abscissae, labs_fill_full.cpp:106-109
    double mean = 0.0;
    for (int j = 0; j < k - 1; ++j) mean += (t[i + 1 + j] - mean) / (j + 1);
    ops.y[i] = mean;
  }
  for (int d = 0; d < 5; ++d) ops.full[d].assign((size_t)n * n, 0.0);
  std::vector<double> dd;
  for (int i = 0; i < n; ++i) {  // labs_fill_full.cpp:110-131
    int s = find_span(t, k, n, ops.y[i]);
    int nd = std::min(4, k - 1);
    basis_derivs(t, k, s, ops.y[i], nd, dd);
    for (int d = 0; d <= nd; ++d)
      for (int r = 0; r < k; ++r) ops.full[d][(size_t)i * n + (s - k + 1 + r)] = dd[d * k + r];
  }
  // integration weights, labs_fill_full.cpp:206-256 (nderiv = 0)
  ops.integ.assign(n, 0.0);
  std::vector<double> gx, gw;
  gauss_legendre((k + 1) / 2, gx, gw);
  for (int i = 0; i < nbreak - 1; ++i) {
    double a = ops.brk[i], b = ops.brk[i + 1];
    for (size_t j = 0; j < gx.size(); ++j) {
      double xj = 0.5 * (b + a) + 0.5 * (b - a) * gx[j];
      double wj = 0.5 * (b - a) * gw[j];
      int s = find_span(t, k, n, xj);
      basis_derivs(t, k, s, xj, 0, dd);
      for (int r = 0; r < k; ++r) ops.integ[s - k + 1 + r] += wj * dd[r];
    }
  }
  ops.center.assign(n, 0.0);  // labs_fill_full.cpp:146-149
  eval_all(t, k, n, 0.0, 0, ops.center.data());
}

// LABS_eval_bw (module_labs.f90:245-293) on FULL(basis, point).
static int eval_bw(const HostOps &ops) {
  const int n = ops.ny;
  auto F = [&](int d, int i, int j) {  // FULL(i=basis, j=point), 1-based
    return std::fabs(ops.full[d][(size_t)(j - 1) * n + (i - 1)]);
  };
  for (int k = 1; k < n; ++k) {
    double err = 0.0;
    for (int d = 0; d < 3; ++d) {
      for (int j = 1; j <= k + 1; ++j)
        for (int i = 2 * k + 2; i <= n; ++i) err = std::max(err, F(d, i, j));
      for (int j = k + 2; j <= n - k - 1; ++j) {
        for (int i = 1; i <= j - k - 1; ++i) err = std::max(err, F(d, i, j));
        for (int i = j + k + 1; i <= n; ++i) err = std::max(err, F(d, i, j));
      }
      for (int j = n - k; j <= n; ++j)
        for (int i = 1; i <= n - 2 * k - 1; ++i) err = std::max(err, F(d, i, j));
    }
    if (err <= 0.0) return k;
  }
  return -1;
}

// LABS_full_to_band (module_labs.f90:301-328).
static void full_to_band(const std::vector<double> &full, int bw, int n, std::vector<double> &band) {
  const int ld = 2 * bw + 1;
  band.assign((size_t)ld * n, 0.0);
  auto F = [&](int i, int j) { return full[(size_t)(j - 1) * n + (i - 1)]; };
  auto B = [&](int r, int j) -> double & { return band[(size_t)(j - 1) * ld + (r - 1)]; };
  for (int j = 1; j <= bw; ++j) {
    for (int i = 1; i <= bw + j; ++i) B(bw + 1 + i - j, j) = F(i, j);
    for (int i = j + bw + 1; i <= 2 * bw + 1; ++i) B(2 * bw + 2 - i, j) = F(i, j);
  }
  for (int j = bw + 1; j <= n - bw; ++j)
    for (int i = 1; i <= 2 * bw + 1; ++i) B(i, j) = F(j + i - bw - 1, j);
  for (int j = n - bw + 1; j <= n; ++j) {
    for (int i = j - bw; i <= n; ++i) B(bw + 1 + i - j, j) = F(i, j);
    for (int i = n - 2 * bw; i <= j - bw - 1; ++i) B(n - i + 1, j) = F(i, j);
  }
}

// fixed_bandec (module_labs.f90:3487-3636), host copy used for LABS_D0_LU.
void host_band_lu(std::vector<double> &a, int bw, int n) {
  const int ld = 2 * bw + 1, m = bw + 1;
  auto A = [&](int r, int c) -> double & { return a[(size_t)(c - 1) * ld + (r - 1)]; };
  for (int i = 1; i <= bw; ++i) {
    double dummy = 1.0 / A(m, i);
    for (int j = 1; j <= bw + 1 - i; ++j) {
      double acc = A(m + j, i);
      for (int k = 1; k <= i - 1; ++k) acc -= A(m - k, i) * A(m + j + k, i - k);
      A(m + j, i) = dummy * acc;
    }
    for (int j = bw + 2 - i; j <= bw; ++j) {
      double acc = A(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A(m - k, i) * A(m + j + k, i - k);
      for (int k = bw - j + 1; k <= i - 1; ++k) acc -= A(m - k, i) * A(m + bw - i - j + 1, i - k);
      A(m + j, i) = dummy * acc;
    }
    for (int j = i; j <= bw; ++j) {
      double acc = A(m - j, i);
      for (int k = 1; k <= i - 1; ++k) acc -= A(m - k, i) * A(m - j, i - k);
      A(m - j, i) = dummy * acc;
    }
    for (int j = 1; j <= bw + 1 - i; ++j) {
      double acc = A(m + 1 - j, i + j);
      for (int k = 1; k <= i; ++k) acc -= A(m + 1 - j - k, i + j) * A(m + k, i + 1 - k);
      A(m + 1 - j, i + j) = acc;
    }
    for (int j = bw + 2 - i; j <= bw; ++j) {
      double acc = A(m + 1 - j, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A(m + 1 - j - k, i + j) * A(m + k, i + 1 - k);
      A(m + 1 - j, i + j) = acc;
    }
  }
  for (int i = m; i <= 2 * bw; ++i) {
    double dummy = 1.0 / A(m, i);
    for (int j = 1; j <= 2 * bw + 1 - i; ++j) {
      double acc = A(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A(m - k, i) * A(m + j + k, i - k);
      for (int k = bw - j + 1; k <= bw; ++k) acc -= A(m - k, i) * A(2 * m - i - j, i - k);
      A(m + j, i) = dummy * acc;
    }
    for (int j = 2 * bw + 2 - i; j <= bw; ++j) {
      double acc = A(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A(m - k, i) * A(m + j + k, i - k);
      A(m + j, i) = dummy * acc;
    }
    for (int j = 1; j <= bw; ++j) {
      double acc = A(m - j + 1, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A(m - j + 1 - k, i + j) * A(m + k, i - k + 1);
      A(m - j + 1, i + j) = acc;
    }
  }
  for (int i = 2 * bw + 1; i <= n - 2 * bw - 1; ++i) {
    double dummy = 1.0 / A(m, i);
    for (int j = 1; j <= bw; ++j) {
      double acc = A(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A(m - k, i) * A(m + j + k, i - k);
      A(m + j, i) = dummy * acc;
    }
    for (int j = 1; j <= bw; ++j) {
      double acc = A(m - j + 1, i + j);
      for (int k = 1; k <= bw - j + 1; ++k) acc -= A(m + 1 - j - k, i + j) * A(m + k, i + 1 - k);
      A(m - j + 1, i + j) = acc;
    }
  }
  for (int i = n - 2 * bw; i <= n - bw - 1; ++i) {
    double dummy = 1.0 / A(m, i);
    for (int j = 1; j <= bw; ++j) {
      double acc = A(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A(m - k, i) * A(m + j + k, i - k);
      A(m + j, i) = dummy * acc;
    }
    for (int j = 1; j <= n - bw - i; ++j) {
      double acc = A(m - j + 1, i + j);
      for (int k = 1; k <= bw - j + 1; ++k) acc -= A(m + 1 - j - k, i + j) * A(m + k, i + 1 - k);
      A(m - j + 1, i + j) = acc;
    }
    for (int j = n - bw - i + 1; j <= bw + 1; ++j) {
      double acc = A(m - j + 1, i + j);
      for (int k = 1; k <= bw + 1 - j; ++k) acc -= A(m + 1 - j - k, i + j) * A(m + k, i + 1 - k);
      for (int k = bw + 2 - j; k <= i - n + 2 * bw + 1; ++k)
        acc -= A(m + n - bw - 1 + k - i, i + j) * A(m + k, i + 1 - k);
      A(m - j + 1, i + j) = acc;
    }
    for (int j = bw + 2; j <= n - i; ++j) {
      double acc = A(m + n - bw - 1 - i, i + j);
      for (int k = 1; k <= i - n + 2 * bw + 1; ++k)
        acc -= A(m + n - bw - 1 - i + k, i + j) * A(m + k, i + 1 - k);
      A(m + n - bw - 1 - i, i + j) = acc;
    }
  }
  for (int i = n - bw; i <= n - 1; ++i) {
    double dummy = 1.0 / A(m, i);
    for (int j = 1; j <= n - i; ++j) {
      double acc = A(m + j, i);
      for (int k = 1; k <= bw - j; ++k) acc -= A(m - k, i) * A(m + j + k, i - k);
      A(m + j, i) = dummy * acc;
    }
    for (int j = 1; j <= n - i; ++j) {
      double acc = A(m - j + 1, i + j);
      for (int k = 1; k <= 1 + bw - j; ++k) acc -= A(m + 1 - j - k, i + j) * A(m + k, i + 1 - k);
      for (int k = 2 + bw - j; k <= bw; ++k)
        acc -= A(m + n - bw - 1 - i + k, i + j) * A(m + k, i + 1 - k);
      A(m - j + 1, i + j) = acc;
    }
  }
}

// Offset-row tables for the per-mode solver: T_d[(r-1)*(4bw+1) + e + 2bw] = D_d(r, r+e) for
// e in [-2bw, 2bw] (zero outside the matrix), and the profile Crout LU of D0 without pivoting:
// L0[(r-1)*(2bw+1) + e] = L(r, r-e) for e = 1..2bw with 1/L(r, r) at e = 0, and
// U0[(r-1)*2bw + e-1] = U(r, r+e) (unit diagonal).  Row r of a collocation matrix spans columns
// lo(r)..hi(r) with lo = max(1, r-bw) (n-2bw for the last bw rows) and hi = min(r+bw, n)
// (2bw+1 for the first bw rows), the structure LABS_full_to_band packs (module_labs.f90:301-328);
// an LU without pivoting keeps L and U inside it.
static void build_offset_tables(HostOps &ops) {
  const int n = ops.ny, bw = ops.bw, w = 4 * bw + 1;
  for (int d = 0; d < 3; ++d) {
    ops.off[d].assign((size_t)n * w, 0.0);
    for (int r = 1; r <= n; ++r)
      for (int e = -2 * bw; e <= 2 * bw; ++e) {
        const int c = r + e;
        if (c >= 1 && c <= n) ops.off[d][(size_t)(r - 1) * w + e + 2 * bw] = ops.full[d][(size_t)(r - 1) * n + (c - 1)];
      }
  }
  ops.l0.assign((size_t)n * (2 * bw + 1), 0.0);
  ops.u0.assign((size_t)n * 2 * bw, 0.0);
  std::vector<double> L(2 * bw + 1);
  auto U = [&](int p, int e) { return (e >= 1 && e <= 2 * bw) ? ops.u0[(size_t)(p - 1) * 2 * bw + e - 1] : 0.0; };
  auto A = [&](int r, int c) { return ops.full[0][(size_t)(r - 1) * n + (c - 1)]; };
  for (int r = 1; r <= n; ++r) {
    const int lo = (r <= n - bw) ? std::max(1, r - bw) : n - 2 * bw;
    const int hi = (r <= bw) ? 2 * bw + 1 : std::min(r + bw, n);
    for (int c = lo; c <= r; ++c) {
      double acc = A(r, c);
      for (int p = lo; p < c; ++p) acc -= L[r - p] * U(p, c - p);
      L[r - c] = acc;
    }
    const double rp = 1.0 / L[0];
    ops.l0[(size_t)(r - 1) * (2 * bw + 1)] = rp;
    for (int e = 1; e <= 2 * bw; ++e) ops.l0[(size_t)(r - 1) * (2 * bw + 1) + e] = (r - e >= lo) ? L[e] : 0.0;
    for (int c = r + 1; c <= hi; ++c) {
      double acc = A(r, c);
      for (int p = lo; p < r; ++p) acc -= L[r - p] * U(p, c - p);
      ops.u0[(size_t)(r - 1) * 2 * bw + (c - r) - 1] = acc * rp;
    }
  }
}

int build_host_ops(int k_order, int ny, double stretch, double ly, int grid, HostOps &ops,
                   std::string &err) {
  if (k_order < 2 || ny <= 2 * (k_order - 1)) {
    err = "K, order of B-spline, is too large (ny must exceed 2*labs_k)";
    return KMM_ERR_CONFIG;
  }
  ops.ny = ny;
  ops.k = k_order;
  fill_full(k_order, ny, stretch, ly, grid, ops);
  for (int d = 0; d < 5; ++d)
    for (double v : ops.full[d])
      if (!std::isfinite(v)) {
        err = "non-finite B-spline operator entry";
        return KMM_ERR_CONFIG;
      }
  ops.bw = eval_bw(ops);
  if (ops.bw < 1 || 4 * ops.bw + 2 > ny) {
    err = "B-spline band width detection failed (grid too coarse)";
    return KMM_ERR_CONFIG;
  }
  for (int d = 0; d < 3; ++d) full_to_band(ops.full[d], ops.bw, ny, ops.band[d]);
  ops.d0_lu = ops.band[0];
  host_band_lu(ops.d0_lu, ops.bw, ny);
  build_offset_tables(ops);
  return KMM_OK;
}

// Solves D0^T w = e(y_d) so that v(y_d) = w . v for collocation values v.
int build_control_weights(HostOps &ops, double yd, std::string &err) {
  const int n = ops.ny;
  auto solve_t = [&](double x, std::vector<double> &w) -> bool {
    std::vector<double> e(n);
    eval_all(ops.knots, ops.k, n, x, 0, e.data());
    // dense A = D0^T, A[r][c] = D0[c][r] = full0[c*n + r]
    std::vector<double> A((size_t)n * n);
    for (int r = 0; r < n; ++r)
      for (int c = 0; c < n; ++c) A[(size_t)r * n + c] = ops.full[0][(size_t)c * n + r];
    w = e;
    for (int col = 0; col < n; ++col) {  // Gaussian elimination, partial pivoting
      int piv = col;
      for (int r = col + 1; r < n; ++r)
        if (std::fabs(A[(size_t)r * n + col]) > std::fabs(A[(size_t)piv * n + col])) piv = r;
      if (A[(size_t)piv * n + col] == 0.0) return false;
      if (piv != col) {
        for (int c = 0; c < n; ++c) std::swap(A[(size_t)piv * n + c], A[(size_t)col * n + c]);
        std::swap(w[piv], w[col]);
      }
      for (int r = col + 1; r < n; ++r) {
        double f = A[(size_t)r * n + col] / A[(size_t)col * n + col];
        if (f == 0.0) continue;
        for (int c = col; c < n; ++c) A[(size_t)r * n + c] -= f * A[(size_t)col * n + c];
        w[r] -= f * w[col];
      }
    }
    for (int r = n - 1; r >= 0; --r) {
      double acc = w[r];
      for (int c = r + 1; c < n; ++c) acc -= A[(size_t)r * n + c] * w[c];
      w[r] = acc / A[(size_t)r * n + r];
    }
    return true;
  };
  if (!(yd > -1.0 && yd < 0.0)) {
    err = "control detection plane y_d must lie in (-1, 0)";
    return KMM_ERR_CONFIG;
  }
  if (!solve_t(yd, ops.wlo) || !solve_t(-yd, ops.whi)) {
    err = "singular collocation matrix while building control weights";
    return KMM_ERR_CONFIG;
  }
  return KMM_OK;
}

}  // namespace kmm

extern "C" void kmm_labs_fill_full(double *M0, double *M1, double *M2, double *M3, double *M4,
                                   double *yc, double *yknot, double *int_coeff,
                                   double *center_coeff, int *K, int *N, double *STRETCH,
                                   double *Ly) {
  kmm::HostOps ops;
  const int k = *K, n = *N;
  ops.ny = n;
  ops.k = k;
  kmm::fill_full(k, n, *STRETCH, *Ly, KMM_GRID_SINE, ops);
  double *M[5] = {M0, M1, M2, M3, M4};
  for (int d = 0; d < 5; ++d)
    if (M[d]) std::memcpy(M[d], ops.full[d].data(), sizeof(double) * (size_t)n * n);
  if (yc) std::memcpy(yc, ops.y.data(), sizeof(double) * n);
  if (yknot) std::memcpy(yknot, ops.brk.data(), sizeof(double) * ops.brk.size());
  if (int_coeff) std::memcpy(int_coeff, ops.integ.data(), sizeof(double) * n);
  if (center_coeff) std::memcpy(center_coeff, ops.center.data(), sizeof(double) * n);
}
