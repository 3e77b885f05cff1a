"""B-spline collocation operators (oracle restatement of labs_fill_full.cpp).

Test infrastructure only (see oracle/__init__.py).

The reference builds its wall-normal operators with GSL (labs_fill_full.cpp:35-195):
breakpoints from a uniform or sine ("Jimenez") map (:80-101), a k-fold end knot
vector (gsl_bspline_knots, :103), collocation at the Greville abscissae (:106-117),
the values and derivatives 0..4 of every basis function at every collocation
point (:110-141), Gauss-Legendre integration weights with (k-nderiv+1)/2 points per
breakpoint interval (:206-256) and the basis values at the centre line y=0
(:146-149).  GSL (1.16 / 2.x, makefile:91-92) is not vendored; this module
restates its published conventions:

* knots: t[0..k-1] = y_0, t[k..n-1] = interior breakpoints, t[n..n+k-1] = y_end,
  n = nbreak + k - 2 basis functions (= ny collocation points);
* Greville abscissa i = running mean of t[i+1..i+k-1] (GSL uses gsl_stats_mean,
  a running-mean recurrence, so the same recurrence is used here);
* basis values and derivatives by the Cox-de Boor triangular recursion on the
  knot span t[s] <= x < t[s+1]; at the right end point the last non-empty span
  is used;
* Gauss-Legendre nodes / weights mapped onto each breakpoint interval.
"""
from __future__ import annotations

import math
import numpy as np

PI = 3.141592653589793238462643  # labs_fill_full.cpp:24


def breakpoints(nbreak: int, stretch: float) -> np.ndarray:
    """Breakpoint locations, labs_fill_full.cpp:80-101 (evaluation order kept)."""
    y = np.empty(nbreak)
    if abs(stretch) <= 0.0000000000000001:
        for i in range(nbreak):
            y[i] = -1.0 + 2.0 / (nbreak - 1) * i
    else:
        den = math.sin(stretch * PI / 2.0)
        for i in range(nbreak):
            y[i] = math.sin(stretch * PI / 2.0 * (-1.0 + (2.0 * i) / (nbreak - 1))) / den
    return y


def tanh_breakpoints(nbreak: int, stretch: float, ly: float = 2.0) -> np.ndarray:
    """Tanh map, the commented-out alternative at labs_fill_full.cpp:89."""
    y = np.empty(nbreak)
    for i in range(nbreak):
        y[i] = 0.5 * ly * math.tanh(stretch * (-1.0 + (2.0 * i) / (nbreak - 1))) / math.tanh(stretch)
    return y


def knot_vector(brk: np.ndarray, k: int) -> np.ndarray:
    """k-fold end knots around the interior breakpoints (gsl_bspline_knots)."""
    return np.concatenate([np.full(k, brk[0]), brk[1:-1], np.full(k, brk[-1])])


def greville(t: np.ndarray, k: int, n: int) -> np.ndarray:
    """Greville abscissae as GSL's running mean of k-1 consecutive knots."""
    out = np.empty(n)
    for i in range(n):
        mean = 0.0
        for j in range(k - 1):
            mean += (t[i + 1 + j] - mean) / (j + 1)
        out[i] = mean
    return out


def find_span(t: np.ndarray, k: int, n: int, x: float) -> int:
    """Index s with t[s] <= x < t[s+1] (k-1 <= s <= n-1); right end -> last span."""
    for s in range(k - 1, n):
        if t[s] <= x < t[s + 1]:
            return s
        if t[s] < x and x == t[s + 1] and t[s + 1] == t[n]:
            return s
    raise ValueError("x outside the knot range")


def basis_derivs(t: np.ndarray, k: int, s: int, x: float, nder: int) -> np.ndarray:
    """Derivatives 0..nder of the k basis functions N_{s-k+1..s} of order k at x.

    Cox-de Boor triangular table of the lower-order bases followed by the
    standard derivative recurrence on the coefficient differences.  Returns an
    array (nder+1, k): [d, r] = d-th derivative of basis s-k+1+r.
    """
    p = k - 1
    ndu = np.zeros((k, k))
    left = np.zeros(k)
    right = np.zeros(k)
    ndu[0, 0] = 1.0
    for j in range(1, k):
        left[j] = x - t[s + 1 - j]
        right[j] = t[s + j] - x
        saved = 0.0
        for r in range(j):
            ndu[j, r] = right[r + 1] + left[j - r]          # knot differences (lower triangle)
            temp = ndu[r, j - 1] / ndu[j, r]
            ndu[r, j] = saved + right[r + 1] * temp         # basis values (upper triangle)
            saved = left[j - r] * temp
        ndu[j, j] = saved
    ders = np.zeros((nder + 1, k))
    ders[0, :] = ndu[:, p]
    a = np.zeros((2, k))
    for r in range(k):
        s1, s2 = 0, 1
        a[0, 0] = 1.0
        for d in range(1, nder + 1):
            acc = 0.0
            rk = r - d
            pk = p - d
            if r >= d:
                a[s2, 0] = a[s1, 0] / ndu[pk + 1, rk]
                acc = a[s2, 0] * ndu[rk, pk]
            j1 = 1 if rk >= -1 else -rk
            j2 = d - 1 if (r - 1) <= pk else p - r
            for j in range(j1, j2 + 1):
                a[s2, j] = (a[s1, j] - a[s1, j - 1]) / ndu[pk + 1, rk + j]
                acc += a[s2, j] * ndu[rk + j, pk]
            if r <= pk:
                a[s2, d] = -a[s1, d - 1] / ndu[pk + 1, r]
                acc += a[s2, d] * ndu[r, pk]
            ders[d, r] = acc
            s1, s2 = s2, s1
    fac = float(p)
    for d in range(1, nder + 1):
        ders[d, :] *= fac
        fac *= (p - d)
    return ders


def eval_all(t: np.ndarray, k: int, n: int, x: float, nder: int) -> np.ndarray:
    """(nder+1, n) derivatives of all n basis functions at x (zeros off support)."""
    out = np.zeros((nder + 1, n))
    s = find_span(t, k, n, x)
    d = basis_derivs(t, k, s, x, min(nder, k - 1))
    out[: d.shape[0], s - k + 1 : s + 1] = d
    return out


def gauss_legendre(npts: int):
    x, w = np.polynomial.legendre.leggauss(npts)
    return x, w


def integration_coefficients(t, k, n, brk, nderiv=0):
    """labs_fill_full.cpp:206-256: integral of each basis over [y_0, y_end]."""
    coeffs = np.zeros(n)
    xg, wg = gauss_legendre((k - nderiv + 1) // 2)
    for i in range(len(brk) - 1):
        a, b = brk[i], brk[i + 1]
        for j in range(len(xg)):
            xj = 0.5 * (b + a) + 0.5 * (b - a) * xg[j]
            wj = 0.5 * (b - a) * wg[j]
            s = find_span(t, k, n, xj)
            vals = basis_derivs(t, k, s, xj, nderiv)[nderiv]
            coeffs[s - k + 1 : s + 1] += wj * vals
    return coeffs


def fill_full(k: int, n: int, stretch: float, ly: float = 2.0, grid: str = "sine"):
    """Restatement of LABS_fill_full(M0..M4, yc, yknot, int, center, K, N, STRETCH, Ly).

    k is the GSL order (= input labs_k + 1, module_labs.f90:102-103), n = ny.
    Returns a dict with D[d] (n, n) arrays indexed [point, basis] for d = 0..4
    (the Fortran FULL(basis, point) of module_labs.f90:52-56 is its transpose),
    the collocation points y, breakpoints, knots, integration weights and the
    centre-line evaluation vector.
    """
    nbreak = n - k + 2
    if grid == "sine":
        brk = breakpoints(nbreak, stretch)
    elif grid == "tanh":
        brk = tanh_breakpoints(nbreak, stretch, ly)
    else:
        raise ValueError(grid)
    t = knot_vector(brk, k)
    yc = greville(t, k, n)
    D = np.zeros((5, n, n))
    for i in range(n):
        D[:, i, :] = eval_all(t, k, n, yc[i], 4)
    integ = integration_coefficients(t, k, n, brk)
    center = eval_all(t, k, n, 0.0, 0)[0]
    return {"D": D, "y": yc, "breakpoints": brk, "knots": t, "integ": integ, "center": center}


def eval_vector(ops_or_knots, k: int, n: int, x: float, nder: int = 0) -> np.ndarray:
    """Basis values (or derivative nder) of all n functions at x (like LABS_CENTER_LINE)."""
    t = ops_or_knots["knots"] if isinstance(ops_or_knots, dict) else ops_or_knots
    return eval_all(t, k, n, x, nder)[nder]
