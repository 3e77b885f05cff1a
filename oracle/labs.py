"""LABS packed-band linear algebra (oracle restatement of module_labs.f90).

Test infrastructure only (see oracle/__init__.py).

Storage: a band matrix is A[r-1, j-1] = A(r, j) of the Fortran (2*bw+1, ny) array;
column j holds collocation row (point) j.  The first and last bw rows carry the
"near-boundary packed" entries (module_labs.f90:301-328).  Every routine is
vectorised over optional trailing "mode" axes: A may be (2bw+1, n) (one matrix
shared by all modes) or (2bw+1, n, *M); vectors are (n, *M).

The elimination and substitution orders follow the generic routines
fixed_bandec (module_labs.f90:3487-3636), fixed_banbks (:4252-4318) and
LABS_mat_mul_bw (:4687-4722), which the hand-unrolled BW=1..10 variants
specialise.
"""
from __future__ import annotations

import numpy as np


def eval_bw(D0, D1, D2) -> int:
    """LABS_eval_bw, module_labs.f90:245-293.  D* are [point, basis] arrays."""
    F = [np.asarray(D0).T, np.asarray(D1).T, np.asarray(D2).T]  # FULL(basis, point)
    n = F[0].shape[0]
    k = 1
    while True:
        err = 0.0
        for M in F:
            # rows (points) 1..k+1 may touch bases 1..2k+1 only
            blk = M[2 * k + 1 :, : k + 1]
            if blk.size:
                err = max(err, np.abs(blk).max())
            for j in range(k + 2, n - k):  # 1-based j = k+2 .. n-k-1
                lo = M[: j - k - 1, j - 1]
                hi = M[j + k :, j - 1]
                if lo.size:
                    err = max(err, np.abs(lo).max())
                if hi.size:
                    err = max(err, np.abs(hi).max())
            blk = M[: n - 2 * k - 1, n - k - 1 :]
            if blk.size:
                err = max(err, np.abs(blk).max())
        if err <= 0.0:
            return k
        k += 1


def full_to_band(D, bw: int) -> np.ndarray:
    """LABS_full_to_band, module_labs.f90:301-328.  D is [point, basis]."""
    F = np.asarray(D).T  # FULL(i=basis, j=point)
    n = F.shape[0]
    B = np.zeros((2 * bw + 1, n))

    def full(i, j):
        return F[i - 1, j - 1]

    for j in range(1, bw + 1):
        for i in range(1, bw + j + 1):
            B[bw + i - j, j - 1] = full(i, j)
        for i in range(j + bw + 1, 2 * bw + 2):
            B[2 * bw + 1 - i, j - 1] = full(i, j)
    for j in range(bw + 1, n - bw + 1):
        for i in range(1, 2 * bw + 2):
            B[i - 1, j - 1] = full(j + i - bw - 1, j)
    for j in range(n - bw + 1, n + 1):
        for i in range(j - bw, n + 1):
            B[bw + i - j, j - 1] = full(i, j)
        for i in range(n - 2 * bw, j - bw):
            B[n - i, j - 1] = full(i, j)
    return B


def band_to_full(B) -> np.ndarray:
    """Inverse of full_to_band for one matrix: returns the dense [point, basis] matrix."""
    B = np.asarray(B)
    bw = (B.shape[0] - 1) // 2
    n = B.shape[1]
    M = np.zeros((n, n))
    for j in range(1, bw + 1):
        for i in range(1, bw + j + 1):
            M[j - 1, i - 1] = B[bw + i - j, j - 1]
        for i in range(j + bw + 1, 2 * bw + 2):
            M[j - 1, i - 1] = B[2 * bw + 1 - i, j - 1]
    for j in range(bw + 1, n - bw + 1):
        for i in range(1, 2 * bw + 2):
            M[j - 1, j + i - bw - 2] = B[i - 1, j - 1]
    for j in range(n - bw + 1, n + 1):
        for i in range(j - bw, n + 1):
            M[j - 1, i - 1] = B[bw + i - j, j - 1]
        for i in range(n - 2 * bw, j - bw):
            M[j - 1, i - 1] = B[n - i, j - 1]
    return M


def lu(A) -> np.ndarray:
    """fixed_bandec (module_labs.f90:3487-3636): in-place packed-band Crout LU, no pivoting.

    Returns the factored copy.  L keeps the pivots on the diagonal; U is unit upper.
    """
    A = np.array(A, dtype=np.float64, copy=True)
    bw = (A.shape[0] - 1) // 2
    n = A.shape[1]
    m = bw + 1

    def g(r, c):
        return A[r - 1, c - 1]

    def s(r, c, v):
        A[r - 1, c - 1] = v

    # Upper region (:3497-3531)
    for i in range(1, bw + 1):
        dummy = 1.0 / g(m, i)
        for j in range(1, bw + 2 - i):
            acc = g(m + j, i)
            for k in range(1, i):
                acc = acc - g(m - k, i) * g(m + j + k, i - k)
            s(m + j, i, dummy * acc)
        for j in range(bw + 2 - i, bw + 1):
            acc = g(m + j, i)
            for k in range(1, bw - j + 1):
                acc = acc - g(m - k, i) * g(m + j + k, i - k)
            for k in range(bw - j + 1, i):
                acc = acc - g(m - k, i) * g(m + bw - i - j + 1, i - k)
            s(m + j, i, dummy * acc)
        for j in range(i, bw + 1):
            acc = g(m - j, i)
            for k in range(1, i):
                acc = acc - g(m - k, i) * g(m - j, i - k)
            s(m - j, i, dummy * acc)
        for j in range(1, bw + 2 - i):
            acc = g(m + 1 - j, i + j)
            for k in range(1, i + 1):
                acc = acc - g(m + 1 - j - k, i + j) * g(m + k, i + 1 - k)
            s(m + 1 - j, i + j, acc)
        for j in range(bw + 2 - i, bw + 1):
            acc = g(m + 1 - j, i + j)
            for k in range(1, bw + 2 - j):
                acc = acc - g(m + 1 - j - k, i + j) * g(m + k, i + 1 - k)
            s(m + 1 - j, i + j, acc)
    # Subupper region (:3533-3556)
    for i in range(m, 2 * bw + 1):
        dummy = 1.0 / g(m, i)
        for j in range(1, 2 * bw + 2 - i):
            acc = g(m + j, i)
            for k in range(1, bw - j + 1):
                acc = acc - g(m - k, i) * g(m + j + k, i - k)
            for k in range(bw - j + 1, bw + 1):
                acc = acc - g(m - k, i) * g(2 * m - i - j, i - k)
            s(m + j, i, dummy * acc)
        for j in range(2 * bw + 2 - i, bw + 1):
            acc = g(m + j, i)
            for k in range(1, bw - j + 1):
                acc = acc - g(m - k, i) * g(m + j + k, i - k)
            s(m + j, i, dummy * acc)
        for j in range(1, bw + 1):
            acc = g(m - j + 1, i + j)
            for k in range(1, bw + 2 - j):
                acc = acc - g(m - j + 1 - k, i + j) * g(m + k, i - k + 1)
            s(m - j + 1, i + j, acc)
    # Center region (:3561-3576)
    for i in range(2 * bw + 1, n - 2 * bw):
        dummy = 1.0 / g(m, i)
        for j in range(1, bw + 1):
            acc = g(m + j, i)
            for k in range(1, bw - j + 1):
                acc = acc - g(m - k, i) * g(m + j + k, i - k)
            s(m + j, i, dummy * acc)
        for j in range(1, bw + 1):
            acc = g(m - j + 1, i + j)
            for k in range(1, bw - j + 2):
                acc = acc - g(m + 1 - j - k, i + j) * g(m + k, i + 1 - k)
            s(m - j + 1, i + j, acc)
    # Sublower region (:3581-3610)
    for i in range(n - 2 * bw, n - bw):
        dummy = 1.0 / g(m, i)
        for j in range(1, bw + 1):
            acc = g(m + j, i)
            for k in range(1, bw - j + 1):
                acc = acc - g(m - k, i) * g(m + j + k, i - k)
            s(m + j, i, dummy * acc)
        for j in range(1, n - bw - i + 1):
            acc = g(m - j + 1, i + j)
            for k in range(1, bw - j + 2):
                acc = acc - g(m + 1 - j - k, i + j) * g(m + k, i + 1 - k)
            s(m - j + 1, i + j, acc)
        for j in range(n - bw - i + 1, bw + 2):
            acc = g(m - j + 1, i + j)
            for k in range(1, bw + 2 - j):
                acc = acc - g(m + 1 - j - k, i + j) * g(m + k, i + 1 - k)
            for k in range(bw + 2 - j, i - n + 2 * bw + 2):
                acc = acc - g(m + n - bw - 1 + k - i, i + j) * g(m + k, i + 1 - k)
            s(m - j + 1, i + j, acc)
        for j in range(bw + 2, n - i + 1):
            acc = g(m + n - bw - 1 - i, i + j)
            for k in range(1, i - n + 2 * bw + 2):
                acc = acc - g(m + n - bw - 1 - i + k, i + j) * g(m + k, i + 1 - k)
            s(m + n - bw - 1 - i, i + j, acc)
    # Lower region (:3613-3631)
    for i in range(n - bw, n):
        dummy = 1.0 / g(m, i)
        for j in range(1, n - i + 1):
            acc = g(m + j, i)
            for k in range(1, bw - j + 1):
                acc = acc - g(m - k, i) * g(m + j + k, i - k)
            s(m + j, i, dummy * acc)
        for j in range(1, n - i + 1):
            acc = g(m - j + 1, i + j)
            for k in range(1, bw + 2 - j):
                acc = acc - g(m + 1 - j - k, i + j) * g(m + k, i + 1 - k)
            for k in range(bw + 2 - j, bw + 1):
                acc = acc - g(m + n - bw - 1 - i + k, i + j) * g(m + k, i + 1 - k)
            s(m - j + 1, i + j, acc)
    return A


def bs(A, b) -> np.ndarray:
    """fixed_banbks (module_labs.f90:4252-4318): solve with the factored band.

    b may be real or complex, shape (n, *M); a new array is returned.
    """
    A = np.asarray(A)
    b = np.array(b, copy=True)
    bw = (A.shape[0] - 1) // 2
    n = A.shape[1]
    m = bw + 1

    def a(r, c):
        return A[r - 1, c - 1]

    # forward: dummy = L^-1 b, upper part
    for i in range(1, bw + 1):
        acc = b[i - 1]
        for j in range(1, i):
            acc = acc - b[j - 1] * a(m - i + j, i)
        b[i - 1] = acc / a(m, i)
    # centre part
    for i in range(bw + 1, n - bw + 1):
        acc = b[i - 1]
        for j in range(1, bw + 1):
            acc = acc - b[i - bw - 2 + j] * a(m - bw - 1 + j, i)
        b[i - 1] = acc / a(m, i)
    # lower part
    for i in range(1, bw + 1):
        r = n - bw + i
        acc = b[r - 1]
        for j in range(1, i + 1):
            acc = acc - b[n - 2 * bw - 2 + j] * a(m + bw + 1 - j, r)
        for j in range(i + 1, i + bw + 1):
            acc = acc - b[n - 2 * bw - 2 + j] * a(m - bw + j - i - 1, r)
        b[r - 1] = acc / a(m, r)
    # backward: f = U^-1 dummy, lower part
    for i in range(1, bw):
        acc = b[n - i - 1]
        for j in range(1, i + 1):
            acc = acc - b[n - i + j - 1] * a(m + j, n - i)
        b[n - i - 1] = acc
    # centre part
    for i in range(n - bw, bw, -1):
        acc = b[i - 1]
        for j in range(1, bw + 1):
            acc = acc - b[i + j - 1] * a(m + j, i)
        b[i - 1] = acc
    # upper part
    for i in range(1, bw + 1):
        r = bw + 1 - i
        acc = b[r - 1]
        for j in range(1, bw + 1):
            acc = acc - b[r + j - 1] * a(m + j, r)
        for j in range(bw + 1, bw + i + 1):
            acc = acc - b[r + j - 1] * a(m + i - j, r)
        b[r - 1] = acc
    return b


def mat_mul(A, x) -> np.ndarray:
    """LABS_mat_mul_bw (module_labs.f90:4687-4722): b = A x (packed band)."""
    A = np.asarray(A)
    x = np.asarray(x)
    bw = (A.shape[0] - 1) // 2
    n = A.shape[1]
    out = np.zeros((n,) + np.broadcast_shapes(x.shape[1:], A.shape[2:]), dtype=np.result_type(A, x))

    def a(r, c):
        return A[r - 1, c - 1]

    for j in range(1, bw + 1):
        acc = 0.0
        for i in range(1 - j, bw + 1):
            acc = acc + a(bw + 1 + i, j) * x[j + i - 1]
        for i in range(1, bw + 2 - j):
            acc = acc + a(bw + 2 - j - i, j) * x[j + bw + i - 1]
        out[j - 1] = acc
    for j in range(bw + 1, n - bw + 1):
        acc = 0.0
        for i in range(-bw, bw + 1):
            acc = acc + a(bw + 1 + i, j) * x[j + i - 1]
        out[j - 1] = acc
    for j in range(n - bw + 1, n + 1):
        acc = 0.0
        for i in range(-bw, n - j + 1):
            acc = acc + a(bw + 1 + i, j) * x[j + i - 1]
        for i in range(1, j - n + bw + 1):
            acc = acc + a(n + bw + 1 - j + i, j) * x[j - bw - i - 1]
        out[j - 1] = acc
    return out


def integration(w, x):
    """LABS_integration (module_labs.f90:401-413): sum_i w_i x_i, accumulated in order."""
    acc = 0.0
    for i in range(len(w)):
        acc = acc + w[i] * x[i]
    return acc
