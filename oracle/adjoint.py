"""Discrete adjoint of the KMM RK3 step (oracle; TEST INFRASTRUCTURE ONLY).

The reference has no adjoint.  This module is the FP64 reference gradient the GPU adjoint is
checked against: the exact transpose of the step that oracle/kmm.py restates (time_march.f90:36-128
and everything it calls), for a fixed time step, with the opposition control of the v solve's wall
rows (the hook of solve_v_f.f90:251-257) parametrised by an amplitude A and per-mode gains g:
v_wall(m) = A g(m) P(w . v_m), P the projection the physical round trip applies to v (the kz Nyquist
row zeroed, the Hermitian part taken on the kx = 0 plane).

Objective: J = (w_tau / N) sum_n tau_w(n) + (w_q / N) sum_n q_w(n) over N steps, tau_w and q_w the
wall shear stress and wall scalar flux of substep 3 (wave00.f90:210-211, 621-622).

Inner product: <a, b> = Re sum conj(a) b over the stored complex coefficients (and the plain sum
over physical points).  Under it the adjoint of a complex-linear map is its conjugate transpose;
the x-direction c2r and r2c (R-linear) have the weighted forms derived in x_pass_adjoint.

Operators are dense per mode here (np.linalg on (n, n) matrices built with labs.band_to_full):
in exact arithmetic they are the packed-band routines of module_labs.f90, and the grids these
checks run on are small.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import kmm as okmm
from . import labs


# ----------------------------------------------------------------------------------------------
# dense operators
# ----------------------------------------------------------------------------------------------
@dataclass
class Dense:
    M0: np.ndarray
    M1: np.ndarray
    M2: np.ndarray
    M0inv: np.ndarray
    w: np.ndarray  # integration weights (LABS_integration)


def dense(ops: okmm.Operators) -> Dense:
    M0, M1, M2 = (labs.band_to_full(b) for b in (ops.D0, ops.D1, ops.D2))
    return Dense(M0, M1, M2, np.linalg.inv(M0), np.asarray(ops.integ, dtype=np.float64))


def dirichlet(M0, M2, a, b):
    """a M0 - b M2 with the first and last rows reduced to their diagonal (solve_g.f90:45-67),
    batched over modes: a, b (M,) -> (M, n, n)."""
    a = np.atleast_1d(a)
    b = np.atleast_1d(b)
    A = a[:, None, None] * M0[None] - b[:, None, None] * M2[None]
    n = M0.shape[0]
    for r in (0, n - 1):
        d = a * M0[r, r] - b * M2[r, r]
        A[:, r, :] = 0.0
        A[:, r, r] = d
    return A


def vop(M0, M2, k2):
    """D2 - k^2 D0 with D0 rows at the walls (solve_v_f.f90:202-231), (M, n, n)."""
    A = M2[None] - k2[:, None, None] * M0[None]
    n = M0.shape[0]
    for r in (0, n - 1):
        A[:, r, :] = 0.0
        A[:, r, r] = M0[r, r]
    return A


def bsolve(A, b):
    """A x = b per mode: A (M, n, n), b (n, M)."""
    return np.linalg.solve(A, b.T[..., None])[..., 0].T


def bsolve_t(A, b):
    """A^T x = b per mode."""
    return np.linalg.solve(np.transpose(A, (0, 2, 1)), b.T[..., None])[..., 0].T


def zwall(x):
    y = np.array(x)
    y[0] = 0.0
    y[-1] = 0.0
    return y


# ----------------------------------------------------------------------------------------------
# per-mode routines: forward (linear in their line arguments) and transposes
# ----------------------------------------------------------------------------------------------
def hvhg_T(d: Dense, lhg, lhv, lht, kx, kz):
    """Transpose of hvhg.f90:28-163 (linear in u1..u5, u7..u9)."""
    E1T = d.M0inv.T @ d.M1.T
    E2T = d.M0inv.T @ d.M2.T
    kx2, kz2, kxkz = kx * kx, kz * kz, kx * kz
    c2 = kx * kx * kx + kx * (kz * kz)
    c4 = (kx * kx) * kz + kz * kz * kz
    e1hg, e1hv, e2hv, e1ht = E1T @ lhg, E1T @ lhv, E2T @ lhv, E1T @ lht
    l1 = kxkz * lhg - kx2 * e1hv
    l3 = -kxkz * lhg - kz2 * e1hv
    l5 = (kz2 - kx2) * lhg - 2.0 * kxkz * e1hv
    l2 = 1j * kz * e1hg - 1j * c2 * lhv - 1j * kx * e2hv
    l4 = -1j * kx * e1hg - 1j * c4 * lhv - 1j * kz * e2hv
    l7 = 1j * kx * lht
    l9 = 1j * kz * lht
    l8 = -e1ht
    return l1, l2, l3, l4, l5, l7, l8, l9


def helmholtz_coefs(p, kx, kz, s, dt, scalar):
    visc = p.nu / p.pr if scalar else p.nu
    k2 = kx * kx + kz * kz
    beta = dt * okmm.rk(2, s) * visc
    c = {"k2": k2, "beta": beta, "alpha": dt * okmm.rk(1, s) * visc, "gamma": dt * okmm.rk(3, s)}
    if s != 3:
        c["alpha1"] = dt * okmm.rk(1, s + 1) * visc
        c["zeta1"] = dt * okmm.rk(4, s + 1)
    return c


def solve_helmholtz_T(d: Dense, p, lf, lst, kx, kz, s, dt, scalar):
    """Transpose of solve_g.f90:28-201 / solve_t.f90:28-201: (lambda of the new field f and the new
    store) -> (lambda of h, lambda of the old store).  Returns also the operator A."""
    c = helmholtz_coefs(p, kx, kz, s, dt, scalar)
    k2 = c["k2"]
    A = dirichlet(d.M0, d.M2, 1.0 + c["beta"] * k2, c["beta"])
    if s != 3:
        lh = c["zeta1"] * lst
        lft = lf + (1.0 - c["alpha1"] * k2) * lst
        lc = d.M0.T @ lft + d.M2.T @ (c["alpha1"] * lst)
    else:
        lh = np.zeros_like(lf)
        lc = d.M0.T @ (lf + lst)
    lb = zwall(bsolve_t(A, lc))
    if s == 1:
        lstore = (1.0 - c["alpha"] * k2) * lb + c["alpha"] * (d.M0inv.T @ (d.M2.T @ lb))
    else:
        lstore = lb
    lh = lh + c["gamma"] * lb
    return lh, lstore, A


def solve_v_f_T(d: Dense, p, lv, ldv, lsp, Ag, kx, kz, s, dt):
    """Transpose of solve_v_f.f90:38-375 with the wall values as inputs: (lambda v, dv, new
    store_phi) -> (lambda hv, lambda old store_phi, lambda v_wall (2, M))."""
    n = lv.shape[0]
    c = helmholtz_coefs(p, kx, kz, s, dt, False)
    k2 = c["k2"]
    # state-independent pieces (parts 3, 6, 7, 8 of the forward)
    p0 = Ag[:, 0, 0]
    b2 = np.zeros_like(lv)
    b2[0] = p0 + 1j * p0
    c2 = bsolve(Ag, b2)
    buf3 = d.M0 @ c2
    V = vop(d.M0, d.M2, k2)
    ch = bsolve(V, zwall(buf3))
    hh = d.M1 @ ch
    d2h = d.M2 @ c2
    hm = d.M0 @ ch
    den = hh[0] * hh[0] - hh[-1] * hh[-1]
    rev = lambda x: x[::-1]
    # part 8
    lv0 = lv.copy()
    lC1 = np.sum(np.conj(hm) * lv, axis=0)
    lC2 = np.sum(np.conj(rev(hm)) * lv, axis=0)
    # part 7
    if s != 3:
        q, a1 = 1.0 - c["alpha1"] * k2, c["alpha1"]
        lC1 += np.sum(np.conj(q * buf3 + a1 * d2h) * lsp, axis=0)
        lC2 += np.sum(np.conj(q * rev(buf3) + a1 * rev(d2h)) * lsp, axis=0)
    else:
        lC1 += np.sum(np.conj(buf3) * lsp, axis=0)
        lC2 += np.sum(np.conj(rev(buf3)) * lsp, axis=0)
    lsp2 = lsp
    # dv = dv0 + C1 hh - C2 rev(hh)
    ldv0 = ldv.copy()
    lC1 += np.sum(np.conj(hh) * ldv, axis=0)
    lC2 -= np.sum(np.conj(rev(hh)) * ldv, axis=0)
    # C1, C2 from the wall values of dv0
    ldv0[-1] += np.conj(hh[-1] / den) * lC1 + np.conj(hh[0] / den) * lC2
    ldv0[0] += np.conj(-hh[0] / den) * lC1 + np.conj(-hh[-1] / den) * lC2
    # v0 = M0 cv, dv0 = M1 cv, cv = V^-1 r
    lr = bsolve_t(V, d.M0.T @ lv0 + d.M1.T @ ldv0)
    lvwall = np.stack([lr[0], lr[-1]])
    lhv2 = zwall(lr)
    # part 4
    if s != 3:
        lsp1 = lsp2
        lhv2 = lhv2 + (1.0 - c["alpha1"] * k2) * lsp2
        ldva = c["alpha1"] * lsp2
    else:
        lsp1 = np.zeros_like(lsp2)
        lhv2 = lhv2 + lsp2
        ldva = np.zeros_like(lsp2)
    # part 3
    lb = zwall(bsolve_t(Ag, d.M0.T @ lhv2 + d.M2.T @ ldva))
    # part 2
    lhv = np.zeros_like(lv)
    lspin = np.zeros_like(lv)
    if s != 3:
        lhv += c["zeta1"] * lsp1
    else:
        lspin += lsp1
    # part 1
    if s == 1:
        lspin += (1.0 - c["alpha"] * k2) * lb + c["alpha"] * (d.M0inv.T @ (d.M2.T @ lb))
    else:
        lspin += lb
    lhv += c["gamma"] * lb
    return lhv, lspin, lvwall


def solve_u_w_T(lu, lw, kx, kz):
    """Transpose of solve_u_w.f90:18-42: (lambda u, lambda w) -> (lambda g, lambda dv)."""
    k2 = kx * kx + kz * kz
    kxx, kzz = kx / k2, kz / k2
    return 1j * kzz * lu - 1j * kxx * lw, -1j * kxx * lu - 1j * kzz * lw


def mean_line_T(d: Dense, p, line, s, dt, lprof, lstore_new, ltau):
    """Transpose of one mean line of wave00.f90:41-685 (U: line 0, W: 1, Theta: 2): (lambda of the
    new profile, of the new store and of the substep-3 wall stress) -> (lambda of the flux product
    line at (0,0), lambda of the old store).  phi (constant flux / constant bulk scalar) enters
    through its affine dependence on the particular solution."""
    n = d.M0.shape[0]
    visc = p.nu / p.pr if line == 2 else p.nu
    beta = dt * okmm.rk(2, s) * visc
    A0 = dirichlet(d.M0, d.M2, 1.0, beta)[0]
    e_int = np.zeros(n)
    e_int[1:-1] = 1.0
    c_im = np.linalg.solve(A0, e_int)
    I_im = float(d.w @ c_im)
    force = line != 1
    if s != 3:
        a1, z1 = dt * okmm.rk(1, s + 1) * visc, dt * okmm.rk(4, s + 1)
        lprof_t = lprof + lstore_new
        lb1 = d.M0.T @ lprof_t.real + a1 * (d.M2.T @ lstore_new.real)
        ld = -z1 * lstore_new
    else:
        lprof_t = lprof + lstore_new
        lb1 = d.M0.T @ lprof_t.real
        ld = np.zeros(n, dtype=np.complex128)
    if s == 3 and ltau != 0.0:
        g = np.zeros(n)
        g[0], g[1] = d.M1[0, 0], d.M1[0, 1]
        g[-2], g[-1] = -d.M1[-1, -2], -d.M1[-1, -1]
        lb1 = lb1 + ltau * 0.5 * visc * g
    # b1 = c_re + phi c_im, phi = (bulk - w.c_re / 2) / (I_im / 2)
    lcre = lb1 - (d.w / I_im) * float(c_im @ lb1) if force else lb1
    lrhs = np.linalg.solve(A0.T, lcre)
    lt = np.zeros(n, dtype=np.complex128)
    lt[1:-1] = lrhs[1:-1]
    gamma = dt * okmm.rk(3, s)
    if s == 1:
        alpha = dt * okmm.rk(1, s) * visc
        lstore = lt + alpha * (d.M0inv.T @ (d.M2.T @ lt))
    else:
        lstore = lt
    ld = ld - gamma * lt
    lflux = d.M0inv.T @ (d.M1.T @ ld)
    return lflux, lstore


# ----------------------------------------------------------------------------------------------
# control probe
# ----------------------------------------------------------------------------------------------
def project_v(v, p):
    """P(v): the kz Nyquist row zeroed and the Hermitian part on kx = 0, i.e. the v the physical
    round trip returns (vold, dft_x_realspace.f90:123).  v is (nz, nxh, ny)."""
    out = np.array(v)
    nz = p.nz
    out[nz // 2] = 0.0
    k0 = v[:, 0].copy()
    mir = (nz - np.arange(nz)) % nz
    out[:, 0] = 0.5 * (k0 + np.conj(k0[mir]))
    out[nz // 2, 0] = 0.0
    return out


def project_v_T(lv, p):
    """Transpose of project_v (R-linear: conj is self-adjoint under Re <.,.>)."""
    out = np.array(lv)
    nz = p.nz
    out[nz // 2] = 0.0
    k0 = lv[:, 0].copy()
    k0[nz // 2] = 0.0
    mir = (nz - np.arange(nz)) % nz
    out[:, 0] = 0.5 * (k0 + np.conj(k0[mir]))
    out[nz // 2, 0] = 0.0
    return out


# ----------------------------------------------------------------------------------------------
# the x pass: products in physical space
# ----------------------------------------------------------------------------------------------
def c2r(a, nx):
    """dft_x_realspace's pad + unnormalised c2r along the last axis (kx, nxh -> nx32 points)."""
    nxh, nx32 = nx // 2, nx * 3 // 2
    buf = np.zeros(a.shape[:-1] + (nx32 // 2 + 1,), dtype=np.complex128)
    buf[..., :nxh] = a
    return np.fft.irfft(buf, n=nx32, axis=-1) * nx32


def r2c(f, nx):
    return np.fft.rfft(f, axis=-1)[..., : nx // 2]


def c2r_T(mu, nx):
    """Transpose of c2r: weight 1 at kx = 0 (its imaginary part dropped), 2 elsewhere."""
    out = 2.0 * r2c(mu, nx)
    out[..., 0] = 0.5 * out[..., 0].real
    return out


def r2c_T(lam, nx):
    """Transpose of r2c with truncation: Re sum_k lam_k e^{+i k x}."""
    b = np.array(lam) * 0.5
    b[..., 0] = lam[..., 0]
    return c2r(b, nx)


PROD_SLOTS = (0, 1, 2, 3, 4, 6, 7, 8)


def x_pass_T(base_mid, lmid_prod, nx):
    """Transpose of dft_x_realspace's products at the base state.  base_mid: (4, y, z32, kx) the
    x-spectral slabs of u, v, w, theta; lmid_prod: dict slot -> lambda of the product slab.
    Returns the lambda of the four input slabs."""
    u, v, w, t = (c2r(base_mid[i], nx) for i in range(4))
    L = {s: r2c_T(lmid_prod[s], nx) for s in PROD_SLOTS}
    lu = 2.0 * u * L[0] + v * L[1] + w * L[4] + t * L[6]
    lv = -2.0 * v * L[0] + u * L[1] - 2.0 * v * L[2] + w * L[3] + t * L[7]
    lw = 2.0 * w * L[2] + v * L[3] + u * L[4] + t * L[8]
    lt = u * L[6] + v * L[7] + w * L[8]
    return [c2r_T(x, nx) for x in (lu, lv, lw, lt)]


# ----------------------------------------------------------------------------------------------
# substep and step
# ----------------------------------------------------------------------------------------------
def _modes(p):
    kxi, kzi = okmm.wavenumbers(p.nx, p.nz)
    KZ, KX = np.meshgrid(kzi, kxi, indexing="ij")
    mask = ~((KX == 0) & (KZ == 0))
    return mask, (KX[mask] / p.lmfx).astype(np.float64), (KZ[mask] / p.lmfz).astype(np.float64)


def substep_T(d: Dense, ops, p, s, dt, S0, lU, lRK, ctrl, w_tau, w_q, grad):
    """Adjoint of one substep (time_march) at fixed dt.  S0: the substep's starting state
    U (10, nz, nxh, ny) (slots 0, 1, 2, 6 used).  lU (10, ...) slots 0, 1, 2, 6 and lRK (3, ...):
    lambda of the substep's outputs.  Returns (lambda of the starting u, v, w, theta as lU-shaped
    array, lambda of the starting stores); accumulates dJ/dA and dJ/dgains into grad."""
    mask, kx, kz = _modes(p)
    lines = lambda a: np.ascontiguousarray(a[mask].T)
    # wavespace^T, modes other than (0,0)
    lg, ldv = solve_u_w_T(lines(lU[0]), lines(lU[2]), kx, kz)
    lth = lines(lU[6])
    lht, lst, _ = solve_helmholtz_T(d, p, lth, lines(lRK[2]), kx, kz, s, dt, True)
    # solve_g's operator is solve_v_f's input
    cg = helmholtz_coefs(p, kx, kz, s, dt, False)
    Ag = dirichlet(d.M0, d.M2, 1.0 + cg["beta"] * cg["k2"], cg["beta"])
    lhv, lsp, lvwall = solve_v_f_T(d, p, lines(lU[1]), ldv, lines(lRK[1]), Ag, kx, kz, s, dt)
    lhg, lsg, _ = solve_helmholtz_T(d, p, lg, lines(lRK[0]), kx, kz, s, dt, False)
    lp = hvhg_T(d, lhg, lhv, lht, kx, kz)
    lP = np.zeros((10, p.nz, p.nxh, p.ny), dtype=np.complex128)
    for slot, val in zip(PROD_SLOTS, lp):
        lP[slot][mask] = val.T
    lRK0 = np.zeros_like(lRK)
    for slot, val in ((0, lsg), (1, lsp), (2, lst)):
        lRK0[slot][mask] = val.T
    lS = np.zeros_like(lU)
    # control: v_wall = A g P(w . v); the probe reads the starting v
    if ctrl is not None:
        w_lo, w_hi, amp, gains = ctrl
        gm = np.ones((p.nz, p.nxh)) if gains is None else np.asarray(gains, dtype=np.float64)
        vproj = project_v(S0[1], p)
        probe = np.stack([vproj @ w_lo, vproj @ w_hi])          # (2, nz, nxh)
        lw = np.zeros((2, p.nz, p.nxh), dtype=np.complex128)
        lw[:, mask] = lvwall
        contrib = np.sum((np.conj(lw) * probe).real, axis=0)     # d/d(A g) per mode
        grad["gains"] += amp * contrib
        grad["amp"] += float(np.sum(gm * contrib))
        lprobe = amp * gm[None] * lw
        lvp = lprobe[0][..., None] * w_lo + lprobe[1][..., None] * w_hi
        lS[1] += project_v_T(lvp, p)
    # mean lines (0,0)
    i0 = (0, 0)
    for line, (uslot, pslot) in enumerate(((0, 1), (2, 3), (6, 7))):
        ltau = (w_tau if line == 0 else w_q if line == 2 else 0.0)
        lflux, lstore = mean_line_T(d, p, line, s, dt, lU[uslot][i0], lRK[line][i0], ltau)
        lP[pslot][i0] += lflux
        lRK0[line][i0] += lstore
    # transforms^T: P = rescale * x_to_y(products(y_to_x(S)))
    base_mid = np.stack([okmm.y_to_x(S0[f], p.nz32) for f in (0, 1, 2, 6)])
    lmid = {slot: p.rescale * okmm.y_to_x(lP[slot], p.nz32) for slot in PROD_SLOTS}
    lin = x_pass_T(base_mid, lmid, p.nx)
    for f, x in zip((0, 1, 2, 6), lin):
        lS[f] += okmm.x_to_y(x, p.nz)
    return lS, lRK0


def gradient(U0, RK0, ops, p, dt, nsteps, ctrl, w_tau=1.0, w_q=0.0):
    """J and its gradient with respect to the control amplitude and per-mode gains over nsteps
    RK3 steps from (U0, RK0) at fixed dt.  Forward with every substep's starting state kept
    (small grids), then the adjoint backwards.  Returns (J, dJ/dA, dJ/dgains (nz, nxh))."""
    d = dense(ops)
    U, RK = U0.copy(), RK0.copy()
    starts = []
    J = 0.0
    dyr = okmm.dyr_vector(ops.y, p.dy_factor)
    for _ in range(nsteps):
        sc = okmm.Scalars()
        for s in (1, 2, 3):
            starts.append((U.copy(), RK.copy()))
            okmm.time_march(U, RK, ops, p, s, dt, sc, dyr, ctrl)
        J += (w_tau * sc.wall_shear_stress + w_q * sc.wall_theta_stress) / nsteps
    grad = {"amp": 0.0, "gains": np.zeros((p.nz, p.nxh))}
    lU = np.zeros_like(U)
    lRK = np.zeros_like(RK)
    for k in range(len(starts) - 1, -1, -1):
        s = k % 3 + 1
        S0, _ = starts[k]
        wt, wq = (w_tau / nsteps, w_q / nsteps) if s == 3 else (0.0, 0.0)
        lS, lRK = substep_T(d, ops, p, s, dt, S0, lU, lRK, ctrl, wt, wq, grad)
        lU = lS
    return J, grad["amp"], grad["gains"]


def objective(U0, RK0, ops, p, dt, nsteps, ctrl, w_tau=1.0, w_q=0.0):
    """J alone (forward), for finite differences."""
    U, RK = U0.copy(), RK0.copy()
    dyr = okmm.dyr_vector(ops.y, p.dy_factor)
    J = 0.0
    for _ in range(nsteps):
        sc = okmm.Scalars()
        for s in (1, 2, 3):
            okmm.time_march(U, RK, ops, p, s, dt, sc, dyr, ctrl)
        J += (w_tau * sc.wall_shear_stress + w_q * sc.wall_theta_stress) / nsteps
    return J
