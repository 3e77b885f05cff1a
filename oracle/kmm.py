"""FP64 CPU restatement of one KMM RK3 substep (oracle; test infrastructure only).

Layouts (numpy C-order, i.e. the Fortran shapes reversed):
  state   U[f, kz, kx, y]        = Fortran U(ny, nxh, nz, 10)        (wavespace.f90:29)
  stores  RK[f, kz, kx, y]       = Fortran RK_STORE(ny, nxh, nz, 3)
  X-pencil Up[f, y, z32, kx]     = Fortran Up(nxh, nz32, ny)          (dft_x_realspace.f90:31)
Field slots are 0-based here: slot s here = Fortran field s+1.

Each routine cites the reference routine it restates.  Per-mode routines are
vectorised over the mode axis (vectors are (ny, M)); the y recurrences of the
band solves stay sequential exactly as in module_labs.f90.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import bspline, labs

PI_F = 3.14159265358979323  # module_global_variable.f90:28

# module_runge_kutta.f90:33-48 (alpha, beta, gamma, zeta) per substep 1..3
RK_ALPHA = (29.0 / 96.0, -3.0 / 40.0, 1.0 / 6.0)
RK_BETA = (37.0 / 160.0, 5.0 / 24.0, 1.0 / 6.0)
RK_GAMMA = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
RK_ZETA = (0.0, -17.0 / 60.0, -5.0 / 12.0)


def rk(coef: int, s: int) -> float:
    """RK_3_COEF(coef, s) with 1-based coef (1=alpha .. 4=zeta) and substep s."""
    return (RK_ALPHA, RK_BETA, RK_GAMMA, RK_ZETA)[coef - 1][s - 1]


# ----------------------------------------------------------------------------
# set-up
# ----------------------------------------------------------------------------
@dataclass
class Params:
    nx: int
    ny: int
    nz: int
    labs_k: int = 6
    lmfx: float = 1.0
    lmfy: float = 1.0
    lmfz: float = 0.5
    stretch: float = 0.9
    nu: float = 1.0 / 2800.0
    pr: float = 0.71
    bulk_u: float = 1.0
    bulk_w: float = 0.0
    bulk_t: float = 1.0
    u_gal: float = 0.0
    cfl: float = 1.0
    dt_factor: float = 0.0
    dy_factor: float = 1.0
    fixed_dt: bool = True
    grid: str = "sine"
    control_amp: float = 0.0        # opposition control amplitude A (0 = off, the reference)
    control_yplus: float = 15.0
    re_tau: float = 180.0
    gains: np.ndarray | None = None  # per-(kz,kx) control gains, default 1
    n_scalar: int = 1                # passive scalars: 1 (the reference) or 2
    pr2: float = 0.2                 # Prandtl number of the second scalar
    bulk_t2: float = 1.0             # target bulk value of the second scalar

    @property
    def nslots(self):
        """Field slots of U: the reference's 10, plus theta2 and its three products (u, v, w
        times theta2) in slots 10..13 when a second scalar runs."""
        return 10 if self.n_scalar == 1 else 14

    # derived, read_input_file.f90:94-116
    @property
    def nxh(self):
        return self.nx // 2

    @property
    def nx32(self):
        return self.nx * 3 // 2

    @property
    def nz32(self):
        return self.nz * 3 // 2

    @property
    def lx(self):
        return self.lmfx * 2 * PI_F

    @property
    def lz(self):
        return self.lmfz * 2 * PI_F

    @property
    def ly(self):
        return self.lmfy * 2

    @property
    def rescale(self):
        return 1.0 / (self.nx32 * self.nz32)

    @property
    def dxr(self):
        return float(self.nx) / self.lx

    @property
    def dzr(self):
        return float(self.nz) / self.lz

    @property
    def cflx(self):
        return self.cfl / PI_F


@dataclass
class Operators:
    bw: int
    y: np.ndarray
    D0: np.ndarray   # bands (2bw+1, ny)
    D1: np.ndarray
    D2: np.ndarray
    D0_lu: np.ndarray
    integ: np.ndarray
    center: np.ndarray
    full: dict = field(repr=False, default=None)


def make_operators(p: Params) -> Operators:
    """LABS_initialize (module_labs.f90:77-238): GSL order = labs_k + 1."""
    k = p.labs_k + 1
    full = bspline.fill_full(k, p.ny, p.stretch, p.ly, p.grid)
    D = full["D"]
    bw = labs.eval_bw(D[0], D[1], D[2])
    b0, b1, b2 = (labs.full_to_band(D[d], bw) for d in range(3))
    return Operators(bw=bw, y=full["y"], D0=b0, D1=b1, D2=b2, D0_lu=labs.lu(b0),
                     integ=full["integ"], center=full["center"], full=full)


def wavenumbers(nx: int, nz: int):
    """set_waveno, module_ppdfftw.f90:347-384 (single rank)."""
    nxh = nx // 2
    nzh = nz // 2
    kx = np.arange(nxh, dtype=np.int64)
    kz = np.empty(nz, dtype=np.int64)
    for i in range(1, nzh + 2):
        kz[i - 1] = i - 1
    for i in range(nzh + 2, nz + 1):
        kz[i - 1] = i - 2 * nzh - 1
    return kx, kz


def dyr_vector(y: np.ndarray, dy_factor: float) -> np.ndarray:
    """ppdfftw_initialize, module_ppdfftw.f90:573-583."""
    ny = len(y)
    out = np.empty(ny)
    for i in range(1, ny + 1):
        if i == 1:
            out[0] = 1.0 / (dy_factor * abs(y[1] - y[0]))
        elif i == ny:
            out[ny - 1] = 1.0 / (dy_factor * abs(y[ny - 1] - y[ny - 2]))
        else:
            out[i - 1] = 1.0 / (dy_factor * min(abs(y[i - 1] - y[i - 2]), abs(y[i - 1] - y[i])))
    return out


# ----------------------------------------------------------------------------
# transforms (rows 3-10)
# ----------------------------------------------------------------------------
def y_to_x(Uf: np.ndarray, nz32: int) -> np.ndarray:
    """y_to_x.f90:21-50 for one field: Y-pencil [kz,kx,y] -> X-pencil [y,z32,kx].

    Transpose to Z-pencil (on_node_reorder_y_to_z, module_ppdfftw.f90:1019-1048),
    pad (ppdfftw_dft_z_inverse :846-854: keep 1..nh, zero nh+1..2nh+1, shift the
    negative modes up), unnormalised FFTW_BACKWARD along z, transpose to X-pencil
    (on_node_reorder_z_to_x :1083-1113).
    """
    nz, nxh, ny = Uf.shape
    nh = nz // 2
    zp = np.transpose(Uf, (1, 2, 0))            # [kx, y, kz]  (Fortran (nz, ny, nxh))
    buf = np.zeros((nxh, ny, nz32), dtype=np.complex128)
    buf[:, :, :nh] = zp[:, :, :nh]
    buf[:, :, 2 * nh + 1 :] = zp[:, :, nh + 1 :]
    big = np.fft.ifft(buf, axis=-1) * nz32       # e^{+i}, unnormalised
    return np.ascontiguousarray(np.transpose(big, (1, 2, 0)))  # [y, z32, kx]


def x_to_y(Upf: np.ndarray, nz: int) -> np.ndarray:
    """x_to_y.f90:21-46 for one field: X-pencil [y,z32,kx] -> Y-pencil [kz,kx,y].

    FFTW_FORWARD along z, keep 1..nh, zero nh+1 (the kz Nyquist), U(j-nh) = buf(j)
    for j = 2nh+2..nz32 (ppdfftw_dft_z_forward, module_ppdfftw.f90:809-818).
    """
    ny, nz32, nxh = Upf.shape
    nh = nz // 2
    zp = np.transpose(Upf, (2, 0, 1))           # [kx, y, z32]
    big = np.fft.fft(zp, axis=-1)
    small = np.zeros((nxh, ny, nz), dtype=np.complex128)
    small[:, :, :nh] = big[:, :, :nh]
    small[:, :, nh + 1 :] = big[:, :, 2 * nh + 1 :]
    return np.ascontiguousarray(np.transpose(small, (2, 0, 1)))  # [kz, kx, y]


def dft_x_realspace(Up: np.ndarray, nx: int, substep: int, dxr: float, dzr: float, dyr: np.ndarray,
                    stat: bool = False):
    """dft_x_realspace.f90:68-213: per x-line pad, c2r, products, CFL max, r2c, truncate.

    Up is [10, y, z32, kx] complex; slots 0,1,2,6 (u,v,w,theta) are read, slots
    0..4 and 6..9 are written, and slot 5 (f6 = v v, dft_x_realspace.f90:192-199) on a
    statistics substep (stat).  Returns velmax (substep 1) or 0.
    """
    nxh = nx // 2
    nx32 = nx * 3 // 2
    nfreq = nx32 // 2 + 1

    def c2r(a):
        buf = np.zeros(a.shape[:-1] + (nfreq,), dtype=np.complex128)
        buf[..., :nxh] = a
        return np.fft.irfft(buf, n=nx32, axis=-1) * nx32   # unnormalised c2r

    u = c2r(Up[0]); v = c2r(Up[1]); w = c2r(Up[2]); t = c2r(Up[6])
    bv2 = v * v
    prods = {8: w * t, 7: v * t, 6: u * t, 4: u * w, 3: v * w, 2: w * w - bv2,
             1: u * v, 0: u * u - bv2, 9: v}
    if Up.shape[0] > 10:
        # a second passive scalar theta2 (slot 10): its products u, v, w theta2 in slots 11..13,
        # formed like f7..f9 (dft_x_realspace.f90:119-121)
        t2 = c2r(Up[10])
        prods.update({11: u * t2, 12: v * t2, 13: w * t2})
    if stat:
        prods[5] = bv2
    velmax = 0.0
    if substep == 1:
        vel = (np.abs(u) * dxr) + (np.abs(v) * dyr[:, None, None]) + (np.abs(w) * dzr)
        velmax = float(vel.max())
    for slot, f in prods.items():
        Up[slot] = np.fft.rfft(f, axis=-1)[..., :nxh]
    return velmax


# ----------------------------------------------------------------------------
# per-mode physics (rows 12-17); vectors are (ny, M), kx/kz are (M,)
# ----------------------------------------------------------------------------
def hvhg(u1, u2, u3, u4, u5, u7, u8, u9, ops: Operators, kx, kz):
    """hvhg.f90:28-163.  Returns (hg, hv, ht)."""
    bs, mm = labs.bs, labs.mat_mul
    kz2 = kz * kz
    kx2 = kx * kx
    kxkz = kx * kz
    ikx = 1j * kx
    ikz = 1j * kz
    ikx3 = 1j * (kx * kx * kx)
    ikxkz2 = 1j * (kx * (kz * kz))
    ikx2kz = 1j * ((kx * kx) * kz)
    ikz3 = 1j * (kz * kz * kz)
    dummy = u1
    u1 = kxkz * (u1 - u3) + (kz2 - kx2) * u5
    u3 = -kx2 * dummy - 2.0 * kxkz * u5 - kz2 * u3
    u3 = bs(ops.D0_lu, u3)
    u5 = mm(ops.D1, u3)
    u5 = u5 + (ikx3 + ikxkz2) * u2 + (ikx2kz + ikz3) * u4
    u3, u4 = ikx * u4 - ikz * u2, ikz * u4 + ikx * u2
    u3 = bs(ops.D0_lu, u3)
    u2 = mm(ops.D1, u3)
    u4 = bs(ops.D0_lu, u4)
    u3 = mm(ops.D2, u4)
    u5 = u5 + u3
    u1 = u1 + u2
    u7 = ikx * u7 + ikz * u9
    u8 = bs(ops.D0_lu, u8)
    u9 = mm(ops.D1, u8)
    u7 = -(u7 + u9)
    return u1, u5, u7


def _helmholtz_band(ops: Operators, a, b):
    """a*D0 - b*D2 per mode with the Dirichlet first/last rows (solve_g.f90:45-67)."""
    bw = ops.bw
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    A = a[None, None] * ops.D0[..., None] - b[None, None] * ops.D2[..., None] if a.ndim else \
        a * ops.D0 - b * ops.D2
    A = np.array(A)
    for col in (0, -1):
        diag = a * ops.D0[bw, col] - b * ops.D2[bw, col]
        A[:, col] = 0.0
        A[bw, col] = diag
    return A


def solve_scalar_helmholtz(u, store, ops: Operators, kx, kz, diff, s, dt):
    """solve_g.f90:28-201 (diff = nu) and solve_t.f90:28-201 (diff = nu/pr).

    Returns (new field, new store, factored band).  diff is passed as the
    (nu, pr) pair so the products keep the reference's evaluation order.
    """
    bs, mm = labs.bs, labs.mat_mul
    nu, pr = diff
    k2 = kx ** 2 + kz ** 2

    def visc(c):
        v = dt * c * nu
        return v if pr is None else v / pr

    beta = visc(rk(2, s))
    dummy = 1.0 + beta * k2
    D_buf = labs.lu(_helmholtz_band(ops, dummy, np.broadcast_to(beta, dummy.shape)))
    if s == 1:
        alpha = visc(rk(1, s))
        gamma = dt * rk(3, s)
        dummy = 1.0 - alpha * k2
        buf1 = dummy * store + gamma * u
        c = bs(ops.D0_lu, store)
        buf2 = mm(ops.D2, c)
        buf1 = buf1 + alpha * buf2
    else:
        gamma = dt * rk(3, s)
        buf1 = store + gamma * u
    buf1 = np.array(buf1)
    buf1[0] = 0.0
    buf1[-1] = 0.0
    if s != 3:
        zeta = dt * rk(4, s + 1)
        store = zeta * u
    buf1 = bs(D_buf, buf1)
    u = mm(ops.D0, buf1)
    buf2 = mm(ops.D2, buf1)
    if s != 3:
        alpha = visc(rk(1, s + 1))
        dummy = 1.0 - alpha * k2
        store = store + dummy * u + alpha * buf2
    else:
        store = u.copy()
    return u, store, D_buf


def solve_v_f(hv, store_phi, vold, ops: Operators, D_buf_g, kx, kz, nu, s, dt, vwall=None):
    """solve_v_f.f90:38-375.  Returns (v, dv/dy, store_phi).

    vwall, when given, is the (2, M) wall-normal velocity imposed at the first
    and last collocation rows of the v Poisson solve (the opposition-control
    hook at solve_v_f.f90:251-257; the reference itself sets 0).
    """
    bs, mm = labs.bs, labs.mat_mul
    bw = ops.bw
    k2 = kx ** 2 + kz ** 2
    # Part 1
    if s == 1:
        alpha = dt * rk(1, s) * nu
        gamma = dt * rk(3, s)
        dummy = 1.0 - alpha * k2
        buf1 = dummy * store_phi + gamma * hv
        c = bs(ops.D0_lu, store_phi)
        buf2 = mm(ops.D2, c)
        buf1 = buf1 + alpha * buf2
    else:
        gamma = dt * rk(3, s)
        buf1 = store_phi + gamma * hv
    buf1 = np.array(buf1)
    buf1[0] = 0.0
    buf1[-1] = 0.0
    # Part 2
    if s != 3:
        zeta = dt * rk(4, s + 1)
        store_phi = zeta * hv
    # Part 3
    buf2 = np.zeros_like(buf1)
    buf2[0] = D_buf_g[bw, 0] + 1j * D_buf_g[bw, 0]
    buf1 = bs(D_buf_g, buf1)
    buf2 = bs(D_buf_g, buf2)
    hv = mm(ops.D0, buf1)
    buf3 = mm(ops.D0, buf2)
    dv = mm(ops.D2, buf1)
    # Part 4
    if s != 3:
        alpha = dt * nu * rk(1, s + 1)
        dummy = 1.0 - alpha * k2
        store_phi = store_phi + dummy * hv + alpha * dv
    else:
        store_phi = hv.copy()
    # Part 5: (D2 - k2 D0) with D0 Dirichlet rows
    M = kx.shape
    A = (-k2)[None, None] * ops.D0[..., None] + ops.D2[..., None] if len(M) else -k2 * ops.D0 + ops.D2
    A = np.array(A)
    for col in (0, -1):
        A[:, col] = 0.0
        A[bw, col] = ops.D0[bw, col]
    D_buf = labs.lu(A)
    # Part 6
    hv = np.array(hv)
    if vwall is None:
        hv[0] = 0.0
        hv[-1] = 0.0
    else:
        hv[0] = vwall[0]
        hv[-1] = vwall[1]
    hv = bs(D_buf, hv)
    buf1 = np.array(buf3)
    buf1[0] = 0.0
    buf1[-1] = 0.0
    buf1 = bs(D_buf, buf1)
    v = mm(ops.D0, hv)
    dv = mm(ops.D1, hv)
    hv = mm(ops.D1, buf1)
    den = hv[0] * hv[0] - hv[-1] * hv[-1]
    C1 = (hv[-1] * dv[-1] - hv[0] * dv[0]) / den
    C2 = (hv[0] * dv[-1] - hv[-1] * dv[0]) / den
    dv = dv + C1 * hv - C2 * hv[::-1]
    # Part 7
    hv = mm(ops.D2, buf2)
    if s != 3:
        alpha = dt * nu * rk(1, s + 1)
        dummy = 1.0 - alpha * k2
        store_phi = (store_phi + C1 * dummy * buf3 + C2 * dummy * buf3[::-1]
                     + C1 * alpha * hv + C2 * alpha * hv[::-1])
    else:
        store_phi = store_phi + C1 * buf3 + C2 * buf3[::-1]
    # Part 8
    hv = mm(ops.D0, buf1)
    v = v + C1 * hv + C2 * hv[::-1]
    return v, dv, store_phi


def solve_u_w(g, f, kx, kz):
    """solve_u_w.f90:18-42.  Returns (u, w)."""
    kxx = (1j * kx) / (kx * kx + kz * kz)
    kzz = (1j * kz) / (kx * kx + kz * kz)
    dxg = kxx * g
    dzg = kzz * g
    dxf = kxx * f
    dzf = kzz * f
    return dxf - dzg, dxg + dzf


def calculate_phi(bulk, integral):
    """wave00.f90:704-714."""
    return (bulk - 0.5 * integral.real) / (0.5 * integral.imag)


def wave00(u2, u4, u8, store1, store2, store3, ops: Operators, p: Params, s, dt, theta2=None):
    """wave00.f90:41-685 for the kx = kz = 0 mode (1-D complex lines of ny).

    Returns dict with u, w, theta (new mean profiles), the stores, phi_dpdx,
    phi_dtdx and (substep 3) the wall shear stress / wall scalar flux.
    """
    bs, mm = labs.bs, labs.mat_mul
    bw, ny = ops.bw, p.ny
    nu, pr = p.nu, p.pr
    out = {}

    def lhs(beta):
        A = ops.D0 - beta * ops.D2
        for col in (0, -1):
            A[:, col] = 0.0
            A[bw, col] = ops.D0[bw, col] - beta * ops.D2[bw, col]
        return labs.lu(A)

    def wall_grad(c):
        D1 = ops.D1
        return (D1[bw, 0] * c[0].real + D1[bw + 1, 0] * c[1].real
                - D1[bw - 1, ny - 1] * c[ny - 2].real - D1[bw, ny - 1] * c[ny - 1].real)

    def mean_line(store, flux_prod, visc, bulk, gal, force):
        """One of the three blocks of wave00 (U: :58-257, W: :298-443, Theta: :473-667)."""
        D_buf = lhs(dt * rk(2, s) * visc)
        buf1 = np.zeros(ny, dtype=np.complex128)
        if s == 1:
            c = bs(ops.D0_lu, store)
            b = bs(ops.D0_lu, flux_prod)
            buf1 = mm(ops.D2, c)
            d = mm(ops.D1, b)
            alpha = dt * rk(1, s) * visc
            gamma = dt * rk(3, s)
            buf1[1:] = store[1:] + alpha * buf1[1:] - gamma * d[1:]
        else:
            b = bs(ops.D0_lu, flux_prod)
            d = mm(ops.D1, b)
            gamma = dt * rk(3, s)
            buf1[1:] = store[1:] - gamma * d[1:]
        buf1[0] = 0.0
        buf1[1:-1] = (buf1[1:-1].real + gal) + 1j
        buf1[-1] = 0.0
        buf1 = bs(D_buf, buf1)
        integral = labs.integration(ops.integ, buf1)
        phi = calculate_phi(bulk, integral)
        if not force:
            phi = 0.0
        buf1 = (buf1.real + phi * buf1.imag) + 0j
        prof = mm(ops.D0, buf1)
        if s != 3:
            st = mm(ops.D2, buf1)
            alpha = dt * rk(1, s + 1) * visc
            zeta = dt * rk(4, s + 1)
        return buf1, prof, phi, (lambda prof_: alpha * st + prof_ - zeta * d) if s != 3 else None

    # U block
    buf1, u1, phi, upd = mean_line(store1, u2, nu, p.bulk_u, p.u_gal, True)
    out["phi_dpdx"] = phi
    if s == 3:
        out["wall_shear_stress"] = 0.5 * nu * wall_grad(buf1)
    u1 = u1 - p.u_gal
    out["store1"] = upd(u1) if upd else u1.copy()
    out["u"] = u1
    # W block (phi forced to 0, wave00.f90:396)
    buf1, u3, _, upd = mean_line(store2, u4, nu, p.bulk_w, 0.0, False)
    out["store2"] = upd(u3) if upd else u3.copy()
    out["w"] = u3
    out["v"] = np.zeros(ny, dtype=np.complex128)
    # Theta block (constant bulk theta, wave00.f90:606-623)
    visc_t = nu / pr
    buf1, u7, phi_t, upd = mean_line(store3, u8, visc_t, p.bulk_t, 0.0, True)
    out["phi_dtdx"] = phi_t
    if s == 3:
        out["wall_theta_stress"] = 0.5 * nu / pr * wall_grad(buf1)
    out["store3"] = upd(u7) if upd else u7.copy()
    out["theta"] = u7
    if theta2 is not None:
        # the second scalar's mean line, same block with nu/pr2 and its own bulk value
        u12, store4 = theta2
        visc_t2 = nu / p.pr2
        buf1, u11, phi_t2, upd = mean_line(store4, u12, visc_t2, p.bulk_t2, 0.0, True)
        out["phi_dtdx2"] = phi_t2
        if s == 3:
            out["wall_theta_stress2"] = 0.5 * nu / p.pr2 * wall_grad(buf1)
        out["store4"] = upd(u11) if upd else u11.copy()
        out["theta2"] = u11
    return out


# ----------------------------------------------------------------------------
# opposition control (build extension at solve_v_f.f90:251-257)
# ----------------------------------------------------------------------------
def control_weights(ops: Operators, p: Params):
    """Vectors w_lo, w_hi with v(y_d) = w . v_values for the two detection planes.

    v(y_d) = e_d^T D0^{-1} v where e_d holds the basis values at y_d (built like
    LABS_CENTER_LINE, labs_fill_full.cpp:146-149).
    """
    yd = -1.0 + p.control_yplus / p.re_tau
    k = p.labs_k + 1
    e_lo = bspline.eval_vector(ops.full, k, p.ny, yd)
    e_hi = bspline.eval_vector(ops.full, k, p.ny, -yd)
    D0 = ops.full["D"][0]
    return np.linalg.solve(D0.T, e_lo), np.linalg.solve(D0.T, e_hi)


# ----------------------------------------------------------------------------
# wavespace + time_march
# ----------------------------------------------------------------------------
@dataclass
class Scalars:
    phi_dpdx: list = field(default_factory=lambda: [0.0] * 4)
    phi_dtdx: list = field(default_factory=lambda: [0.0] * 4)
    wall_shear_stress: float = 0.0
    wall_theta_stress: float = 0.0
    velmax: float = 0.0
    dt: float = 0.0
    phi_dtdx2: list = field(default_factory=lambda: [0.0] * 4)
    wall_theta_stress2: float = 0.0


def wavespace(U, RK, ops: Operators, p: Params, s: int, dt: float, sc: Scalars, ctrl=None):
    """wavespace.f90:22-113: (0,0) -> wave00, others -> hvhg, solve_g, solve_v_f, solve_u_w, solve_t."""
    kxi, kzi = wavenumbers(p.nx, p.nz)
    nz, nxh = len(kzi), len(kxi)
    KZ, KX = np.meshgrid(kzi, kxi, indexing="ij")
    mask = ~((KX == 0) & (KZ == 0))
    kx = (KX[mask] * (1.0 / p.lmfx)).astype(np.float64)
    kz = (KZ[mask] * (1.0 / p.lmfz)).astype(np.float64)

    def lines(slot, arr=U):
        return np.ascontiguousarray(arr[slot][mask].T)  # (ny, M)

    u1, u2, u3, u4, u5, u7, u8, u9, u10 = (lines(i) for i in (0, 1, 2, 3, 4, 6, 7, 8, 9))
    sg, sp, st = lines(0, RK), lines(1, RK), lines(2, RK)
    # (0,0) first: it reads the unmodified product lines
    i0 = np.argwhere((KX == 0) & (KZ == 0))[0]
    two = p.n_scalar == 2
    m00 = wave00(U[1][tuple(i0)], U[3][tuple(i0)], U[7][tuple(i0)],
                 RK[0][tuple(i0)], RK[1][tuple(i0)], RK[2][tuple(i0)], ops, p, s, dt,
                 (U[12][tuple(i0)], RK[3][tuple(i0)]) if two else None)
    hg, hv, ht = hvhg(u1, u2, u3, u4, u5, u7, u8, u9, ops, kx, kz)
    g, sg, D_buf_g = solve_scalar_helmholtz(hg, sg, ops, kx, kz, (p.nu, None), s, dt)
    vwall = None
    if ctrl is not None:
        w_lo, w_hi, amp, gains = ctrl
        gm = gains[mask] if gains is not None else 1.0
        vwall = np.stack([amp * gm * (w_lo @ u10), amp * gm * (w_hi @ u10)])
    v, dv, sp = solve_v_f(hv, sp, u10, ops, D_buf_g, kx, kz, p.nu, s, dt, vwall)
    u, w = solve_u_w(g, dv, kx, kz)
    th, st, _ = solve_scalar_helmholtz(ht, st, ops, kx, kz, (p.nu, p.pr), s, dt)
    for slot, val in ((0, u), (1, v), (2, w), (6, th)):
        U[slot][mask] = val.T
    for slot, val in ((0, sg), (1, sp), (2, st)):
        RK[slot][mask] = val.T
    if two:
        # theta2: h = -(i kx (u theta2) + i kz (w theta2) + D1 D0^-1 (v theta2)) as hvhg forms h_theta
        # (hvhg.f90:146-159), then solve_t with pr2
        u11, u12, u13, s4 = lines(11), lines(12), lines(13), lines(3, RK)
        ht2 = -((1j * kx) * u11 + (1j * kz) * u13 + labs.mat_mul(ops.D1, labs.bs(ops.D0_lu, u12)))
        th2, s4, _ = solve_scalar_helmholtz(ht2, s4, ops, kx, kz, (p.nu, p.pr2), s, dt)
        U[10][mask] = th2.T
        RK[3][mask] = s4.T
    idx = tuple(i0)
    U[0][idx], U[1][idx], U[2][idx], U[6][idx] = m00["u"], m00["v"], m00["w"], m00["theta"]
    RK[0][idx], RK[1][idx], RK[2][idx] = m00["store1"], m00["store2"], m00["store3"]
    sc.phi_dpdx[s - 1] = m00["phi_dpdx"]
    sc.phi_dtdx[s - 1] = m00["phi_dtdx"]
    if s == 3:
        sc.wall_shear_stress = m00["wall_shear_stress"]
        sc.wall_theta_stress = m00["wall_theta_stress"]
    if two:
        U[10][idx] = m00["theta2"]
        RK[3][idx] = m00["store4"]
        sc.phi_dtdx2[s - 1] = m00["phi_dtdx2"]
        if s == 3:
            sc.wall_theta_stress2 = m00["wall_theta_stress2"]


class DtError(RuntimeError):
    """dft_x_realspace.f90:494-497 aborts the run when dt leaves (1e-14, 1e5]."""


def time_march(U, RK, ops: Operators, p: Params, s: int, dt: float, sc: Scalars, dyr=None, ctrl=None):
    """time_march.f90:36-128 (non-statistics substep).  Returns the dt used.

    U (10, nz, nxh, ny) and RK (3, nz, nxh, ny) complex128 are updated in place.
    """
    if dyr is None:
        dyr = dyr_vector(ops.y, p.dy_factor)
    two = p.n_scalar == 2
    Up = np.zeros((p.nslots, p.ny, p.nz32, p.nxh), dtype=np.complex128)
    for f in (0, 1, 2, 6) + ((10,) if two else ()):
        Up[f] = y_to_x(U[f], p.nz32)
    velmax = dft_x_realspace(Up, p.nx, s, p.dxr, p.dzr, dyr)
    if s == 1:
        sc.velmax = velmax
        if not p.fixed_dt:
            dt = p.dt_factor * dt + (1.0 - p.dt_factor) * p.cflx / velmax
        if dt <= 1e-14 or dt > 1e5:
            raise DtError(f"ABORT due to timestep dt = {dt}")
    for f in (0, 1, 2, 3, 4, 6, 7, 8, 9) + ((11, 12, 13) if two else ()):
        U[f] = x_to_y(Up[f], p.nz)
    if two:
        theta2 = U[10].copy()
        U *= p.rescale
        U[10] = theta2  # the scalar itself is not a transformed product
    else:
        U *= p.rescale
    wavespace(U, RK, ops, p, s, dt, sc, ctrl)
    sc.dt = dt
    return dt


def rk3_step(U, RK, ops, p, dt, sc=None, dyr=None, ctrl=None):
    """Three substeps of main.f90:134-156; phi_dpdx(4) = sum/dt (main.f90:147-148)."""
    sc = sc or Scalars()
    for s in (1, 2, 3):
        dt = time_march(U, RK, ops, p, s, dt, sc, dyr, ctrl)
    sc.phi_dpdx[3] = (sc.phi_dpdx[0] + sc.phi_dpdx[1] + sc.phi_dpdx[2]) / dt
    sc.phi_dtdx[3] = (sc.phi_dtdx[0] + sc.phi_dtdx[1] + sc.phi_dtdx[2]) / dt
    sc.phi_dtdx2[3] = (sc.phi_dtdx2[0] + sc.phi_dtdx2[1] + sc.phi_dtdx2[2]) / dt
    return dt, sc


def set_initial_data_uvw(U, ops: Operators, p: Params):
    """initial_step.f90:139-179: RK stores from u, v, w, theta (returns RK)."""
    kxi, kzi = wavenumbers(p.nx, p.nz)
    RK = np.zeros((3 + (p.n_scalar - 1), p.nz, p.nxh, p.ny), dtype=np.complex128)
    if p.n_scalar == 2:
        RK[3] = U[10]  # the second scalar's store is the scalar (as RK_STORE 3 is theta)
    lmfxr, lmfzr = 1.0 / p.lmfx, 1.0 / p.lmfz
    for j, kzv in enumerate(kzi):
        for k, kxv in enumerate(kxi):
            if kxv == 0 and kzv == 0:
                RK[0, j, k] = U[0, j, k]
                RK[1, j, k] = U[2, j, k]
                RK[2, j, k] = U[6, j, k]
            else:
                c = labs.bs(ops.D0_lu, U[1, j, k])
                d2 = labs.mat_mul(ops.D2, c)
                kxr, kzr = kxv * lmfxr, kzv * lmfzr
                RK[1, j, k] = d2 - (kxr ** 2 + kzr ** 2) * U[1, j, k]
                RK[0, j, k] = (1j * kzr) * U[0, j, k] - (1j * kxr) * U[2, j, k]
                RK[2, j, k] = U[6, j, k]
    return RK


def set_initial_data_gphi(RK, ops: Operators, p: Params):
    """initial_step.f90:430-513 (restart option 2): u, v, w and theta from the stores g, phi,
    theta (RK[0..2]; their (0, 0) mode holds the mean U, W, theta).  Returns U (10 fields)."""
    kxi, kzi = wavenumbers(p.nx, p.nz)
    U = np.zeros((10, p.nz, p.nxh, p.ny), dtype=np.complex128)
    lmfxr, lmfzr = 1.0 / p.lmfx, 1.0 / p.lmfz
    ny, bw = p.ny, ops.bw
    for j, kzv in enumerate(kzi):
        for k, kxv in enumerate(kxi):
            if kxv == 0 and kzv == 0:
                U[0, j, k], U[2, j, k], U[6, j, k] = RK[0, j, k], RK[1, j, k], RK[2, j, k]
                continue
            k2 = (kzv * lmfzr) ** 2 + (kxv * lmfxr) ** 2
            kxx, kzz = 1j * kxv * lmfxr / k2, 1j * kzv * lmfzr / k2
            D = -k2 * ops.D0 + ops.D2
            for col in (0, ny - 1):  # Dirichlet rows: only the diagonal of D2 - k^2 D0
                keep = D[bw, col]
                D[:, col] = 0.0
                D[bw, col] = keep
            c = RK[1, j, k].copy()
            c[0] = c[-1] = 0.0
            c = labs.bs(labs.lu(D), c)
            U[1, j, k] = labs.mat_mul(ops.D0, c)
            dv = labs.mat_mul(ops.D1, c)
            g = RK[0, j, k]
            U[0, j, k] = kxx * dv - kzz * g
            U[2, j, k] = kxx * g + kzz * dv
            U[6, j, k] = RK[2, j, k]
    return U


def set_initial_data_vg(U, RK, ops: Operators, p: Params):
    """initial_step.f90:301-353 (restart option 3): u, w (and phi into RK[1]) from v = U[1] and
    g = RK[0]; theta from RK[2]; the (0, 0) mode takes U, W, theta from the stores.  Returns
    (U, RK), both new arrays."""
    kxi, kzi = wavenumbers(p.nx, p.nz)
    U, RK = U.copy(), RK.copy()
    lmfxr, lmfzr = 1.0 / p.lmfx, 1.0 / p.lmfz
    for j, kzv in enumerate(kzi):
        for k, kxv in enumerate(kxi):
            if kxv == 0 and kzv == 0:
                U[0, j, k], U[1, j, k], U[2, j, k], U[6, j, k] = RK[0, j, k], 0.0, RK[1, j, k], RK[2, j, k]
                continue
            c = labs.bs(ops.D0_lu, U[1, j, k])
            dv = labs.mat_mul(ops.D1, c)
            k2 = (kxv * lmfxr) ** 2 + (kzv * lmfzr) ** 2
            RK[1, j, k] = labs.mat_mul(ops.D2, c) - k2 * U[1, j, k]
            kxx, kzz = 1j * kxv * lmfxr / k2, 1j * kzv * lmfzr / k2
            g = RK[0, j, k]
            U[0, j, k] = kxx * dv - kzz * g
            U[2, j, k] = kxx * g + kzz * dv
            U[6, j, k] = RK[2, j, k]
    return U, RK


# ----------------------------------------------------------------------------
# pressure (row 19): get_pressure / cal_pressure / solve_ppe, get_pressure.f90:1-137
# ----------------------------------------------------------------------------
def get_uv(a, b):
    """get_uv, get_statistics.f90:982-1017: <ab>(y) = sum over the stored modes of
    Re a Re b + Im a Im b, with weight 1 on the kx = 0 plane and 2 elsewhere.
    a, b are (nz, nxh, ny)."""
    w = np.full(a.shape[1], 2.0)
    w[0] = 1.0
    return np.einsum("zxy,x->y", a.real * b.real + a.imag * b.imag, w)


def solve_ppe(u1, u2, u3, u4, u5, u6, ops: Operators, kx, kz, bc1=0.0, bc2=0.0):
    """solve_ppe, get_pressure.f90:57-137, on lines (ny, M): the pressure Poisson equation
    (D2 - k^2 D0) c = rhs with Neumann rows (D1) at the walls, p = D0 c.

    u1..u6 are the spectral products u u - v v, u v, w w - v v, v w, u w, v v.  As in the
    reference, rows 1 and ny of the second D0 solve keep D0^{-1}(v v) (u6 is overwritten only
    on rows 2..ny-1 before the solve)."""
    bs, mm = labs.bs, labs.mat_mul
    k2 = kx * kx + kz * kz
    kxkz = kx * kz
    buf1 = np.zeros_like(u1)
    buf1[1:-1] = kx * kx * u1[1:-1] + kz * kz * u3[1:-1] + k2 * u6[1:-1] + 2.0 * kxkz * u5[1:-1]
    c6 = bs(ops.D0_lu, u6)
    buf2 = mm(ops.D2, c6)
    buf1[1:-1] = buf1[1:-1] - buf2[1:-1]
    u6b = np.array(c6)
    u6b[1:-1] = (1j * kx) * u2[1:-1] + (1j * kz) * u4[1:-1]
    c6b = bs(ops.D0_lu, u6b)
    buf2 = mm(ops.D1, c6b)
    buf1[0] = bc1
    buf1[1:-1] = buf1[1:-1] - 2.0 * buf2[1:-1]
    buf1[-1] = bc2
    A = np.array((-k2)[None, None] * ops.D0[..., None] + ops.D2[..., None])
    A[:, 0] = ops.D1[:, 0][:, None]
    A[:, -1] = ops.D1[:, -1][:, None]
    D_buf = labs.lu(A)
    c = bs(D_buf, buf1)
    return mm(ops.D0, c)


def ppe_boundary(v, ops: Operators, p: Params):
    """get_y_dir_deriv_of_field_with_PPE_BC, get_statistics.f90:689-719 (called from
    get_statistics_1 before get_pressure): with c = D0^{-1} v per mode,
    BC1 = nu (D2 c) on row 1 from columns 1..3 and BC2 = nu (D2 c) on row ny from columns
    ny-2..ny (the band entries LABS_D2_B(bw+1..bw+3, 1) and LABS_D2_B(bw-1..bw+1, ny)).
    v is (nz, nxh, ny); returns (bc1, bc2), each (nz, nxh) complex."""
    c = labs.bs(ops.D0_lu, np.ascontiguousarray(v.reshape(-1, v.shape[-1]).T))
    bw = ops.bw
    D2 = ops.D2
    bc1 = p.nu * (D2[bw, 0] * c[0] + D2[bw + 1, 0] * c[1] + D2[bw + 2, 0] * c[2])
    bc2 = p.nu * (D2[bw - 2, -1] * c[-3] + D2[bw - 1, -1] * c[-2] + D2[bw, -1] * c[-1])
    return bc1.reshape(v.shape[:2]), bc2.reshape(v.shape[:2])


def get_pressure(P, vv, ops: Operators, p: Params, bc=None):
    """cal_pressure, get_pressure.f90:17-54: solve_ppe on every mode of the products
    P (6, nz, nxh, ny) = f1..f6 with the wall values bc = (bc1, bc2) (stat_PPE_boundary,
    (nz, nxh) each; zero when None); the (0,0) mode gets -<vv>.  Returns p (nz, nxh, ny)."""
    kxi, kzi = wavenumbers(p.nx, p.nz)
    KZ, KX = np.meshgrid(kzi, kxi, indexing="ij")
    mask = ~((KX == 0) & (KZ == 0))
    kx = KX[mask] * (1.0 / p.lmfx)
    kz = KZ[mask] * (1.0 / p.lmfz)
    lines = [np.ascontiguousarray(P[i][mask].T) for i in range(6)]
    bc1, bc2 = (0.0, 0.0) if bc is None else (bc[0][mask], bc[1][mask])
    out = np.zeros((p.nz, p.nxh, p.ny), dtype=np.complex128)
    out[mask] = solve_ppe(*lines, ops, kx, kz, bc1, bc2).T
    out[0, 0] = -vv
    return out


def pressure(U, ops: Operators, p: Params):
    """The pressure of the state U (10, nz, nxh, ny) as a statistics step computes it
    (time_march.f90:47-110): <vv> and the wall values nu d2v/dy2 (ppe_boundary) from the state
    (get_statistics_1), the substep-1 products with f6 = v v through y_to_x, dft_x_realspace
    and x_to_y, rescale_data, get_pressure."""
    vv = get_uv(U[1], U[1])
    bc = ppe_boundary(U[1], ops, p)
    Up = np.zeros((10, p.ny, p.nz32, p.nxh), dtype=np.complex128)
    for f in (0, 1, 2, 6):
        Up[f] = y_to_x(U[f], p.nz32)
    dft_x_realspace(Up, p.nx, 2, p.dxr, p.dzr, np.zeros(p.ny), stat=True)
    P = np.stack([x_to_y(Up[f], p.nz) for f in range(6)]) * p.rescale
    return get_pressure(P, vv, ops, p, bc)
