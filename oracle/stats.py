"""FP64 CPU restatement of a statistics step (oracle; test infrastructure only).

A statistics step (time_march.f90:47-110) evaluates, on the state at the start of RK substep 1:
  get_statistics_1 (get_statistics.f90:9-368)      mean lines, <ab> lines, dissipation and
                                                  vorticity lines, the PPE wall values
                                                  (kmm.ppe_boundary);
  write_spectra (write_energy_spectra.f90:9-399)  1-D (co)spectra in kx and in kz;
  dft_x_realspace on the statistics substep        physical-space moment sums
                                                  (dft_x_realspace.f90:41-57, 128-155, 238-484);
  get_statistics_2 (get_statistics.f90:376-539)   moments, transport lines, the pressure and its
                                                  covariance and pressure-strain lines.
statistics() returns every line in the order of LINE_NAMES (the dataset names of the reference's
stat file), the spectra in the order of SPEC_NAMES, the centre-line values and the pressure.

Layouts (numpy C-order): state U[f, kz, kx, y]; lines [q, y]; spec_kx [q, kx, y] and
spec_kz [q, kz, y] = the reference's io_plane arrays STAT(ny, nxh) / STAT(ny, nz).
"""
from __future__ import annotations

import numpy as np

from . import kmm, labs

LINE_NAMES = (
    "U", "W", "Theta", "dUdy", "dWdy", "dTdy",
    "uu", "vv", "P", "ww", "tt", "uv", "uw", "vw", "ut", "wt", "vt",
    "2nududxidudxi", "2nudvdxidvdxi", "2nudwdxidwdxi", "2nududxidvdxi",
    "omega_x_omega_x", "omega_y_omega_y", "omega_z_omega_z", "omega_x_omega_y",
    "omega_y_omega_z", "omega_x_omega_z", "v_omega_z", "w_omega_y",
    "uuu", "vvv", "www", "uuuu", "vvvv", "wwww",
    "u6", "v6", "w6", "u8", "v8", "w8", "u10", "v10", "w10",
    "-duuvdy", "-dvvvdy", "-dvwwdy", "-duvvdy",
    "up", "-dpudy", "vp", "-2dpvdy", "wp", "pp",
    "2pdudx", "2pdvdy", "2pdwdz", "pdudy+pdvdx",
)
SPEC_NAMES = ("uu", "vv", "ww", "tt", "uv", "vw", "uw", "ut", "vt", "wt",
              "oxox", "oyoy", "ozoz", "oxoy", "oxoz", "oyoz", "voz", "woy")
LINE = {n: i for i, n in enumerate(LINE_NAMES)}
SPEC = {n: i for i, n in enumerate(SPEC_NAMES)}


def _lines(a):
    """(nz, nxh, ny) -> (ny, nz*nxh) mode columns for the band routines."""
    return a.reshape(-1, a.shape[-1]).T


def _unlines(b, shape):
    return np.ascontiguousarray(b.T).reshape(shape)


def y_deriv(a, ops: kmm.Operators):
    """get_y_dir_deriv_of_field, get_statistics.f90:658-681: D1 D0^{-1} a per mode."""
    c = labs.bs(ops.D0_lu, _lines(a))
    return _unlines(labs.mat_mul(ops.D1, c), a.shape)


def _wave(p: kmm.Params):
    """kx_wave = LMFxr kx, kz_wave = LMFzr kz (get_statistics.f90:777-782), (nz, nxh, 1)."""
    kxi, kzi = kmm.wavenumbers(p.nx, p.nz)
    kx = (kxi * (1.0 / p.lmfx))[None, :, None]
    kz = (kzi * (1.0 / p.lmfz))[:, None, None]
    return kx, kz


def _weight(nxh):
    """get_uv's weight: 1 on the kx = 0 plane, 2 elsewhere (get_statistics.f90:998-1012)."""
    w = np.full(nxh, 2.0)
    w[0] = 1.0
    return w[None, :, None]


def _re(a, b):
    return a.real * b.real + a.imag * b.imag


def vorticity(u, v, w, dudy, dwdy, p: kmm.Params):
    """get_vorticity_field, get_statistics.f90:912-948: omega_x = dw/dy - i kz v,
    omega_y = i kz u - i kx w, omega_z = i kx v - du/dy."""
    kx, kz = _wave(p)
    ox = dwdy - 1j * kz * v
    oy = 1j * kz * u - 1j * kx * w
    oz = 1j * kx * v - dudy
    return ox, oy, oz


def spectrum_x(a, b):
    """get_E_uu_x, write_energy_spectra.f90:326-359: E(kx, y) = sum over kz of w Re(a b*)."""
    return np.sum(_weight(a.shape[1]) * _re(a, b), axis=0)


def spectrum_z(a, b):
    """get_E_uu_z, write_energy_spectra.f90:366-399: E(kz, y) = sum over kx of w Re(a b*)."""
    return np.sum(_weight(a.shape[1]) * _re(a, b), axis=1)


def dissipation(a1, a2, d1, d2, p: kmm.Params):
    """get_turb_transport_e_ij, get_statistics.f90:761-810: 2 nu w (kx^2 Re(a1 a2*)
    + Re(d1 d2*) + kz^2 Re(a1 a2*)) summed over the modes."""
    kx, kz = _wave(p)
    t = kx * kx * _re(a1, a2) + _re(d1, d2) + kz * kz * _re(a1, a2)
    return np.sum(2.0 * p.nu * _weight(a1.shape[1]) * t, axis=(0, 1))


def pressure_strain(P, u, v, w, dudy, dvdy, p: kmm.Params):
    """get_turb_transport_PI1_ij, get_statistics.f90:817-902: (2<p du/dx>, 2<p dv/dy>,
    2<p dw/dz>, <p du/dy> + <p dv/dx>) with get_uv's weights."""
    kx, kz = _wave(p)
    wt = _weight(u.shape[1])

    def cross(a):  # Re a Im p - Im a Re p
        return a.real * P.imag - a.imag * P.real

    pi_uu = np.sum(wt * 2.0 * kx * cross(u), axis=(0, 1))
    pi_ww = np.sum(wt * 2.0 * kz * cross(w), axis=(0, 1))
    pi_vv = np.sum(wt * 2.0 * _re(dvdy, P), axis=(0, 1))
    pi_uv = np.sum(wt * kx * cross(v), axis=(0, 1)) + np.sum(wt * _re(dudy, P), axis=(0, 1))
    return pi_uu, pi_vv, pi_ww, pi_uv


def _d1_d0inv_real(line, ops: kmm.Operators):
    """labs_bs(D0_LU) then labs_mat_mul(D1) of a real line, real part kept."""
    c = labs.bs(ops.D0_lu, np.asarray(line, dtype=np.complex128))
    return labs.mat_mul(ops.D1, c).real


def physical_moments(U, p: kmm.Params):
    """dft_x_realspace.f90:128-155 on a statistics substep: per y, the sums over the physical
    plane of u^3, v^3, w^3, u^4, v^4, w^4, u^6, v^6, w^6, u^8, v^8, w^8, u^10, v^10, w^10,
    -u u v, -v w w, -u v v (raw velocities: the mean subtraction is commented out there).
    Returns (18, ny)."""
    nxh = p.nxh
    nfreq = p.nx32 // 2 + 1
    phys = []
    for f in (0, 1, 2):
        Up = kmm.y_to_x(U[f], p.nz32)                       # [y, z32, kx]
        buf = np.zeros(Up.shape[:-1] + (nfreq,), dtype=np.complex128)
        buf[..., :nxh] = Up
        phys.append(np.fft.irfft(buf, n=p.nx32, axis=-1) * p.nx32)
    u, v, w = phys
    sums = []
    for k in (3, 4, 6, 8, 10):
        for a in (u, v, w):
            sums.append(np.sum(a ** k, axis=(1, 2)))
    sums.append(np.sum(-(u * u * v), axis=(1, 2)))
    sums.append(np.sum(-(v * w * w), axis=(1, 2)))
    sums.append(np.sum(-(u * v * v), axis=(1, 2)))
    return np.array(sums)


def statistics(U, ops: kmm.Operators, p: kmm.Params):
    """Every line and spectrum of a statistics step of the state U (10, nz, nxh, ny).

    Returns a dict: lines (58, ny), spec_kx (18, nxh, ny), spec_kz (18, nz, ny),
    u_center, t_center and P (nz, nxh, ny), the pressure (kmm.pressure)."""
    ny = p.ny
    u, v, w, t = U[0], U[1], U[2], U[6]
    L = np.zeros((len(LINE_NAMES), ny))
    # get_statistics_1: mean lines (get_u, get_dudy_u_center, get_dwdy, get_dtdy_t_center)
    L[LINE["U"]] = u[0, 0].real + p.u_gal
    L[LINE["W"]] = w[0, 0].real
    L[LINE["Theta"]] = t[0, 0].real
    cu = labs.bs(ops.D0_lu, u[0, 0].copy())
    u_center = p.u_gal
    for k in range(ny):
        u_center = u_center + cu[k].real * ops.center[k]
    L[LINE["dUdy"]] = labs.mat_mul(ops.D1, cu).real
    L[LINE["dWdy"]] = labs.mat_mul(ops.D1, labs.bs(ops.D0_lu, w[0, 0].copy())).real
    ct = labs.bs(ops.D0_lu, t[0, 0].copy())
    t_center = 0.0
    for k in range(ny):
        t_center = t_center + ct[k].real * ops.center[k]
    L[LINE["dTdy"]] = labs.mat_mul(ops.D1, ct).real
    # derivatives, the PPE wall values, vorticity
    dudy, dvdy, dwdy = y_deriv(u, ops), y_deriv(v, ops), y_deriv(w, ops)
    ox, oy, oz = vorticity(u, v, w, dudy, dwdy, p)
    # spectra (write_spectra): the kz list repeats (ox, oz) for "Eozoz_kz" as the reference's
    # call does (write_energy_spectra.f90:218-219)
    pairs_x = [(u, u), (v, v), (w, w), (t, t), (u, v), (v, w), (u, w), (u, t), (v, t), (t, w),
               (ox, ox), (oy, oy), (oz, oz), (ox, oy), (ox, oz), (oy, oz), (v, oz), (w, oy)]
    pairs_z = list(pairs_x)
    pairs_z[SPEC["ozoz"]] = (ox, oz)
    spec_kx = np.array([spectrum_x(a, b) for a, b in pairs_x])
    spec_kz = np.array([spectrum_z(a, b) for a, b in pairs_z])
    # <ab> lines (get_uv) in the reference's order
    for name, (a, b) in (("uu", (u, u)), ("vv", (v, v)), ("ww", (w, w)), ("tt", (t, t)),
                         ("uv", (u, v)), ("uw", (u, w)), ("vw", (v, w)), ("ut", (u, t)),
                         ("wt", (t, w)), ("vt", (v, t)),
                         ("omega_x_omega_x", (ox, ox)), ("omega_y_omega_y", (oy, oy)),
                         ("omega_z_omega_z", (oz, oz)), ("omega_x_omega_y", (ox, oy)),
                         ("omega_y_omega_z", (oy, oz)), ("omega_x_omega_z", (ox, oz)),
                         ("v_omega_z", (v, oz)), ("w_omega_y", (w, oy))):
        L[LINE[name]] = kmm.get_uv(a, b)
    L[LINE["P"]] = -L[LINE["vv"]]
    L[LINE["2nududxidudxi"]] = dissipation(u, u, dudy, dudy, p)
    L[LINE["2nudvdxidvdxi"]] = dissipation(v, v, dvdy, dvdy, p)
    L[LINE["2nudwdxidwdxi"]] = dissipation(w, w, dwdy, dwdy, p)
    L[LINE["2nududxidvdxi"]] = dissipation(u, v, dudy, dvdy, p)
    # physical moments (dft_x_realspace on the statistics substep), get_statistics_2
    S = physical_moments(U, p) * p.rescale
    for i, name in enumerate(("uuu", "vvv", "www", "uuuu", "vvvv", "wwww", "u6", "v6", "w6",
                              "u8", "v8", "w8", "u10", "v10", "w10")):
        L[LINE[name]][1:-1] = S[i][1:-1]       # rows 1 and ny are set to 0
    L[LINE["-duuvdy"]] = _d1_d0inv_real(S[15], ops)
    L[LINE["-dvvvdy"]] = _d1_d0inv_real(-S[1], ops)
    L[LINE["-dvwwdy"]] = _d1_d0inv_real(S[16], ops)
    L[LINE["-duvvdy"]] = _d1_d0inv_real(S[17], ops)
    # pressure and its statistics
    P = kmm.pressure(U, ops, p)
    L[LINE["up"]] = kmm.get_uv(u, P)
    L[LINE["-dpudy"]] = -_d1_d0inv_real(L[LINE["up"]], ops)
    L[LINE["vp"]] = kmm.get_uv(v, P)
    L[LINE["-2dpvdy"]] = -2.0 * _d1_d0inv_real(L[LINE["vp"]], ops)
    L[LINE["wp"]] = kmm.get_uv(w, P)
    L[LINE["pp"]] = kmm.get_uv(P, P)
    pi_uu, pi_vv, pi_ww, pi_uv = pressure_strain(P, u, v, w, dudy, dvdy, p)
    L[LINE["2pdudx"]] = pi_uu
    L[LINE["2pdvdy"]] = pi_vv
    L[LINE["2pdwdz"]] = pi_ww
    L[LINE["pdudy+pdvdx"]] = pi_uv
    return {"lines": L, "spec_kx": spec_kx, "spec_kz": spec_kz, "u_center": float(u_center),
            "t_center": float(t_center), "P": P}
