"""Initial conditions in the reference's Y-pencil layout U[f, kz, kx, y] (complex128).

Two generators:

* ``reference_ic``: the deterministic start of the reference,
  set_initial_value_in_y_pencil (initial_step.f90:63-121): laminar
  1.5(1-y^2) - u_gal in the (0,0) mode, three fixed low modes, theta = u.
* ``seeded_ic``: the synthetic benchmark start: laminar 1.5(1-y^2) plus a
  divergence-free random-phase perturbation in the modes |kx|,|kz| <= kmax
  (integer wavenumbers), built as v = (1-y^2)^2 a_k and omega_y = g = (1-y^2) b_k with
  complex normal a_k, b_k from ``numpy.random.default_rng(seed)``; u and w
  follow from the solve_u_w relation (solve_u_w.f90:27-38) with the exact
  dv/dy; the perturbation is scaled so that the RMS of (u', v', w') over the
  collocation grid is ``amplitude``.  theta_0 = 1.5(1-y^2) (the reference sets
  theta_0 = U_0, initial_step.f90:87).  The kx = 0 plane is Hermitian
  (U(0,-kz) = conj U(0,kz)), so the physical field is real.
"""
from __future__ import annotations

import numpy as np

NFIELD = 10


def _wavenumbers(nx, nz):
    nxh, nzh = nx // 2, nz // 2
    kx = np.arange(nxh)
    kz = np.array([i - 1 if i <= nzh + 1 else i - 2 * nzh - 1 for i in range(1, nz + 1)])
    return kx, kz


def reference_ic(nx, ny, nz, y, u_gal=0.0):
    """set_initial_value_in_y_pencil, initial_step.f90:63-121 (single rank)."""
    nxh = nx // 2
    U = np.zeros((NFIELD, nz, nxh, ny), dtype=np.complex128)
    one_m_y2 = 1.0 - y ** 2
    U[0, 0, 0] = one_m_y2 * 1.5 - u_gal
    U[6, 0, 0] = U[0, 0, 0]
    if nxh > 1:
        q = ((1.0 - y) * (1.0 + y)) ** 2
        U[1, 0, 1] = q * 2e-2 + 1j * q * 1e-2
        U[6, 0, 1] = U[0, 0, 1]
    if nz > 1:
        U[0, 1, 0] = one_m_y2 * 2e-2 + 1j * one_m_y2 * 1e-2
        U[1, 1, 0] = -one_m_y2 * 1e-2 + 1j * one_m_y2 * 1e-2
        U[2, 1, 0] = -one_m_y2 * 1e-2 - 1j * one_m_y2 * 2e-2
        U[6, 1, 0] = U[0, 1, 0]
        U[0, nz - 1, 0] = one_m_y2 * 2e-2 - 1j * one_m_y2 * 1e-2
        U[1, nz - 1, 0] = -one_m_y2 * 1e-2 - 1j * one_m_y2 * 1e-2
        U[2, nz - 1, 0] = -one_m_y2 * 1e-2 + 1j * one_m_y2 * 2e-2
        U[6, nz - 1, 0] = U[0, nz - 1, 0]
    return U


def seeded_ic(nx, ny, nz, y, lmfx, lmfz, seed=20261203, amplitude=0.1, kmax=8, u_gal=0.0):
    """Laminar profile plus a seeded divergence-free random-phase perturbation."""
    nxh = nx // 2
    kxi, kzi = _wavenumbers(nx, nz)
    rng = np.random.default_rng(seed)
    U = np.zeros((NFIELD, nz, nxh, ny), dtype=np.complex128)
    q = 1.0 - y * y
    vshape = q * q                   # (1-y^2)^2
    dvshape = -4.0 * y * q           # d/dy (1-y^2)^2
    gshape = q
    pert = np.zeros((3, nz, nxh, ny), dtype=np.complex128)
    for j, kz in enumerate(kzi):
        for k, kx in enumerate(kxi):
            if (kx == 0 and kz == 0) or abs(kx) > kmax or abs(kz) > kmax:
                continue
            if kx == 0 and kz < 0:
                continue  # filled from the Hermitian partner below
            a = rng.standard_normal() + 1j * rng.standard_normal()
            b = rng.standard_normal() + 1j * rng.standard_normal()
            kxr, kzr = kx / lmfx, kz / lmfz
            k2 = kxr * kxr + kzr * kzr
            v = vshape * a
            f = dvshape * a
            g = gshape * b
            u = 1j * (kxr * f - kzr * g) / k2
            w = 1j * (kzr * f + kxr * g) / k2
            pert[:, j, k] = (u, v, w)
    # Hermitian completion of the kx = 0 plane
    for j, kz in enumerate(kzi):
        if kz < 0 and abs(kz) <= kmax:
            jp = int(np.where(kzi == -kz)[0][0])
            pert[:, j, 0] = np.conj(pert[:, jp, 0])
    # RMS of the physical perturbation over the collocation grid (Parseval:
    # kx > 0 modes count twice for their conjugate partners)
    wgt = np.where(kxi == 0, 1.0, 2.0)[None, None, :, None]
    ms = float((wgt * np.abs(pert) ** 2).sum() / (3 * ny))
    if ms > 0:
        pert *= amplitude / np.sqrt(ms)
    U[0:3] = pert
    U[0, 0, 0] = 1.5 * q - u_gal
    U[6, 0, 0] = 1.5 * q
    return U
