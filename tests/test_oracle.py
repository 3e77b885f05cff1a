"""The oracle pinned against the reference's known answers (CPU only)."""
import os

import numpy as np
import pytest

from oracle import bspline, kmm, labs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("stretch", [0.0, 0.99])
def test_bspline_reference_known_answer(stretch):
    """tests/test_bspline.cpp:4-26: k=7, n=32; finite entries, sum of integration weights 2
    within 1e-12, D0 rows sum to 1 and D1..D4 rows to 0 within 1e-11 * (1 + sum |row|)."""
    o = bspline.fill_full(7, 32, stretch)
    assert np.all(np.isfinite(o["integ"]))
    assert abs(o["integ"].sum() - 2.0) <= 1e-12
    for d in range(5):
        M = o["D"][d]
        assert np.all(np.isfinite(M))
        val = M.sum(axis=1)
        scale = 1.0 + np.abs(M).sum(axis=1)
        assert np.all(np.abs(val - (1.0 if d == 0 else 0.0)) <= 1e-11 * scale)


@pytest.mark.parametrize("n,stretch", [(33, 0.0), (65, 0.9), (129, 0.9)])
def test_bspline_polynomial_exactness(n, stretch):
    """Order-7 B-splines reproduce polynomials of degree <= 6: D1, D2 are exact on y^5."""
    o = bspline.fill_full(7, n, stretch)
    y = o["y"]
    c = np.linalg.solve(o["D"][0], y ** 5)
    assert np.abs(o["D"][1] @ c - 5 * y ** 4).max() < 1e-9
    assert np.abs(o["D"][2] @ c - 20 * y ** 3).max() < 1e-6 * np.abs(o["D"][2]).max()
    # integration weights integrate the basis exactly: int_{-1}^{1} y^4 = 2/5
    c4 = np.linalg.solve(o["D"][0], y ** 4)
    assert abs(o["integ"] @ c4 - 0.4) < 1e-13


def test_bspline_golden_fixture():
    g = np.load(os.path.join(GOLDEN, "bspline_k7_n32.npz"))
    for tag, st in (("s0", 0.0), ("s099", 0.99)):
        o = bspline.fill_full(7, 32, st)
        for d in range(5):
            np.testing.assert_array_equal(o["D"][d], g[f"{tag}_D{d}"])
        np.testing.assert_array_equal(o["y"], g[f"{tag}_y"])
        np.testing.assert_allclose(o["integ"], g[f"{tag}_integ"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("n", [33, 65, 129])
def test_labs_packed_band_matches_dense(n):
    o = bspline.fill_full(7, n, 0.9)
    D = o["D"]
    bw = labs.eval_bw(D[0], D[1], D[2])
    bands = [labs.full_to_band(D[d], bw) for d in range(3)]
    for d in range(3):
        np.testing.assert_array_equal(labs.band_to_full(bands[d]), D[d])
    rng = np.random.default_rng(n)
    r = rng.standard_normal((n, 4)) + 1j * rng.standard_normal((n, 4))
    for d in range(3):
        np.testing.assert_allclose(labs.mat_mul(bands[d], r), D[d] @ r, rtol=0, atol=1e-12 * np.abs(D[d]).max() * 10)
    # Helmholtz matrix with Dirichlet rows, per mode
    a, b = 1.0 + rng.random(4), 0.01 * rng.random(4)
    A = a[None, None] * bands[0][..., None] - b[None, None] * bands[2][..., None]
    for col in (0, -1):
        A[:, col] = 0.0
        A[bw, col] = a * bands[0][bw, col] - b * bands[2][bw, col]
    x = labs.bs(labs.lu(A), r)
    for m in range(4):
        ref = np.linalg.solve(labs.band_to_full(A[..., m]), r[:, m])
        assert np.abs(x[:, m] - ref).max() <= 1e-13 * np.abs(ref).max()


def test_wavenumbers_bitexact():
    kx, kz = kmm.wavenumbers(192, 192)
    assert kx.tolist() == list(range(96))
    assert kz.tolist() == list(range(97)) + list(range(-95, 0))


def test_dealias_masks():
    """y_to_x zeroes kz = nz/2 and pads; x_to_y keeps 0..nh-1, zeroes nh (module_ppdfftw.f90:794-861)."""
    nz, nxh, ny = 8, 4, 3
    rng = np.random.default_rng(0)
    u = rng.standard_normal((nz, nxh, ny)) + 1j * rng.standard_normal((nz, nxh, ny))
    xp = kmm.y_to_x(u, 12)
    back = kmm.x_to_y(xp, nz) / 12.0
    keep = [0, 1, 2, 3, 5, 6, 7]
    np.testing.assert_allclose(back[keep], u[keep], atol=1e-14)
    assert np.all(back[4] == 0)


def _laminar(p, ops):
    U = np.zeros((10, p.nz, p.nxh, p.ny), dtype=np.complex128)
    U[0, 0, 0] = 1.5 * (1 - ops.y ** 2)
    U[6, 0, 0] = U[0, 0, 0]
    return U


def test_laminar_poiseuille_fixed_point():
    p = kmm.Params(nx=8, ny=33, nz=8)
    ops = kmm.make_operators(p)
    U = _laminar(p, ops)
    RK = kmm.set_initial_data_uvw(U, ops, p)
    U0 = U.copy()
    dt, sc = kmm.rk3_step(U, RK, ops, p, 0.01)
    assert np.abs(U - U0).max() < 1e-13
    assert abs(sc.wall_shear_stress - 3 * p.nu) < 1e-13
    assert abs(sc.phi_dpdx[3] - 3 * p.nu) < 1e-13


def test_step_divergence_free_and_hermitian():
    from channel_passive_b200 import ic
    p = kmm.Params(nx=16, ny=33, nz=16, control_amp=-1.0)
    ops = kmm.make_operators(p)
    U = ic.seeded_ic(p.nx, p.ny, p.nz, ops.y, p.lmfx, p.lmfz)
    RK = kmm.set_initial_data_uvw(U, ops, p)
    ctrl = (*kmm.control_weights(ops, p), p.control_amp, None)
    kmm.rk3_step(U, RK, ops, p, 0.01, None, None, ctrl)
    kxi, kzi = kmm.wavenumbers(p.nx, p.nz)
    div = 0.0
    for j, kz in enumerate(kzi):
        for k, kx in enumerate(kxi):
            dv = labs.mat_mul(ops.D1, labs.bs(ops.D0_lu, U[1, j, k]))
            d = 1j * kx / p.lmfx * U[0, j, k] + dv + 1j * kz / p.lmfz * U[2, j, k]
            div = max(div, np.abs(d).max())
    assert div < 1e-13
    for f in (0, 1, 2, 6):
        for j in range(1, p.nz):
            if j == p.nz // 2:
                continue
            assert np.abs(U[f, j, 0] - np.conj(U[f, p.nz - j, 0])).max() < 1e-14


def test_step_golden_fixture():
    """Regression of one full oracle RK3 step (16x33x16, control on) against the fixture."""
    from channel_passive_b200 import ic
    g = np.load(os.path.join(GOLDEN, "step_16x33x16.npz"))
    p = kmm.Params(nx=16, ny=33, nz=16, control_amp=-1.0)
    ops = kmm.make_operators(p)
    U = ic.seeded_ic(p.nx, p.ny, p.nz, ops.y, p.lmfx, p.lmfz)
    np.testing.assert_array_equal(U[[0, 1, 2, 6]], g["U0"])
    RK = kmm.set_initial_data_uvw(U, ops, p)
    ctrl = (*kmm.control_weights(ops, p), p.control_amp, None)
    dt, sc = kmm.rk3_step(U, RK, ops, p, 0.01, None, None, ctrl)
    np.testing.assert_allclose(U[[0, 1, 2, 6]], g["U1"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(RK, g["RK1"], rtol=0, atol=1e-13)
    assert abs(sc.wall_shear_stress - float(g["tau_w"])) < 1e-15


def test_cfl_dt_rule_and_abort():
    p = kmm.Params(nx=8, ny=33, nz=8, fixed_dt=False, cfl=1.0, dt_factor=0.0)
    ops = kmm.make_operators(p)
    U = _laminar(p, ops)
    RK = kmm.set_initial_data_uvw(U, ops, p)
    sc = kmm.Scalars()
    dt = kmm.time_march(U, RK, ops, p, 1, 0.0, sc)
    assert dt == pytest.approx(p.cflx / sc.velmax, rel=1e-15)
    q = kmm.Params(nx=8, ny=33, nz=8, fixed_dt=True)
    with pytest.raises(kmm.DtError):
        kmm.time_march(U, RK, ops, q, 1, 2e5, sc)


def test_pressure_ppe_banded_matches_dense():
    """solve_ppe (get_pressure.f90:57-137): the banded LU solve equals a dense solve of the same
    system -- interior rows (D2 - k^2 D0) c = rhs, Neumann rows D1 c = 0 -- with rhs built as
    the reference builds it, and p = D0 c."""
    from channel_passive_b200 import ic
    p = kmm.Params(nx=16, ny=33, nz=16)
    ops = kmm.make_operators(p)
    U = ic.seeded_ic(p.nx, p.ny, p.nz, ops.y, p.lmfx, p.lmfz)
    rng = np.random.default_rng(7)
    M = 5
    lines = [rng.standard_normal((p.ny, M)) + 1j * rng.standard_normal((p.ny, M)) for _ in range(6)]
    kx = np.array([0.0, 1.0, 2.0, 0.5, 3.0])
    kz = np.array([1.5, 0.0, -2.0, 4.5, -1.5])
    P = kmm.solve_ppe(*lines, ops, kx, kz)
    D0, D1, D2 = (labs.band_to_full(ops.D0), labs.band_to_full(ops.D1), labs.band_to_full(ops.D2))
    u1, u2, u3, u4, u5, u6 = lines
    for i in range(M):
        k2 = kx[i] ** 2 + kz[i] ** 2
        c6 = np.linalg.solve(D0, u6[:, i])
        rhs = kx[i] ** 2 * u1[:, i] + kz[i] ** 2 * u3[:, i] + k2 * u6[:, i] + 2 * kx[i] * kz[i] * u5[:, i] - D2 @ c6
        g = c6.copy()
        g[1:-1] = 1j * kx[i] * u2[1:-1, i] + 1j * kz[i] * u4[1:-1, i]
        rhs = rhs - 2 * (D1 @ np.linalg.solve(D0, g))
        rhs[0] = rhs[-1] = 0.0
        A = D2 - k2 * D0
        A[0], A[-1] = D1[0], D1[-1]
        c = np.linalg.solve(A, rhs)
        assert np.abs(P[:, i] - D0 @ c).max() <= 1e-10 * max(1.0, np.abs(D0 @ c).max())


def test_pressure_mean_mode_and_laminar():
    """cal_pressure: the (0,0) mode is -<vv> (get_uv weights 1 at kx = 0, 2 elsewhere); a laminar
    state (v = w = 0) has zero pressure."""
    from channel_passive_b200 import ic
    p = kmm.Params(nx=16, ny=33, nz=16)
    ops = kmm.make_operators(p)
    U = ic.seeded_ic(p.nx, p.ny, p.nz, ops.y, p.lmfx, p.lmfz)
    P = kmm.pressure(U, ops, p)
    v = U[1]
    vv = (np.abs(v[:, 0]) ** 2).sum(axis=0) + 2 * (np.abs(v[:, 1:]) ** 2).sum(axis=(0, 1))
    assert np.allclose(P[0, 0].real, -vv, rtol=1e-13, atol=0)
    assert np.all(P[0, 0].imag == 0)
    assert np.all(np.isfinite(P))
    L = _laminar(p, ops)
    assert np.abs(kmm.pressure(L, ops, p)).max() < 1e-12
