"""The statistics oracle (oracle/stats.py) against checks that do not go through it (CPU only):
dense restatements, Parseval's relation between the spectral sums and physical-space plane
averages, a laminar state with known answers, and the C-ABI's dataset-name tables."""
import numpy as np
import pytest

from channel_passive_b200 import _lib, ic
from oracle import kmm, labs, stats

P16 = dict(nx=16, ny=33, nz=16, lmfx=1.0, lmfz=0.5, stretch=0.9)


@pytest.fixture(scope="module")
def case():
    """A seeded state without kz-Nyquist content: the z transform drops that row
    (ppdfftw_dft_z_inverse pads around it) while the spectral sums keep it, so physical-space
    checks need it empty (a state after one step has it empty too)."""
    p = kmm.Params(**P16)
    ops = kmm.make_operators(p)
    U = ic.seeded_ic(p.nx, p.ny, p.nz, ops.y, p.lmfx, p.lmfz)
    U[:, p.nz // 2] = 0.0
    return p, ops, U, stats.statistics(U, ops, p)


def _physical(U, p, f):
    """u(x, z) on the 3/2 grid of each y: backward z transform (padded), c2r in x."""
    Up = kmm.y_to_x(U[f], p.nz32)
    buf = np.zeros(Up.shape[:-1] + (p.nx32 // 2 + 1,), dtype=np.complex128)
    buf[..., : p.nxh] = Up
    return np.fft.irfft(buf, n=p.nx32, axis=-1) * p.nx32   # [y, z32, x32]


def test_ppe_wall_values_are_nu_d2v_at_the_walls():
    """get_y_dir_deriv_of_field_with_PPE_BC keeps three columns of the D2 wall rows; at the
    clamped boundary knot the other basis functions have zero second derivative, so the wall
    values equal nu (D2 D0^{-1} v) on rows 1 and ny of the dense operators."""
    p = kmm.Params(**P16)
    ops = kmm.make_operators(p)
    U = ic.seeded_ic(p.nx, p.ny, p.nz, ops.y, p.lmfx, p.lmfz)
    bc1, bc2 = kmm.ppe_boundary(U[1], ops, p)
    D0, D2 = labs.band_to_full(ops.D0), labs.band_to_full(ops.D2)
    assert np.all(D2[0, 3:] == 0.0) or np.abs(D2[0, 3:]).max() < 1e-12 * np.abs(D2[0]).max()
    c = np.linalg.solve(D0, U[1].reshape(-1, p.ny).T)
    d2 = D2 @ c
    scale = p.nu * np.abs(d2[[0, -1]]).max()
    assert np.abs(bc1.ravel() - p.nu * d2[0]).max() <= 1e-10 * scale
    assert np.abs(bc2.ravel() - p.nu * d2[-1]).max() <= 1e-10 * scale


def test_pressure_ppe_with_wall_values_matches_dense():
    """solve_ppe with nonzero wall values: rows 1 and ny of the right-hand side are BC1, BC2."""
    p = kmm.Params(**P16)
    ops = kmm.make_operators(p)
    rng = np.random.default_rng(11)
    M = 4
    lines = [rng.standard_normal((p.ny, M)) + 1j * rng.standard_normal((p.ny, M)) for _ in range(6)]
    kx = np.array([1.0, 2.0, 0.5, 3.0])
    kz = np.array([0.0, -2.0, 4.5, -1.5])
    bc1 = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    bc2 = rng.standard_normal(M) + 1j * rng.standard_normal(M)
    P = kmm.solve_ppe(*lines, ops, kx, kz, bc1, bc2)
    D0, D1, D2 = (labs.band_to_full(ops.D0), labs.band_to_full(ops.D1), labs.band_to_full(ops.D2))
    u1, u2, u3, u4, u5, u6 = lines
    for i in range(M):
        k2 = kx[i] ** 2 + kz[i] ** 2
        c6 = np.linalg.solve(D0, u6[:, i])
        rhs = kx[i] ** 2 * u1[:, i] + kz[i] ** 2 * u3[:, i] + k2 * u6[:, i] + 2 * kx[i] * kz[i] * u5[:, i] - D2 @ c6
        g = c6.copy()
        g[1:-1] = 1j * kx[i] * u2[1:-1, i] + 1j * kz[i] * u4[1:-1, i]
        rhs = rhs - 2 * (D1 @ np.linalg.solve(D0, g))
        rhs[0], rhs[-1] = bc1[i], bc2[i]
        A = D2 - k2 * D0
        A[0], A[-1] = D1[0], D1[-1]
        ref = D0 @ np.linalg.solve(A, rhs)
        assert np.abs(P[:, i] - ref).max() <= 1e-10 * max(1.0, np.abs(ref).max())


def test_spectra_sum_to_the_lines(case):
    """Summing a kx spectrum over kx, or a kz spectrum over kz, gives the <ab> line of the same
    pair (get_uv sums the same weighted products); "Eozoz_kz" sums to the ox-oz line."""
    p, ops, U, s = case
    L = s["lines"]
    pair_line = {"uu": "uu", "vv": "vv", "ww": "ww", "tt": "tt", "uv": "uv", "vw": "vw", "uw": "uw",
                 "ut": "ut", "vt": "vt", "wt": "wt", "oxox": "omega_x_omega_x",
                 "oyoy": "omega_y_omega_y", "ozoz": "omega_z_omega_z", "oxoy": "omega_x_omega_y",
                 "oxoz": "omega_x_omega_z", "oyoz": "omega_y_omega_z", "voz": "v_omega_z",
                 "woy": "w_omega_y"}
    for q, name in enumerate(stats.SPEC_NAMES):
        line = L[stats.LINE[pair_line[name]]]
        tol = 1e-12 * max(1.0, np.abs(line).max())
        assert np.abs(s["spec_kx"][q].sum(axis=0) - line).max() <= tol, name
        zname = "omega_x_omega_z" if name == "ozoz" else pair_line[name]
        zline = L[stats.LINE[zname]]
        assert np.abs(s["spec_kz"][q].sum(axis=0) - zline).max() <= 1e-12 * max(1.0, np.abs(zline).max()), name
    assert np.array_equal(L[stats.LINE["P"]], -L[stats.LINE["vv"]])


def test_lines_match_physical_plane_averages(case):
    """Parseval on the dealiased grid: <ab>(y) = the plane average of a b in physical space, and
    the moment lines are plane averages of powers (rows 1 and ny zero)."""
    p, ops, U, s = case
    L = s["lines"]
    u, v, w, t = (_physical(U, p, f) for f in (0, 1, 2, 6))
    avg = lambda a: a.mean(axis=(1, 2))  # noqa: E731
    for name, prod in (("uu", u * u), ("vv", v * v), ("ww", w * w), ("tt", t * t), ("uv", u * v),
                       ("uw", u * w), ("vw", v * w), ("ut", u * t), ("vt", v * t), ("wt", w * t)):
        ref = avg(prod)
        assert np.abs(L[stats.LINE[name]] - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), name
    for name, prod in (("uuu", u ** 3), ("wwww", w ** 4), ("v6", v ** 6), ("u10", u ** 10)):
        ref = avg(prod)
        ref[0] = ref[-1] = 0.0
        assert np.abs(L[stats.LINE[name]] - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()), name


def test_pressure_lines_and_strain(case):
    """<up>, <pp> and the pressure-strain lines from the oracle's pressure field by plain sums;
    -d<up>/dy from a dense D1 D0^{-1}."""
    p, ops, U, s = case
    L, P = s["lines"], s["P"]
    assert np.allclose(L[stats.LINE["up"]], kmm.get_uv(U[0], P), rtol=1e-13, atol=1e-16)
    assert np.allclose(L[stats.LINE["pp"]], kmm.get_uv(P, P), rtol=1e-13, atol=1e-16)
    D0, D1 = labs.band_to_full(ops.D0), labs.band_to_full(ops.D1)
    ref = -(D1 @ np.linalg.solve(D0, L[stats.LINE["up"]]))
    assert np.abs(L[stats.LINE["-dpudy"]] - ref).max() <= 1e-10 * max(1e-12, np.abs(ref).max())
    # 2 <p du/dx> in physical space equals the spectral sum (Parseval)
    up = kmm.y_to_x(U[0], p.nz32)
    kx = np.arange(p.nxh) / p.lmfx
    dudx = 1j * kx[None, None, :] * up
    buf = np.zeros(up.shape[:-1] + (p.nx32 // 2 + 1,), dtype=np.complex128)
    buf[..., : p.nxh] = dudx
    dudx_phys = np.fft.irfft(buf, n=p.nx32, axis=-1) * p.nx32
    pp = kmm.y_to_x(P, p.nz32)
    buf[..., : p.nxh] = pp
    p_phys = np.fft.irfft(buf, n=p.nx32, axis=-1) * p.nx32
    ref = 2.0 * (p_phys * dudx_phys).mean(axis=(1, 2))
    got = L[stats.LINE["2pdudx"]]
    assert np.abs(got - ref).max() <= 1e-10 * max(1e-12, np.abs(ref).max())


def test_laminar_statistics_known_answers():
    """U = 1.5 (1 - y^2), v = w = 0, theta = U: <uu> = U^2, dU/dy = -3y, U_c = 1.5, the
    dissipation of uu is 2 nu (dU/dy)^2, <oz oz> = (dU/dy)^2, <uuu> = U^3 inside, and every
    v- or pressure-carrying line vanishes."""
    p = kmm.Params(nx=8, ny=33, nz=8)
    ops = kmm.make_operators(p)
    U = np.zeros((10, p.nz, p.nxh, p.ny), dtype=np.complex128)
    Ub = 1.5 * (1 - ops.y ** 2)
    U[0, 0, 0] = Ub
    U[6, 0, 0] = Ub
    s = stats.statistics(U, ops, p)
    L = s["lines"]
    y = ops.y
    assert np.allclose(L[stats.LINE["U"]], Ub, atol=1e-14)
    assert np.allclose(L[stats.LINE["uu"]], Ub ** 2, atol=1e-13)
    assert np.allclose(L[stats.LINE["dUdy"]], -3 * y, atol=1e-10)
    assert np.allclose(L[stats.LINE["dTdy"]], -3 * y, atol=1e-10)
    assert abs(s["u_center"] - 1.5) < 1e-10 and abs(s["t_center"] - 1.5) < 1e-10
    assert np.allclose(L[stats.LINE["2nududxidudxi"]], 2 * p.nu * 9 * y ** 2, atol=1e-12)
    assert np.allclose(L[stats.LINE["omega_z_omega_z"]], 9 * y ** 2, atol=1e-9)
    inner = np.zeros_like(Ub)
    inner[1:-1] = Ub[1:-1] ** 3
    assert np.allclose(L[stats.LINE["uuu"]], inner, atol=1e-12)
    for name in ("vv", "uv", "-duuvdy", "-dvvvdy", "up", "pp", "2pdudx", "2pdvdy", "pdudy+pdvdx"):
        assert np.abs(L[stats.LINE[name]]).max() < 1e-12, name
    assert np.abs(s["P"]).max() < 1e-12


def test_abi_dataset_names_match_oracle():
    lib = _lib.load()
    assert _lib.KMM_STAT_NLINES == len(stats.LINE_NAMES)
    assert _lib.KMM_STAT_NSPEC == len(stats.SPEC_NAMES)
    for i, n in enumerate(stats.LINE_NAMES):
        assert lib.kmm_stat_line_name(i).decode() == n
    for i, n in enumerate(stats.SPEC_NAMES):
        assert lib.kmm_stat_spec_name(i).decode() == n
    assert lib.kmm_stat_line_name(len(stats.LINE_NAMES)) is None
    assert lib.kmm_stat_spec_name(-1) is None
    assert lib.kmm_get_statistics(None, None, None, None, None, None) == _lib.KMM_ERR_ARG
