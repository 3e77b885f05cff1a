"""GPU parity of libkmm against the FP64 oracle, through the C ABI (include/kmm.h).

Bars: bit-exact for the layout permutations, wavenumber order and dealias masks; FP64 kernels
within 1e-12 relative L2 of the oracle per operation and 1e-10 after many steps; the mixed
path within 1e-5 relative L2 of the FP64 oracle.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from channel_passive_b200 import Channel, KmmError
from channel_passive_b200 import _lib
from oracle import kmm as okmm, labs as olabs
from tests.helpers import STATE_SLOTS, make_pair, oracle_ctrl, rel_l2, seeded_state

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _setup(nx=16, ny=33, nz=16, **kw):
    cfg, p = make_pair(nx=nx, ny=ny, nz=nz, **kw)
    ops = okmm.make_operators(p)
    return cfg, p, ops


def _cplx(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def test_operators_match_oracle():
    cfg, p, ops = _setup(nx=8, ny=65, nz=8)
    with Channel(cfg) as ch:
        assert ch.bw == ops.bw
        np.testing.assert_array_equal(ch.y, ops.y)
        np.testing.assert_array_equal(ch.D0, ops.D0)
        np.testing.assert_array_equal(ch.D1, ops.D1)
        np.testing.assert_array_equal(ch.D2, ops.D2)
        np.testing.assert_allclose(ch.D0_lu, ops.D0_lu, rtol=0, atol=1e-14 * np.abs(ops.D0_lu).max())


def test_state_roundtrip_bitexact():
    cfg, p, ops = _setup(nx=16, ny=33, nz=24)
    rng = np.random.default_rng(3)
    U = rng.standard_normal((10, cfg.nz, cfg.nxh, cfg.ny)) + 1j * rng.standard_normal((10, cfg.nz, cfg.nxh, cfg.ny))
    RK = rng.standard_normal((3, cfg.nz, cfg.nxh, cfg.ny)) + 1j * rng.standard_normal((3, cfg.nz, cfg.nxh, cfg.ny))
    with Channel(cfg) as ch:
        ch.upload_state(U, RK, 0.01)
        U2, RK2 = ch.download_state()
        for s in STATE_SLOTS:
            assert np.array_equal(U2[s], U[s])
        assert np.array_equal(RK2, RK)
        assert ch.dt == 0.01


@pytest.mark.parametrize("nx,nz,ny", [(16, 16, 33), (8, 24, 21), (64, 64, 65), (20, 40, 21)])
def test_y_to_x_matches_oracle(nx, nz, ny):
    cfg, p, ops = _setup(nx=nx, ny=ny, nz=nz)
    rng = np.random.default_rng(nx + nz)
    u = rng.standard_normal((nz, nx // 2, ny)) + 1j * rng.standard_normal((nz, nx // 2, ny))
    ref = okmm.y_to_x(u, cfg.nz32)
    with Channel(cfg) as ch:
        xp = torch.zeros((ny, cfg.nz32, cfg.nxh), dtype=torch.complex128, device=DEV)
        ch.y_to_x(_cplx(u), xp)
        torch.cuda.synchronize()
        got = xp.cpu().numpy()
    assert rel_l2(got, ref) < 1e-14


@pytest.mark.parametrize("nx,nz,ny", [(16, 16, 33), (8, 24, 21), (64, 64, 65)])
def test_x_to_y_matches_oracle_and_masks(nx, nz, ny):
    cfg, p, ops = _setup(nx=nx, ny=ny, nz=nz)
    rng = np.random.default_rng(7)
    xp = rng.standard_normal((ny, cfg.nz32, cfg.nxh)) + 1j * rng.standard_normal((ny, cfg.nz32, cfg.nxh))
    ref = okmm.x_to_y(xp, nz) * p.rescale
    with Channel(cfg) as ch:
        u = torch.zeros((nz, cfg.nxh, ny), dtype=torch.complex128, device=DEV)
        ch.x_to_y(_cplx(xp), u, rescale=True)
        torch.cuda.synchronize()
        got = u.cpu().numpy()
    assert rel_l2(got, ref) < 1e-14
    # the kz Nyquist row is exactly zero (module_ppdfftw.f90:815)
    assert np.all(got[nz // 2] == 0)


def test_dft_x_realspace_matches_oracle():
    cfg, p, ops = _setup(nx=16, ny=33, nz=16)
    rng = np.random.default_rng(11)
    Up = np.zeros((10, cfg.ny, cfg.nz32, cfg.nxh), dtype=np.complex128)
    for s in STATE_SLOTS:
        Up[s] = rng.standard_normal(Up[s].shape) + 1j * rng.standard_normal(Up[s].shape)
    ref = Up.copy()
    dyr = okmm.dyr_vector(ops.y, p.dy_factor)
    vref = okmm.dft_x_realspace(ref, p.nx, 1, p.dxr, p.dzr, dyr)
    with Channel(cfg) as ch:
        xp = _cplx(Up)
        vm = torch.zeros(1, dtype=torch.float64, device=DEV)
        ch.dft_x_realspace(xp, 1, vm)
        torch.cuda.synchronize()
        got = xp.cpu().numpy()
        velmax = float(vm.item())
    for s in (0, 1, 2, 3, 4, 6, 7, 8):
        assert rel_l2(got[s], ref[s]) < 1e-13, s
    assert abs(velmax - vref) <= 1e-13 * vref


def _random_helmholtz_modes(ops, nm, rng):
    bw = ops.bw
    ld = 2 * bw + 1
    a = 1.0 + rng.random(nm)
    b = 0.01 * rng.random(nm)
    A = a[None, None] * ops.D0[..., None] - b[None, None] * ops.D2[..., None]
    for col in (0, -1):
        diag = a * ops.D0[bw, col] - b * ops.D2[bw, col]
        A[:, col] = 0.0
        A[bw, col] = diag
    return A  # (ld, ny, nm)


def test_labs_batched_matches_oracle():
    cfg, p, ops = _setup(nx=8, ny=65, nz=8)
    rng = np.random.default_rng(5)
    nm = 97
    A = _random_helmholtz_modes(ops, nm, rng)
    lu_ref = olabs.lu(A)
    b = rng.standard_normal((cfg.ny, nm)) + 1j * rng.standard_normal((cfg.ny, nm))
    x_ref = olabs.bs(lu_ref, b)
    mm_ref = [olabs.mat_mul(B, b) for B in (ops.D0, ops.D1, ops.D2)]
    with Channel(cfg) as ch:
        # device band layout: ((j*(2bw+1)) + r) * nm + m  == numpy (ny, ld, nm) C order
        a_dev = torch.from_numpy(np.ascontiguousarray(np.transpose(A, (1, 0, 2)))).to(DEV)
        ch.labs_lu(a_dev)
        b_dev = _cplx(b)
        ch.labs_bs(a_dev, b_dev)
        outs = []
        for w in range(3):
            o = torch.zeros_like(b_dev)
            ch.labs_mat_mul(w, _cplx(b), o)
            outs.append(o)
        torch.cuda.synchronize()
        lu_got = np.transpose(a_dev.cpu().numpy(), (1, 0, 2))
        x_got = b_dev.cpu().numpy()
    assert rel_l2(lu_got, lu_ref) < 1e-14
    assert rel_l2(x_got, x_ref) < 1e-13
    for w in range(3):
        assert rel_l2(outs[w].cpu().numpy(), mm_ref[w]) < 1e-14


def _wavespace_inputs(cfg, rng):
    U = rng.standard_normal((10, cfg.nz, cfg.nxh, cfg.ny)) + 1j * rng.standard_normal((10, cfg.nz, cfg.nxh, cfg.ny))
    RK = rng.standard_normal((3, cfg.nz, cfg.nxh, cfg.ny)) + 1j * rng.standard_normal((3, cfg.nz, cfg.nxh, cfg.ny))
    U *= 0.1
    RK *= 0.1
    # slot 10 is v after the physical round trip: no kz Nyquist row, Hermitian kx = 0 plane
    nz = cfg.nz
    U[9, nz // 2] = 0.0
    for j in range(1, nz // 2):
        U[9, nz - j, 0] = np.conj(U[9, j, 0])
    U[9, 0, 0] = U[9, 0, 0].real
    return U, RK


@pytest.mark.parametrize("substep", [1, 2, 3])
@pytest.mark.parametrize("control", [0.0, -1.0])
def test_wavespace_matches_oracle(substep, control):
    cfg, p, ops = _setup(nx=16, ny=33, nz=16, control_amp=control)
    rng = np.random.default_rng(100 + substep)
    U, RK = _wavespace_inputs(cfg, rng)
    dt = 0.01
    Uo, RKo = U.copy(), RK.copy()
    sc = okmm.Scalars()
    okmm.wavespace(Uo, RKo, ops, p, substep, dt, sc, oracle_ctrl(ops, p))
    with Channel(cfg) as ch:
        Ud, RKd = _cplx(U), _cplx(RK)
        out = ch.wavespace(Ud, RKd, substep, dt)
        Ug, RKg = Ud.cpu().numpy(), RKd.cpu().numpy()
    for s in STATE_SLOTS:
        assert rel_l2(Ug[s], Uo[s]) < 1e-12, (s, rel_l2(Ug[s], Uo[s]))
    for s in range(3):
        assert rel_l2(RKg[s], RKo[s]) < 1e-12, s
    assert abs(out["phi_dpdx"][substep - 1] - sc.phi_dpdx[substep - 1]) <= 1e-12 * max(1.0, abs(sc.phi_dpdx[substep - 1]))
    assert abs(out["phi_dtdx"][substep - 1] - sc.phi_dtdx[substep - 1]) <= 1e-12 * max(1.0, abs(sc.phi_dtdx[substep - 1]))
    if substep == 3:
        assert abs(out["wall_shear_stress"] - sc.wall_shear_stress) <= 1e-12 * abs(sc.wall_shear_stress)
        assert abs(out["wall_theta_stress"] - sc.wall_theta_stress) <= 1e-12 * abs(sc.wall_theta_stress)


def _run_pair(cfg, p, ops, nsteps, dt=0.01, use_graph=True, ctrl=True):
    U = seeded_state(cfg, ops.y)
    RK = okmm.set_initial_data_uvw(U.copy(), ops, p)
    Uo, RKo = U.copy(), RK.copy()
    sco = okmm.Scalars()
    c = oracle_ctrl(ops, p) if ctrl else None
    dyr = okmm.dyr_vector(ops.y, p.dy_factor)
    d = dt
    for _ in range(nsteps):
        d, sco = okmm.rk3_step(Uo, RKo, ops, p, d, sco, dyr, c)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, dt)
        if use_graph:
            out = ch.step(nsteps)
        else:
            for _ in range(nsteps):
                for s in (1, 2, 3):
                    out = ch.time_march(s)
        Ug, RKg = ch.download_state()
    return Ug, RKg, out, Uo, RKo, sco


def test_set_initial_data_uvw_matches_oracle():
    cfg, p, ops = _setup(nx=16, ny=33, nz=16)
    U = seeded_state(cfg, ops.y)
    RKo = okmm.set_initial_data_uvw(U, ops, p)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        _, RKg = ch.download_state()
    assert rel_l2(RKg, RKo) < 1e-13


@pytest.mark.parametrize("control", [0.0, -1.0])
def test_substeps_match_oracle(control):
    cfg, p, ops = _setup(nx=16, ny=33, nz=16, control_amp=control)
    Ug, RKg, out, Uo, RKo, sco = _run_pair(cfg, p, ops, 2, use_graph=False)
    for s in STATE_SLOTS:
        assert rel_l2(Ug[s], Uo[s]) < 1e-12, s
    assert rel_l2(RKg, RKo) < 1e-12
    assert abs(out["velmax"] - sco.velmax) <= 1e-12 * sco.velmax


def test_graph_step_matches_oracle_cfl_dt():
    cfg, p, ops = _setup(nx=16, ny=33, nz=24, fixed_dt=0, control_amp=-1.0)
    Ug, RKg, out, Uo, RKo, sco = _run_pair(cfg, p, ops, 4, dt=0.0, use_graph=True)
    for s in STATE_SLOTS:
        assert rel_l2(Ug[s], Uo[s]) < 1e-11, s
    assert abs(out["dt"] - sco.dt) <= 1e-13 * sco.dt
    assert abs(out["phi_dpdx"][3] - sco.phi_dpdx[3]) <= 1e-10 * abs(sco.phi_dpdx[3])
    assert abs(out["wall_shear_stress"] - sco.wall_shear_stress) <= 1e-10 * abs(sco.wall_shear_stress)


def test_trajectory_100_steps_fp64():
    """100 RK3 steps on a 32x33x32 channel (fixed dt 0.01): rel L2 <= 1e-10 field by field."""
    cfg, p, ops = _setup(nx=32, ny=33, nz=32, lmfx=1.0, lmfz=0.5)
    Ug, RKg, out, Uo, RKo, sco = _run_pair(cfg, p, ops, 100)
    errs = {s: rel_l2(Ug[s], Uo[s]) for s in STATE_SLOTS}
    assert max(errs.values()) < 1e-10, errs


def test_mixed_precision_within_1e5():
    cfg64, p, ops = _setup(nx=32, ny=33, nz=32)
    cfg, _ = make_pair(nx=32, ny=33, nz=32, precision=1)
    U = seeded_state(cfg, ops.y)
    RK = okmm.set_initial_data_uvw(U.copy(), ops, p)
    Uo, RKo = U.copy(), RK.copy()
    dyr = okmm.dyr_vector(ops.y, p.dy_factor)
    d = 0.01
    for _ in range(20):
        d, _sc = okmm.rk3_step(Uo, RKo, ops, p, d, None, dyr)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        ch.step(20)
        Ug, _ = ch.download_state()
    errs = {s: rel_l2(Ug[s], Uo[s]) for s in STATE_SLOTS}
    assert max(errs.values()) < 1e-5, errs


def test_step_host_matches_resident():
    cfg, p, ops = _setup(nx=16, ny=33, nz=16)
    U = seeded_state(cfg, ops.y)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        Ua, RKa = ch.download_state()
        ch.step(3)
        Ub, RKb = ch.download_state()
        Uh, RKh = Ua.copy(), RKa.copy()
        ch.upload_state(Ua, RKa, 0.01)
        ch.step_host(Uh, RKh, 3)
    for s in STATE_SLOTS:
        assert np.array_equal(Uh[s], Ub[s])
    assert np.array_equal(RKh, RKb)


def test_step_host_without_stores_matches_resident():
    """kmm_step_host with rk = NULL rebuilds RK_STORE from U every call (restart option 1);
    between RK3 steps the stores are functions of U, so 3 such calls track 3 resident steps."""
    cfg, p, ops = _setup(nx=16, ny=33, nz=24, control_amp=-1.0)
    U = seeded_state(cfg, ops.y)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        Ua, _ = ch.download_state()
        ch.step(3)
        Ub, _ = ch.download_state()
        Uh = Ua.copy()
        for _ in range(3):
            ch.step_host(Uh, None, 1)
    for s in STATE_SLOTS:
        assert rel_l2(Uh[s], Ub[s]) < 1e-12, s


def test_laminar_fixed_point_gpu():
    cfg, p, ops = _setup(nx=16, ny=33, nz=16)
    U = np.zeros((10, cfg.nz, cfg.nxh, cfg.ny), dtype=np.complex128)
    U[0, 0, 0] = 1.5 * (1 - ops.y ** 2)
    U[6, 0, 0] = U[0, 0, 0]
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        out = ch.step(5)
        Ug, _ = ch.download_state()
    assert np.abs(Ug[0] - U[0]).max() < 1e-13
    assert abs(out["wall_shear_stress"] - 3 * cfg.nu) < 1e-12
    assert abs(out["phi_dpdx"][3] - 3 * cfg.nu) < 1e-12


def test_dt_out_of_range_is_a_status_not_a_fault():
    cfg, p, ops = _setup(nx=16, ny=33, nz=16)
    U = seeded_state(cfg, ops.y)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 2e5)  # above the 1e5 bound of dft_x_realspace.f90:494
        before, _ = ch.download_state()
        with pytest.raises(KmmError) as ei:
            ch.time_march(1)
        assert ei.value.code == _lib.KMM_ERR_DT
        after, _ = ch.download_state()
        assert np.array_equal(before[0], after[0])
        # the handle stays usable
        ch.dt = 0.01
        ch.step(1)


def test_nonfinite_state_is_reported():
    cfg, p, ops = _setup(nx=16, ny=33, nz=16)
    U = seeded_state(cfg, ops.y)
    U[0, 1, 1, 5] = np.nan
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        with pytest.raises(KmmError) as ei:
            ch.time_march(1)
        assert ei.value.code == _lib.KMM_ERR_NONFINITE


@pytest.mark.parametrize("precision", [0, 1])
def test_pressure_matches_oracle(precision):
    """kmm_get_pressure (get_pressure.f90) against the oracle's statistics-step pressure of the
    same state, after two steps so that all modes carry energy.  The products of the pressure
    pass are formed in FP64 on a mixed handle too, so both precisions meet 1e-11."""
    tol = 1e-11
    cfg, p, ops = _setup(nx=16, ny=33, nz=24, precision=precision, control_amp=-1.0)
    U = seeded_state(cfg, ops.y)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        ch.step(2)
        Us, _ = ch.download_state()
        Pg = ch.get_pressure()
        Ua, _ = ch.download_state()
    assert np.array_equal(Us, Ua)  # the state is not changed
    Po = okmm.pressure(Us, ops, p)
    assert rel_l2(Pg, Po) < tol
    assert rel_l2(Pg[0, 0], Po[0, 0]) < 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_statistics_match_oracle(precision):
    """kmm_get_statistics (get_statistics_1, write_spectra, the physical moments of
    dft_x_realspace, get_statistics_2) against the oracle's statistics of the same state, line by
    line and spectrum by spectrum; a second call gives identical numbers (fixed-order sums) and the
    state is unchanged.  Every line is within 1e-11 of its maximum in both precisions: the
    statistics pass computes in FP64 on a mixed handle too (in FP32 products, the y derivatives of
    the third-moment and pressure-covariance lines, whose terms cancel to ~1e-2 of their size,
    had reached 1.2e-5 of the line)."""
    tol = 1e-11
    from oracle import stats as ostats
    cfg, p, ops = _setup(nx=16, ny=33, nz=24, precision=precision, control_amp=-1.0)
    U = seeded_state(cfg, ops.y)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        ch.step(2)
        Us, _ = ch.download_state()
        g = ch.get_statistics(pressure=True)
        g2 = ch.get_statistics()
        Ua, _ = ch.download_state()
    assert np.array_equal(Us, Ua)
    for name in ostats.LINE_NAMES:
        assert np.array_equal(g["lines"][name], g2["lines"][name]), name
    o = ostats.statistics(Us, ops, p)
    errs = {}
    for i, name in enumerate(ostats.LINE_NAMES):
        ref = o["lines"][i]
        if np.abs(ref).max() < 1e-14:
            continue
        errs[name] = np.abs(g["lines"][name] - ref).max() / np.abs(ref).max()
    for name, err in errs.items():
        assert err < tol, (name, err, sorted(errs.items(), key=lambda x: -x[1])[:5])
    for i, name in enumerate(ostats.SPEC_NAMES):
        assert rel_l2(g["spec_kx"][name], o["spec_kx"][i]) < tol, ("kx", name)
        assert rel_l2(g["spec_kz"][name], o["spec_kz"][i]) < tol, ("kz", name)
    assert abs(g["U_c"] - o["u_center"]) <= 1e-12 * abs(o["u_center"])
    assert abs(g["T_c"] - o["t_center"]) <= 1e-12 * abs(o["t_center"])
    assert rel_l2(g["P"], o["P"]) < tol


def test_statistics_other_shape_tanh_grid_fp64():
    """kmm_get_statistics in FP64 on another shape (nx > nz, 41 tanh-mapped collocation points,
    no control) against the oracle: all lines, both spectra, the centre-line values and p."""
    from oracle import stats as ostats
    cfg, p = make_pair(nx=24, ny=41, nz=16, stretch=2.0, grid=1)
    p.grid = "tanh"
    ops = okmm.make_operators(p)
    U = seeded_state(cfg, ops.y)
    with Channel(cfg) as ch:
        np.testing.assert_allclose(ch.y, ops.y, rtol=0, atol=1e-14)
        ch.set_initial_data_uvw(U, 0.01)
        ch.step(1)
        Us, _ = ch.download_state()
        g = ch.get_statistics(pressure=True)
    o = ostats.statistics(Us, ops, p)
    for i, name in enumerate(ostats.LINE_NAMES):
        ref = o["lines"][i]
        if np.abs(ref).max() < 1e-14:
            continue
        err = np.abs(g["lines"][name] - ref).max() / np.abs(ref).max()
        assert err < 1e-11, (name, err)
    for i, name in enumerate(ostats.SPEC_NAMES):
        assert rel_l2(g["spec_kx"][name], o["spec_kx"][i]) < 1e-11, ("kx", name)
        assert rel_l2(g["spec_kz"][name], o["spec_kz"][i]) < 1e-11, ("kz", name)
    assert abs(g["U_c"] - o["u_center"]) <= 1e-12 * abs(o["u_center"])
    assert abs(g["T_c"] - o["t_center"]) <= 1e-12 * abs(o["t_center"])
    assert rel_l2(g["P"], o["P"]) < 1e-11
