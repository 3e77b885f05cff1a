"""Restart files of a handle on the GPU: kmm_data_store (data_store.f90:11-173) and kmm_restart
(initial_step.f90:15-56, 184-513) through the C ABI.

* The file holds what data_store writes: the state fields (U_gal added to the mean of u), g and
  phi from the stores, the mean profiles, the problem definition and the operators.
* Restart option 1 gives back u, v, w, theta bit for bit and the stores within 1e-12 away from
  the wall rows of phi (which set_initial_data_uvw recomputes and the step never reads); the
  restarted handle then steps like the original.
* Options 2 and 3 rebuild u, v, w (and phi) as the oracle's set_initial_data_gphi / _vg do
  (1e-12 relative), and without opposition control (walls at v = 0, which the rebuild assumes)
  the rebuilt u, v, w, theta are the state the file was written from (1e-9).
* Argument, file and grid errors.
"""
import numpy as np
import pytest

from channel_passive_b200 import Channel, IoFile, KmmError
from channel_passive_b200 import _lib
from oracle import kmm as okmm
from tests.helpers import STATE_SLOTS, make_pair, rel_l2, seeded_state

pytestmark = pytest.mark.gpu


def _stored(tmp_path, nsteps=2, control_amp=-1.0, **kw):
    cfg, p = make_pair(nx=32, ny=33, nz=32, control_amp=control_amp, precision=0, **kw)
    U0 = seeded_state(cfg, okmm.make_operators(p).y)
    path = str(tmp_path / "restart.h5")
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U0, 0.01)
        ch.step(nsteps)
        U, RK = ch.download_state(10)
        dt = ch.dt
        ch.data_store(path, timestep=17, time=0.25)
        ops = (ch.y.copy(), ch.integ.copy(), ch.D0.copy(), ch.D1.copy(), ch.D2.copy())
    return cfg, p, path, U, RK, dt, ops


def test_data_store_writes_the_reference_datasets(tmp_path):
    cfg, p, path, U, RK, dt, (y, integ, D0, D1, D2) = _stored(tmp_path)
    ny, nxh, nz = cfg.ny, cfg.nxh, cfg.nz
    with IoFile(path) as f:
        assert f.line_read("timestep", 1, np.int32)[0] == 17
        assert f.line_read("time", 1)[0] == 0.25 and f.line_read("dt", 1)[0] == dt
        assert f.line_read("nx", 1, np.int32)[0] == cfg.nx and f.line_read("ny", 1, np.int32)[0] == ny
        assert f.line_read("Re", 1)[0] == 1.0 / cfg.nu and f.line_read("Pr", 1)[0] == cfg.pr
        u = f.field_read("u", ny, nxh, nz)
        mean = U[0].copy()
        mean[0, 0] += cfg.u_gal  # data_store adds U_gal back
        assert np.array_equal(u, mean)
        for name, want in (("v", U[1]), ("w", U[2]), ("theta", U[6]), ("g", RK[0]), ("phi", RK[1])):
            assert np.array_equal(f.field_read(name, ny, nxh, nz), want), name
        assert np.array_equal(f.line_read("U_mean", ny), mean[0, 0].real)
        assert np.array_equal(f.line_read("T_mean", ny), U[6][0, 0].real)
        assert np.array_equal(f.line_read("LABS_COL", ny), y)
        assert np.array_equal(f.line_read("LABS_INTEGRATE", ny), integ)
        bw = f.line_read("LABS_BW", 1, np.int32)[0]
        for name, band in (("LABS_D0_BAND", D0), ("LABS_D1_BAND", D1), ("LABS_D2_BAND", D2)):
            assert np.array_equal(f.plane_read(name, 2 * bw + 1, ny), band.T), name
        full = f.plane_read("LABS_D0_FULL", ny, ny)
        assert full.shape == (ny, ny) and np.all(np.isfinite(full))
        assert "restart inhomogeneous channel flow" in f.string_get("Readme")


def test_restart_option1_roundtrip_and_continuation(tmp_path):
    cfg, p, path, U, RK, dt, _ = _stored(tmp_path)
    with Channel(cfg) as ch:
        info = ch.restart(path, 1)
        assert info == {"timestep": 17, "time": 0.25, "dt": dt}
        assert ch.dt == dt
        U1, RK1 = ch.download_state(10)
        for f in STATE_SLOTS:
            assert np.array_equal(U1[f], U[f]), f
        # set_initial_data_uvw rebuilds phi as D2 D0^-1 v - k^2 v, which differs from the evolved
        # store only in its wall rows: the step never reads them (phi's rows there are Dirichlet
        # rows), so the stores agree inside and the continuation below is unaffected
        assert rel_l2(RK1[:, :, :, 1:-1], RK[:, :, :, 1:-1]) < 1e-12
        assert np.array_equal(RK1[0], RK[0]) or rel_l2(RK1[0], RK[0]) < 1e-13
        ch.step(2)
        Ua, _ = ch.download_state(10)
    with Channel(cfg) as ch:
        ch.upload_state(U, RK, dt)
        ch.step(2)
        Ub, _ = ch.download_state(10)
    for f in STATE_SLOTS:
        assert rel_l2(Ua[f], Ub[f]) < 1e-11, f


@pytest.mark.parametrize("option", [2, 3])
def test_restart_options_2_3_match_oracle(tmp_path, option):
    cfg, p, path, U, RK, dt, _ = _stored(tmp_path, control_amp=0.0)
    ops = okmm.make_operators(p)
    ny, nxh, nz = cfg.ny, cfg.nxh, cfg.nz
    # the oracle's inputs: what data_read_gphi / data_read_vg take from the file
    with IoFile(path) as f:
        RKo = np.zeros((3, nz, nxh, ny), dtype=np.complex128)
        RKo[0] = f.field_read("g", ny, nxh, nz)
        RKo[2] = f.field_read("theta", ny, nxh, nz)
        Uo = np.zeros((10, nz, nxh, ny), dtype=np.complex128)
        if option == 2:
            RKo[1] = f.field_read("phi", ny, nxh, nz)
        else:
            Uo[1] = f.field_read("v", ny, nxh, nz)
        RKo[0, 0, 0] = f.line_read("U_mean", ny) - cfg.u_gal
        RKo[1, 0, 0] = f.line_read("W_mean", ny)
        RKo[2, 0, 0] = f.line_read("T_mean", ny)
    if option == 2:
        Uw = okmm.set_initial_data_gphi(RKo, ops, p)
        RKw = RKo
    else:
        Uw, RKw = okmm.set_initial_data_vg(Uo, RKo, ops, p)
    with Channel(cfg) as ch:
        info = ch.restart(path, option)
        assert info["timestep"] == 17 and info["dt"] == dt
        Ug, RKg = ch.download_state(10)
    for f in STATE_SLOTS:
        assert rel_l2(Ug[f], Uw[f]) < 1e-12, (option, f)
        # and the rebuilt fields are the state that was stored
        assert rel_l2(Ug[f], U[f]) < 1e-9, (option, f)
    assert rel_l2(RKg, RKw) < 1e-12


def test_restart_errors(tmp_path):
    cfg, p, path, U, RK, dt, _ = _stored(tmp_path, nsteps=1)
    with Channel(cfg) as ch:
        with pytest.raises(KmmError) as e:
            ch.restart(path, 4)
        assert e.value.code == _lib.KMM_ERR_ARG
        with pytest.raises(KmmError) as e:
            ch.restart(str(tmp_path / "absent.h5"), 1)
        assert e.value.code == _lib.KMM_ERR_IO
    small, _ = make_pair(nx=16, ny=33, nz=16, precision=0)
    with Channel(small) as ch:
        with pytest.raises(KmmError) as e:
            ch.restart(path, 1)
        assert e.value.code == _lib.KMM_ERR_IO and "restart dimensions do not match input: u" in str(e.value)
    two, _ = make_pair(nx=32, ny=33, nz=32, precision=0, n_scalar=2)
    with Channel(two) as ch:
        with pytest.raises(KmmError) as e:
            ch.restart(path, 2)
        assert e.value.code == _lib.KMM_ERR_CONFIG
