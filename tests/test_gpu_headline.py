"""Parity of the benchmark's own configurations against the FP64 oracle, through the C ABI (GPU).

* The benchmark grid: 192x129x192, Lx = 4 pi, Lz = 4 pi / 3 (LMFx 2, LMFz 2/3), order-7 B-splines
  on the sine map, nu = 1/2800, Pr 0.71, opposition control A = -1 at y+ = 15, fixed dt 0.01,
  seeded random-phase IC.  The FP64 GPU path is held to the oracle within 1e-10 relative L2
  after 3 and after 100 RK3 steps, and the mixed-precision path within 1e-5 after 100 steps,
  field by field (u, v, w, theta).
* The small channel with control: 64x65x64, Lx = 2 pi, Lz = pi, A = -1 at y+ = 15, fixed dt
  0.01, 100 steps: FP64 within 1e-10, mixed within 1e-5.
* kmm_set_control on a handle created without control reproduces the oracle's controlled
  trajectory with per-mode gains.

The oracle here is the compiled FP64 restatement (oracle/kmm_cpu.c), which tests/test_oracle_cpu.py
holds to the numpy oracle; one oracle trajectory feeds all comparisons of a configuration.
"""
import numpy as np
import pytest

from channel_passive_b200 import Channel
from channel_passive_b200 import _lib
from oracle import cpu as ocpu
from oracle import kmm as okmm
from tests.helpers import STATE_SLOTS, make_pair, oracle_ctrl, rel_l2, seeded_state

pytestmark = pytest.mark.gpu

NAMES = {0: "u", 1: "v", 2: "w", 6: "theta"}


def _oracle_trajectory(cfg, p, checkpoints, gains=None):
    ops = okmm.make_operators(p)
    U = seeded_state(cfg, ops.y)
    prob = ocpu.Problem(p, ops, oracle_ctrl(ops, p, gains))
    Uo = U.copy()
    RKo = prob.set_initial_data_uvw(Uo)
    out, done, dt = {}, 0, 0.01
    for k in sorted(checkpoints):
        dt, sc = prob.rk3(Uo, RKo, dt, k - done)
        done = k
        out[k] = (Uo.copy(), sc[-1])
    return U, out


def _gpu_states(cfg, U, checkpoints, gains=None, set_control=None):
    res, done = {}, 0
    with Channel(cfg) as ch:
        if set_control is not None:
            ch.set_control(*set_control)
        elif gains is not None:
            ch.set_control_gains(gains)
        ch.set_initial_data_uvw(U, 0.01)
        for k in sorted(checkpoints):
            sc = ch.step(k - done)
            done = k
            res[k] = (ch.download_state(7)[0], sc)
    return res


def _errs(Ug, Uo):
    return {NAMES[f]: rel_l2(Ug[f], Uo[f]) for f in STATE_SLOTS}


@pytest.fixture(scope="module")
def headline():
    kw = dict(nx=192, ny=129, nz=192, lmfx=2.0, lmfz=2.0 / 3.0, stretch=0.9, control_amp=-1.0,
              control_yplus=15.0, fixed_dt=1)
    cfg, p = make_pair(precision=0, **kw)
    U, traj = _oracle_trajectory(cfg, p, (3, 100))
    return kw, U, traj


def test_headline_fp64_matches_oracle_3_and_100_steps(headline):
    kw, U, traj = headline
    cfg, _ = make_pair(precision=_lib.KMM_PREC_FP64, **kw)
    got = _gpu_states(cfg, U, (3, 100))
    for k in (3, 100):
        errs = _errs(got[k][0], traj[k][0])
        assert max(errs.values()) < 1e-10, (k, errs)
        sco, scg = traj[k][1], got[k][1]
        assert abs(scg["phi_dpdx"][3] - sco["phi_dpdx"][3]) <= 1e-9 * abs(sco["phi_dpdx"][3])
        assert abs(scg["wall_shear_stress"] - sco["wall_shear_stress"]) <= 1e-10 * abs(sco["wall_shear_stress"])
        assert abs(scg["wall_theta_stress"] - sco["wall_theta_stress"]) <= 1e-10 * abs(sco["wall_theta_stress"])


def test_headline_mixed_matches_oracle_100_steps(headline):
    kw, U, traj = headline
    cfg, _ = make_pair(precision=_lib.KMM_PREC_MIXED, **kw)
    got = _gpu_states(cfg, U, (100,))
    errs = _errs(got[100][0], traj[100][0])
    assert max(errs.values()) < 1e-5, errs


@pytest.mark.parametrize("precision,tol", [(_lib.KMM_PREC_FP64, 1e-10), (_lib.KMM_PREC_MIXED, 1e-5)])
def test_small_channel_with_control_100_steps(precision, tol):
    kw = dict(nx=64, ny=65, nz=64, lmfx=1.0, lmfz=0.5, stretch=0.9, control_amp=-1.0, control_yplus=15.0,
              fixed_dt=1)
    cfg, p = make_pair(precision=precision, **kw)
    U, traj = _oracle_trajectory(cfg, p, (100,))
    got = _gpu_states(cfg, U, (100,))
    errs = _errs(got[100][0], traj[100][0])
    assert max(errs.values()) < tol, errs


def test_set_control_with_gains_matches_oracle():
    """A handle made without control, then kmm_set_control(A = -1, gains, y_d at y+ = 15)."""
    kw = dict(nx=32, ny=33, nz=32, lmfx=1.0, lmfz=0.5, stretch=0.9, control_amp=-1.0, control_yplus=15.0,
              fixed_dt=1)
    cfg, p = make_pair(precision=_lib.KMM_PREC_FP64, **kw)
    rng = np.random.default_rng(11)
    gains = (1.0 + 0.05 * rng.standard_normal((p.nz, p.nxh))).astype(np.float32)
    U, traj = _oracle_trajectory(cfg, p, (5,), gains=gains.astype(np.float64))
    yd = cfg.control_yd
    cfg.control_amp = 0.0
    got = _gpu_states(cfg, U, (5,), set_control=(-1.0, gains, yd))
    errs = _errs(got[5][0], traj[5][0])
    assert max(errs.values()) < 1e-11, errs
    # and back off: amplitude 0 gives the uncontrolled trajectory
    cfg0, p0 = make_pair(precision=_lib.KMM_PREC_FP64, **dict(kw, control_amp=0.0))
    U0, traj0 = _oracle_trajectory(cfg0, p0, (2,))
    with Channel(cfg0) as ch:
        ch.set_control(-1.0, gains, yd)
        ch.set_control(0.0)
        ch.set_initial_data_uvw(U0, 0.01)
        ch.step(2)
        Ug, _ = ch.download_state(7)
    assert max(_errs(Ug, traj0[2][0]).values()) < 1e-11
