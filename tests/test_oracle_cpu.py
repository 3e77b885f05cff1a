"""The compiled oracle (oracle/kmm_cpu.c) against the numpy oracle (oracle/kmm.py), on the CPU.

Both restate the same reference routines in FP64 (time_march.f90:36-128 and everything it
calls); they differ only in evaluation order (the C twin batches its FFTs as a Stockham
transform and groups some products differently), so they agree to a few ulps per substep.
"""
import numpy as np
import pytest

from oracle import cpu as ocpu
from oracle import kmm as okmm
from tests.helpers import STATE_SLOTS, make_pair, oracle_ctrl, rel_l2, seeded_state


@pytest.fixture(scope="module", autouse=True)
def _built():
    ocpu.build()


def _case(**kw):
    cfg, p = make_pair(**kw)
    ops = okmm.make_operators(p)
    U = seeded_state(cfg, ops.y)
    return cfg, p, ops, U


def _max_err(Ua, RKa, Ub, RKb):
    e = [rel_l2(Ua[f], Ub[f]) for f in STATE_SLOTS]
    e += [rel_l2(RKa[i], RKb[i]) for i in range(3)]
    return max(e)


@pytest.mark.parametrize("kw", [
    dict(nx=16, ny=33, nz=16),
    dict(nx=16, ny=33, nz=24, control_amp=-1.0),
    dict(nx=24, ny=33, nz=16, control_amp=-0.5, fixed_dt=0),
    dict(nx=20, ny=21, nz=40, lmfx=2.0, lmfz=2.0 / 3.0),
])
def test_substeps_match_numpy_oracle(kw):
    cfg, p, ops, U = _case(**kw)
    RK = okmm.set_initial_data_uvw(U, ops, p)
    ctrl = oracle_ctrl(ops, p)
    prob = ocpu.Problem(p, ops, ctrl)
    Un, RKn = U.copy(), RK.copy()
    Uc, RKc = U.copy(), RK.copy()
    dt_n = dt_c = 0.01
    for s in (1, 2, 3):
        sc = okmm.Scalars()
        dt_n = okmm.time_march(Un, RKn, ops, p, s, dt_n, sc, ctrl=ctrl)
        dt_c, scc = prob.substep(Uc, RKc, s, dt_c)
        assert _max_err(Uc, RKc, Un, RKn) < 1e-13, s
        assert abs(dt_c - dt_n) <= 1e-14 * dt_n
        # phi = (bulk - int/2) / (int_1/2) cancels O(1) terms down to ~1e-6: compare absolutely
        assert abs(scc["phi_dpdx"][s - 1] - sc.phi_dpdx[s - 1]) <= 1e-13
        assert abs(scc["phi_dtdx"][s - 1] - sc.phi_dtdx[s - 1]) <= 1e-13
        if s == 1:
            assert abs(scc["velmax"] - sc.velmax) <= 1e-13 * sc.velmax
    assert abs(scc["wall_shear_stress"] - sc.wall_shear_stress) <= 1e-10 * abs(sc.wall_shear_stress)
    assert abs(scc["wall_theta_stress"] - sc.wall_theta_stress) <= 1e-10 * abs(sc.wall_theta_stress)


def test_steps_with_gains_match_numpy_oracle():
    cfg, p, ops, U = _case(nx=16, ny=33, nz=16, control_amp=-1.0)
    rng = np.random.default_rng(5)
    gains = (1.0 + 0.05 * rng.standard_normal((p.nz, p.nxh))).astype(np.float32).astype(np.float64)
    ctrl = oracle_ctrl(ops, p, gains)
    RK = okmm.set_initial_data_uvw(U, ops, p)
    Un, RKn = U.copy(), RK.copy()
    Uc, RKc = U.copy(), RK.copy()
    dt = 0.01
    for _ in range(3):
        _, scn = okmm.rk3_step(Un, RKn, ops, p, dt, ctrl=ctrl)
    _, scc = ocpu.Problem(p, ops, ctrl).rk3(Uc, RKc, dt, 3)
    assert _max_err(Uc, RKc, Un, RKn) < 1e-12
    assert abs(scc[-1]["phi_dpdx"][3] - scn.phi_dpdx[3]) <= 1e-11  # sum of three phi / dt


def test_initial_stores_match_numpy_oracle():
    cfg, p, ops, U = _case(nx=16, ny=33, nz=24)
    RKn = okmm.set_initial_data_uvw(U, ops, p)
    RKc = ocpu.Problem(p, ops).set_initial_data_uvw(U)
    for i in range(3):
        assert rel_l2(RKc[i], RKn[i]) < 1e-14


def test_thread_count_does_not_change_results():
    cfg, p, ops, U = _case(nx=16, ny=33, nz=16, control_amp=-1.0)
    ctrl = oracle_ctrl(ops, p)
    RK = okmm.set_initial_data_uvw(U, ops, p)
    out = []
    for nt in (1, 3):
        Uc, RKc = U.copy(), RK.copy()
        ocpu.Problem(p, ops, ctrl, nthreads=nt).rk3(Uc, RKc, 0.01, 2)
        out.append((Uc, RKc))
    for f in STATE_SLOTS:
        assert np.array_equal(out[0][0][f], out[1][0][f])
    assert np.array_equal(out[0][1], out[1][1])


def test_dt_abort_matches_reference_rule():
    """dt outside (1e-14, 1e5] aborts (dft_x_realspace.f90:494-497)."""
    cfg, p, ops, U = _case(nx=16, ny=33, nz=16)
    RK = okmm.set_initial_data_uvw(U, ops, p)
    with pytest.raises(okmm.DtError):
        ocpu.Problem(p, ops).rk3(U.copy(), RK.copy(), 1e-15, 1)
