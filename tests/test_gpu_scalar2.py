"""A second passive scalar (n_scalar = 2, the production configuration's Pr 0.71 and Pr 0.2) on the
GPU, through the C ABI.  The reference carries one scalar, so the second is checked against the
build's own FP64 oracle extended the same way (oracle/kmm.py: theta2 in field 11, its products
u, v, w theta2 formed like f7..f9, its solve as solve_t with Pr2, its mean line as the theta block
of wave00 with its own bulk value).

* Given the first scalar's Prandtl number and bulk value, theta2 must reproduce theta bit for bit,
  and the velocity must equal a one-scalar run's (a passive scalar does not feed back).
* With Pr2 = 0.2: u, v, w, theta, theta2 and both scalars' forcing and wall flux against the
  oracle, FP64 within 1e-11 after 3 steps with opposition control, mixed precision within 1e-5.
"""
import numpy as np
import pytest

from channel_passive_b200 import Channel, KmmError
from channel_passive_b200 import _lib
from oracle import kmm as okmm
from tests.helpers import STATE_SLOTS, STATE_SLOTS2, make_pair, oracle_ctrl, rel_l2, seeded_state, with_scalar2

pytestmark = pytest.mark.gpu


def test_second_scalar_with_the_first_ones_parameters_reproduces_it():
    kw = dict(nx=16, ny=33, nz=16, control_amp=-1.0, fixed_dt=1, precision=0)
    cfg1, p = make_pair(**kw)
    cfg2, _ = make_pair(n_scalar=2, pr2=cfg1.pr, bulk_t2=cfg1.bulk_t, **kw)
    U = seeded_state(cfg1, okmm.make_operators(p).y)
    with Channel(cfg1) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        s1 = ch.step(3)
        U1, _ = ch.download_state(10)
    with Channel(cfg2) as ch:
        ch.set_initial_data_uvw(with_scalar2(U), 0.01)
        s2 = ch.step(3)
        U2, RK2 = ch.download_state(11)
    # theta2 rides in its own packed FFT line, so it equals theta to rounding, not bit for bit
    assert rel_l2(U2[10], U2[6]) < 1e-13
    assert rel_l2(RK2[3], RK2[2]) < 1e-13
    assert abs(s2["wall_theta_stress2"] - s2["wall_theta_stress"]) <= 1e-12 * abs(s2["wall_theta_stress"])
    # the velocity and the first scalar are the one-scalar run's, bit for bit
    for f in STATE_SLOTS:
        assert np.array_equal(U2[f], U1[f]), f
    assert s2["phi_dpdx"] == s1["phi_dpdx"] and s2["phi_dtdx"] == s1["phi_dtdx"]


@pytest.mark.parametrize("precision,tol,nsteps", [(0, 1e-11, 3), (1, 1e-5, 20)])
def test_second_scalar_matches_oracle(precision, tol, nsteps):
    cfg, p = make_pair(nx=32, ny=33, nz=32, control_amp=-1.0, fixed_dt=1, precision=precision, n_scalar=2,
                       pr2=0.2, bulk_t2=0.5)
    ops = okmm.make_operators(p)
    U10 = seeded_state(cfg, ops.y)
    rng = np.random.default_rng(8)
    theta2 = U10[6] * (0.5 + 0.1 * rng.standard_normal(U10[6].shape))
    theta2[0, 0] = 0.5 * U10[6][0, 0]
    U = with_scalar2(U10, theta2)
    Uo = U.copy()
    RKo = okmm.set_initial_data_uvw(Uo, ops, p)
    ctrl = oracle_ctrl(ops, p)
    for _ in range(nsteps):
        _, sco = okmm.rk3_step(Uo, RKo, ops, p, 0.01, ctrl=ctrl)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        scg = ch.step(nsteps)
        Ug, RKg = ch.download_state(11)
    errs = {f: rel_l2(Ug[f], Uo[f]) for f in STATE_SLOTS2}
    assert max(errs.values()) < tol, errs
    if precision == 0:
        assert rel_l2(RKg, RKo) < tol
        assert abs(scg["phi_dtdx2"][3] - sco.phi_dtdx2[3]) <= 1e-9 * abs(sco.phi_dtdx2[3])
        assert abs(scg["wall_theta_stress2"] - sco.wall_theta_stress2) <= 1e-10 * abs(sco.wall_theta_stress2)
        assert abs(scg["wall_theta_stress"] - sco.wall_theta_stress) <= 1e-10 * abs(sco.wall_theta_stress)


def test_second_scalar_needs_field_11():
    cfg, p = make_pair(nx=16, ny=33, nz=16, n_scalar=2)
    with Channel(cfg) as ch:
        U = np.zeros((10, cfg.nz, cfg.nxh, cfg.ny), dtype=np.complex128)
        with pytest.raises(KmmError) as e:
            ch.set_initial_data_uvw(U, 0.01)
        assert e.value.code == _lib.KMM_ERR_ARG


@pytest.mark.parametrize("precision", [0, 1])
def test_second_scalar_block_shapes_are_bit_identical(precision):
    """The two-scalar Helmholtz kernel with 64 or 96 modes per block and the operator tables in
    shared memory (the shapes a large grid starts with) gives the 32-mode blocks' results bit
    for bit: the shapes spread the modes over blocks, not the arithmetic."""
    cfg, p = make_pair(nx=32, ny=33, nz=32, control_amp=-1.0, fixed_dt=1, precision=precision, n_scalar=2,
                       pr2=0.2, bulk_t2=0.5)
    U10 = seeded_state(cfg, okmm.make_operators(p).y)
    U = with_scalar2(U10, 0.5 * U10[6])
    out = []
    for shape in (dict(helm_modes_per_block=32, helm_tables_shared=0),
                  dict(helm_modes_per_block=64, helm_tables_shared=1),
                  dict(helm_modes_per_block=96, helm_tables_shared=1),
                  dict(helm_modes_per_block=96, helm_tables_shared=0)):
        with Channel(cfg) as ch:
            ch.set_tuning(**shape)
            assert ch.tuning["helm_modes_per_block"] == shape["helm_modes_per_block"]
            ch.set_initial_data_uvw(U, 0.01)
            ch.step(3)
            out.append(ch.download_state(11))
    for Ug, RKg in out[1:]:
        for f in STATE_SLOTS2:
            assert np.array_equal(Ug[f], out[0][0][f]), f
        assert np.array_equal(RKg, out[0][1])
