"""kmm_ensemble_step: independent channels of different sizes, precisions and control settings
stepped together, each channel's CUDA graph enqueued on its own stream before any is waited on.
Every channel must come out bit-identical to the same channel stepped alone, and one failing
channel must be reported without spoiling the others."""
import numpy as np
import pytest

pytest.importorskip("torch")

from channel_passive_b200 import Channel, KmmError, ensemble_step
from channel_passive_b200 import _lib
from oracle import kmm as okmm
from tests.helpers import STATE_SLOTS, make_pair, seeded_state

pytestmark = pytest.mark.gpu

# (nx, ny, nz, precision, control_amp, fixed_dt): uneven shapes, both precisions, control on
# and off, fixed and CFL time steps
MEMBERS = [(16, 33, 16, 0, 0.0, 1), (24, 41, 16, 0, -1.0, 1), (32, 33, 32, 1, 0.0, 1),
           (16, 21, 24, 1, -0.5, 0), (48, 49, 32, 0, -1.5, 0)]


def _members():
    out = []
    for i, (nx, ny, nz, prec, amp, fdt) in enumerate(MEMBERS):
        cfg, p = make_pair(nx=nx, ny=ny, nz=nz, precision=prec, control_amp=amp, fixed_dt=fdt)
        y = okmm.make_operators(p).y
        out.append((cfg, seeded_state(cfg, y, seed=100 + i)))
    return out


def _solo(cfg, U, nsteps):
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        sc = ch.step(nsteps)
        Ug, RKg = ch.download_state()
    return Ug, RKg, sc


def test_ensemble_matches_each_channel_alone():
    members = _members()
    solo = [_solo(cfg, U, 3) for cfg, U in members]
    chans = [Channel(cfg) for cfg, _ in members]
    try:
        for ch, (_, U) in zip(chans, members):
            ch.set_initial_data_uvw(U, 0.01)
        ensemble_step(chans, 1)
        outs = ensemble_step(chans, 2)
        for k, ch in enumerate(chans):
            Ug, RKg = ch.download_state()
            Us, RKs, scs = solo[k]
            for s in STATE_SLOTS:
                assert np.array_equal(Ug[s], Us[s]), (k, s)
            assert np.array_equal(RKg, RKs), k
            assert outs[k]["dt"] == scs["dt"], k
            assert outs[k]["velmax"] == scs["velmax"], k
            assert outs[k]["wall_shear_stress"] == scs["wall_shear_stress"], k
    finally:
        for ch in chans:
            ch.close()


def test_ensemble_reports_a_failing_member_and_steps_the_rest():
    members = _members()[:3]
    bad = members[1][1].copy()
    bad[0, 1, 1, 5] = np.nan
    members[1] = (members[1][0], bad)
    chans = [Channel(cfg) for cfg, _ in members]
    try:
        for ch, (_, U) in zip(chans, members):
            ch.set_initial_data_uvw(U, 0.01)
        with pytest.raises(KmmError) as ei:
            ensemble_step(chans, 2)
        assert ei.value.code == _lib.KMM_ERR_NONFINITE
        for k in (0, 2):
            Us, RKs, _ = _solo(members[k][0], members[k][1], 2)
            Ug, RKg = chans[k].download_state()
            for s in STATE_SLOTS:
                assert np.array_equal(Ug[s], Us[s]), (k, s)
    finally:
        for ch in chans:
            ch.close()


def test_ensemble_argument_checks():
    assert ensemble_step([], 3) == []
    cfg, _ = make_pair()
    with Channel(cfg) as ch:
        with pytest.raises(ValueError):
            ensemble_step([ch, ch], 1)
