"""The autotuner (kmm_autotune / kmm_set_tuning) on the GPU: every candidate launch shape gives the
default's results bit for bit (the shapes change how lines and modes are spread over blocks, not
their arithmetic), tuning leaves the state unchanged, and its choices are reported."""
import numpy as np
import pytest

from channel_passive_b200 import Channel, KmmError
from channel_passive_b200 import _lib
from oracle import kmm as okmm
from tests.helpers import STATE_SLOTS, make_pair, seeded_state

pytestmark = pytest.mark.gpu


def _run(cfg, U, tuning=None, nsteps=2):
    with Channel(cfg) as ch:
        if tuning:
            ch.set_tuning(**tuning)
        ch.set_initial_data_uvw(U, 0.01)
        ch.step(nsteps)
        return ch.download_state(10)[0]


@pytest.mark.parametrize("precision", [0, 1])
def test_every_candidate_shape_is_bit_identical(precision):
    cfg, p = make_pair(nx=64, ny=65, nz=64, control_amp=-1.0, precision=precision)
    U = seeded_state(cfg, okmm.make_operators(p).y)
    ref = _run(cfg, U)
    with Channel(cfg) as ch:
        rep = ch.autotune()
    assert rep["tuned"] == 1
    # the candidates: variant shapes reported by the tuner's timings are tried one knob at a time
    z_lines = {16: (8, 32), 8: (4, 16)}[8 if precision == 0 else 16]
    x_shapes = [(1, 128), (4, 256)] if precision == 1 else [(1, 128), (2, 128)]
    cases = [dict(z_lines_per_block=z) for z in z_lines]
    # the z transforms with TMA-staged input tiles, at the default and both other z shapes
    cases += [dict(z_tma=1)] + [dict(z_lines_per_block=z, z_tma=1) for z in z_lines]
    cases += [dict(x_rows_per_block=r, x_threads=t) for r, t in x_shapes]
    cases += [dict(modes_per_block=64), dict(u_layout=1), dict(assemble_threads=128), dict(assemble_threads=512)]
    # hvhg: block size x the operator tables through L1 or from shared memory x staging
    cases += [dict(modes_per_block=mb, tables_shared=ts, hvhg_stage_ahead=sa)
              for mb in (32, 64) for ts in (0, 1) for sa in (0, 1, 2)]
    # Helmholtz: block size x tables x staging look-ahead
    cases += [dict(helm_modes_per_block=mb, helm_tables_shared=ts, helm_stage_ahead=sa)
              for mb in (32, 64, 128) for ts in (0, 1) for sa in (1, 2)]
    for case in cases:
        got = _run(cfg, U, case)
        for f in STATE_SLOTS:
            assert np.array_equal(got[f], ref[f]), (case, f)


def test_autotune_keeps_the_state_and_reports_its_choice():
    cfg, p = make_pair(nx=64, ny=65, nz=64, control_amp=-1.0, precision=1)
    U = seeded_state(cfg, okmm.make_operators(p).y)
    ref = _run(cfg, U, nsteps=3)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        ch.step(1)
        before, rk_before = ch.download_state(10)
        rep = ch.autotune()
        after, rk_after = ch.download_state(10)
        for f in STATE_SLOTS:
            assert np.array_equal(after[f], before[f])
        assert np.array_equal(rk_after, rk_before)
        ch.step(2)
        got, _ = ch.download_state(10)
        t = ch.tuning
    for f in STATE_SLOTS:
        assert np.array_equal(got[f], ref[f]), f
    assert t["tuned"] == 1 and t["modes_per_block"] in (32, 64) and t["assemble_threads"] in (128, 256, 512)
    assert all(x > 0 for x in rep["ms_z"] + rep["ms_x"] + rep["ms_modes"] + rep["ms_assemble"] + rep["ms_tables"])
    assert t["tables_shared"] in (0, 1) and t["helm_stage_ahead"] in (1, 2)
    # every Helmholtz shape that fits this grid was timed, and the chosen one is the fastest
    helm = [x for x in rep["ms_helm"] if x > 0]
    assert len(helm) >= 8 and min(helm) == rep["ms_layout"][0]
    assert rep["ms_step"][0] > 0 and rep["ms_step"][1] > 0
    assert t["helm_modes_per_block"] in (32, 64, 128)
    with pytest.raises(KmmError) as e:
        with Channel(cfg) as ch:
            ch.set_tuning(z_lines_per_block=7)
    assert e.value.code == _lib.KMM_ERR_ARG


def test_create_with_autotune_flag():
    cfg, p = make_pair(nx=64, ny=65, nz=64, precision=1, autotune=1)
    with Channel(cfg) as ch:
        t = ch.tuning
    # the timings of the tuning run at creation stay with the handle
    assert t["tuned"] == 1 and all(x > 0 for x in t["ms_z"] + t["ms_x"] + t["ms_modes"] + t["ms_assemble"])
    # whole substeps decide, knob group by knob group, which per-kernel picks stay: the kept set is
    # never slower than the shapes the handle had, and each group is either its pick or those
    assert 0 < t["ms_step"][0] <= t["ms_step"][1]
    assert t["u_layout"] in (0, int(np.argmin(t["ms_layout"])))


@pytest.mark.parametrize("precision", [0, 1])
def test_factor_cache_gives_the_same_numbers_across_dt_changes(precision):
    """factor_cache (fixed time step, the default there): the Helmholtz sweeps that read each
    substep's cached operator factors and influence solutions give the per-substep factorisation's
    results bit for bit, also when dt changes between steps (the cache is rebuilt for the new dt)
    and changes back."""
    cfg, p = make_pair(nx=32, ny=33, nz=32, control_amp=-1.0, precision=precision)
    U = seeded_state(cfg, okmm.make_operators(p).y)
    out = {}
    for fc in (0, 1):
        with Channel(cfg) as ch:
            assert ch.tuning["factor_cache"] == 1
            ch.set_tuning(factor_cache=fc)
            assert ch.tuning["factor_cache"] == fc
            ch.set_initial_data_uvw(U, 0.01)
            ch.step(2)
            ch.dt = 0.005
            ch.step(2)
            ch.dt = 0.01
            ch.step(1)
            out[fc] = ch.download_state(10)
    for f in STATE_SLOTS:
        assert np.array_equal(out[0][0][f], out[1][0][f]), f
    assert np.array_equal(out[0][1], out[1][1])  # the RK stores


def test_factor_cache_needs_a_fixed_time_step():
    cfg, _ = make_pair(nx=16, ny=33, nz=16, fixed_dt=0)
    with Channel(cfg) as ch:
        assert ch.tuning["factor_cache"] == 0
        with pytest.raises(KmmError) as e:
            ch.set_tuning(factor_cache=1)
        assert e.value.code == _lib.KMM_ERR_ARG
