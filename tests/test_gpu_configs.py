"""The benchmark's other configurations as parity cases (GPU).

- Small channel, plain FP64 (64x65x64, Lx = 2 pi, Lz = pi, no control, fixed dt 0.01): 100 RK3
  steps against the oracle, field by field, within 1e-10 relative L2.
- Production grid (384x257x384, Lx = 2 pi, Lz = pi, tanh-stretched, nu = 1/10850, CFL 0.8,
  opposition control at y+ = 15 of Re_tau 590): too large for the oracle, so it is held to the
  properties the step must keep at any size -- a finite state, the CFL dt rule, zero divergence,
  the Hermitian kx = 0 plane -- and the mixed path to the FP64 path within 1e-5.  One passive
  scalar: the reference carries one (its second scalar does not exist there).
"""
import numpy as np
import pytest

from channel_passive_b200 import Channel
from oracle import cpu as ocpu
from oracle import kmm as okmm
from oracle import labs

from helpers import STATE_SLOTS, make_pair, rel_l2, seeded_state

pytestmark = pytest.mark.gpu


@pytest.mark.slow
def test_small_channel_fp64_100_steps_match_oracle():
    cfg, p = make_pair(nx=64, ny=65, nz=64, lmfx=1.0, lmfz=0.5, stretch=0.9)
    ops = okmm.make_operators(p)
    U = seeded_state(cfg, ops.y)
    with Channel(cfg) as ch:
        ch.set_initial_data_uvw(U, 0.01)
        out = ch.step(100)
        Ug, _ = ch.download_state()
    # the compiled FP64 restatement (held to the numpy oracle in tests/test_oracle_cpu.py)
    prob = ocpu.Problem(p, ops)
    Uo = U.copy()
    RKo = prob.set_initial_data_uvw(Uo)
    _, scs = prob.rk3(Uo, RKo, 0.01, 100)
    sc = scs[-1]
    errs = {s: rel_l2(Ug[s], Uo[s]) for s in STATE_SLOTS}
    assert max(errs.values()) < 1e-10, errs
    assert abs(out["phi_dpdx"][3] - sc["phi_dpdx"][3]) <= 1e-10 * abs(sc["phi_dpdx"][3])


def _divergence(U, ops, p, modes):
    """max |i kx u + dv/dy + i kz w| over the given (kz_index, kx) modes, with dv/dy = D1 D0^-1 v."""
    kxi, kzi = okmm.wavenumbers(p.nx, p.nz)
    j = np.array([m[0] for m in modes])
    k = np.array([m[1] for m in modes])
    v = np.ascontiguousarray(U[1][j, k].T)
    dv = labs.mat_mul(ops.D1, labs.bs(ops.D0_lu, v))
    kx = kxi[k] / p.lmfx
    kz = kzi[j] / p.lmfz
    d = 1j * kx * U[0][j, k].T + dv + 1j * kz * U[2][j, k].T
    return float(np.abs(d).max())


@pytest.mark.slow
def test_production_grid_properties_and_mixed_vs_fp64():
    re_tau = 590.0
    kw = dict(nx=384, ny=257, nz=384, lmfx=1.0, lmfz=0.5, stretch=2.0, fixed_dt=0, control_amp=-1.0,
              grid=1, nu=1.0 / 10850.0, cfl=0.8)
    cfg64, p = make_pair(precision=0, **kw)
    cfgm, _ = make_pair(precision=1, **kw)
    # detection plane y+ = 15 at Re_tau 590
    cfg64.control_yd = cfgm.control_yd = -1.0 + 15.0 / re_tau
    p.grid = "tanh"
    p.re_tau = re_tau
    ops = okmm.make_operators(p)
    U = seeded_state(cfg64, ops.y)
    outs, states = {}, {}
    for name, cfg in (("fp64", cfg64), ("mixed", cfgm)):
        with Channel(cfg) as ch:
            ch.set_initial_data_uvw(U, 1e-3)
            outs[name] = ch.step(3)
            states[name], _ = ch.download_state()
    Ud, Um = states["fp64"], states["mixed"]
    for s in STATE_SLOTS:
        assert np.all(np.isfinite(Ud[s])) and np.all(np.isfinite(Um[s]))
        assert rel_l2(Um[s], Ud[s]) < 1e-5, s
    # the CFL rule: dt = CFL / pi / velmax (dt_factor 0, read_input_file.f90:107 and
    # dft_x_realspace.f90:490-493)
    for o in outs.values():
        assert o["dt"] > 0 and abs(o["dt"] - cfg64.cfl / np.pi / o["velmax"]) <= 1e-12 * o["dt"]
    rng = np.random.default_rng(5)
    modes = [(int(a), int(b)) for a, b in zip(rng.integers(0, p.nz, 400), rng.integers(0, p.nxh, 400))
             if not (a == 0 and b == 0) and a != p.nz // 2]
    scale = max(np.abs(Ud[s]).max() for s in (0, 1, 2))
    assert _divergence(Ud, ops, p, modes) < 1e-10 * scale
    for f in STATE_SLOTS:
        for j in (1, 7, 100, p.nz // 2 - 1):
            assert np.abs(Ud[f, j, 0] - np.conj(Ud[f, p.nz - j, 0])).max() <= 1e-12 * scale
