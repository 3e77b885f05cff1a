"""The discrete adjoint on the GPU (kmm_adjoint_forward / kmm_adjoint_backward through the C ABI,
and the torch.autograd.Function over them).

* Against the FP64 reference gradient of the oracle's own adjoint (oracle/adjoint.py, itself held
  to central finite differences on the CPU): objective, dJ/dA and dJ/dgains of the time-averaged
  wall shear stress and wall scalar flux, 1e-8 relative.
* Against central finite differences of the GPU step itself (eps = 1e-4):
  dJ/dA and the gains gradient along a random direction, 1e-4 relative.
* The state after backward is the state forward left; the configuration checks hold.
* The per-substep band cache of the backward follows dt: gradients bit-identical to a fresh
  handle after dt changes between backward calls.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from channel_passive_b200 import Channel, KmmError
from channel_passive_b200 import _lib
from channel_passive_b200.autograd import control_objective
from oracle import adjoint as oadj
from oracle import kmm as okmm
from tests.helpers import STATE_SLOTS, make_pair, seeded_state

pytestmark = pytest.mark.gpu


def _gains(p, seed=4):
    rng = np.random.default_rng(seed)
    return (1.0 + 0.05 * rng.standard_normal((p.nz, p.nxh))).astype(np.float32)


def _gpu_grad(cfg, U, amp, gains, nsteps, w_tau, w_q, dt=0.01):
    with Channel(cfg) as ch:
        ch.set_control(amp, gains)
        ch.set_initial_data_uvw(U, dt)
        J = ch.adjoint_forward(nsteps, w_tau, w_q)
        Uf, RKf = ch.download_state(7)
        dA, dg = ch.adjoint_backward()
        Ub, RKb = ch.download_state(7)
    for f in STATE_SLOTS:
        assert np.array_equal(Ub[f], Uf[f])
    assert np.array_equal(RKb, RKf)
    return J, dA, dg


@pytest.mark.parametrize("w_tau,w_q", [(1.0, 0.0), (0.0, 1.0)])
def test_adjoint_matches_oracle_gradient(w_tau, w_q):
    amp, nsteps = -0.5, 3
    cfg, p = make_pair(nx=16, ny=33, nz=16, control_amp=amp, precision=0, fixed_dt=1)
    ops = okmm.make_operators(p)
    U = seeded_state(cfg, ops.y)
    gains = _gains(p)
    RK = okmm.set_initial_data_uvw(U, ops, p)
    w_lo, w_hi = okmm.control_weights(ops, p)
    Jo, gAo, gGo = oadj.gradient(U, RK, ops, p, 0.01, nsteps, (w_lo, w_hi, amp, gains.astype(np.float64)),
                                 w_tau, w_q)
    J, dA, dg = _gpu_grad(cfg, U, amp, gains, nsteps, w_tau, w_q)
    assert abs(J - Jo) <= 1e-10 * abs(Jo)
    assert abs(dA - gAo) <= 1e-8 * abs(gAo), (dA, gAo)
    assert np.linalg.norm(dg - gGo) <= 1e-8 * np.linalg.norm(gGo)


def test_adjoint_matches_central_differences_32():
    """32x33x32 channel, A = -1 at y+ = 15, 10 steps: the adjoint against central differences of
    the GPU step (eps = 1e-4) for A and for the gains along a random direction."""
    amp, nsteps, eps = -1.0, 10, 1e-4
    cfg, p = make_pair(nx=32, ny=33, nz=32, control_amp=amp, precision=0, fixed_dt=1)
    ops = okmm.make_operators(p)
    U = seeded_state(cfg, ops.y)
    gains = _gains(p, 7)
    J, dA, dg = _gpu_grad(cfg, U, amp, gains, nsteps, 1.0, 0.0)
    rng = np.random.default_rng(9)
    dgd = rng.standard_normal(gains.shape)
    with Channel(cfg) as ch:
        def obj(a, g):
            ch.set_control(a, g)
            ch.set_initial_data_uvw(U, 0.01)
            return ch.adjoint_forward(nsteps, 1.0, 0.0)
        # gains are float32 in the ABI: perturb them by an amount float32 represents
        fdA = (obj(amp + eps, gains) - obj(amp - eps, gains)) / (2 * eps)
        gp = (gains.astype(np.float64) + eps * dgd).astype(np.float32)
        gm = (gains.astype(np.float64) - eps * dgd).astype(np.float32)
        step = (gp.astype(np.float64) - gm.astype(np.float64))  # the difference float32 kept
        fdG = obj(amp, gp) - obj(amp, gm)
    assert abs(dA - fdA) <= 1e-4 * abs(fdA), (dA, fdA)
    assert abs(float(np.sum(dg * step)) - fdG) <= 1e-4 * abs(fdG), (float(np.sum(dg * step)), fdG)


def test_autograd_function_gives_the_adjoint_gradients():
    amp0, nsteps = -0.5, 3
    cfg, p = make_pair(nx=16, ny=33, nz=16, control_amp=amp0, precision=0, fixed_dt=1)
    ops = okmm.make_operators(p)
    U = seeded_state(cfg, ops.y)
    gains = _gains(p)
    J_ref, dA_ref, dg_ref = _gpu_grad(cfg, U, amp0, gains, nsteps, 0.3, 0.7)
    with Channel(cfg) as ch:
        amp = torch.tensor(amp0, dtype=torch.float64, requires_grad=True)
        g = torch.tensor(gains, dtype=torch.float64, requires_grad=True)
        J = control_objective(amp, g, ch, U, nsteps, 0.01, 0.3, 0.7)
        (2.0 * J).backward()
    assert abs(float(J) - J_ref) <= 1e-14 * abs(J_ref)
    assert abs(float(amp.grad) - 2.0 * dA_ref) <= 1e-12 * abs(dA_ref)
    np.testing.assert_allclose(g.grad.numpy(), 2.0 * dg_ref, rtol=1e-12, atol=0)


def test_adjoint_configuration_checks():
    cfg, p = make_pair(nx=16, ny=33, nz=16, control_amp=-0.5, precision=1, fixed_dt=1)
    with Channel(cfg) as ch:
        with pytest.raises(KmmError) as e:
            ch.adjoint_forward(2)
        assert e.value.code == _lib.KMM_ERR_CONFIG
    cfg, p = make_pair(nx=16, ny=33, nz=16, control_amp=-0.5, precision=0, fixed_dt=0)
    with Channel(cfg) as ch:
        with pytest.raises(KmmError) as e:
            ch.adjoint_forward(2)
        assert e.value.code == _lib.KMM_ERR_CONFIG
    cfg, p = make_pair(nx=16, ny=33, nz=16, control_amp=-0.5, precision=0, fixed_dt=1)
    with Channel(cfg) as ch:
        with pytest.raises(KmmError) as e:
            ch.adjoint_backward()
        assert e.value.code == _lib.KMM_ERR_ARG


def test_adjoint_band_cache_follows_dt():
    """The backward caches each substep's factored bands for its fixed dt: a second backward at
    another dt on the same handle rebuilds them, and gives the gradients of a fresh handle at that
    dt bit for bit (and a third, back at the first dt, those of the first call)."""
    amp, nsteps = -0.5, 2
    cfg, p = make_pair(nx=16, ny=33, nz=16, control_amp=amp, precision=0, fixed_dt=1)
    U = seeded_state(cfg, okmm.make_operators(p).y)
    gains = _gains(p)
    fresh = {dt: _gpu_grad(cfg, U, amp, gains, nsteps, 1.0, 0.5, dt=dt) for dt in (0.01, 0.005)}
    with Channel(cfg) as ch:
        ch.set_control(amp, gains)
        for dt in (0.01, 0.005, 0.01):
            ch.set_initial_data_uvw(U, dt)
            J = ch.adjoint_forward(nsteps, 1.0, 0.5)
            dA, dg = ch.adjoint_backward()
            Jf, dAf, dgf = fresh[dt]
            assert J == Jf and dA == dAf and np.array_equal(dg, dgf), dt
