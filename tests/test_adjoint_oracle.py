"""The oracle's discrete adjoint (oracle/adjoint.py) on the CPU: its transposes pass dot-product
tests against the forward pieces, and its gradients of the time-averaged wall shear stress and
wall scalar flux agree with central finite differences of the oracle's own step (eps = 1e-4)."""
import numpy as np
import pytest

from oracle import adjoint as oadj
from oracle import kmm as okmm
from tests.helpers import make_pair, seeded_state


def _re_dot(a, b):
    return float(np.sum((np.conj(a) * b).real))


def test_x_direction_transposes():
    """c2r and r2c (with the 3/2 padding and truncation of dft_x_realspace) against their
    transposes: <C a, mu> = <a, C^T mu> and <lam, R f> = <R^T lam, f>."""
    rng = np.random.default_rng(0)
    nx = 16
    a = rng.standard_normal((5, nx // 2)) + 1j * rng.standard_normal((5, nx // 2))
    mu = rng.standard_normal((5, nx * 3 // 2))
    assert abs(_re_dot(oadj.c2r(a, nx), mu) - _re_dot(a, oadj.c2r_T(mu, nx))) < 1e-12
    lam = rng.standard_normal((5, nx // 2)) + 1j * rng.standard_normal((5, nx // 2))
    f = rng.standard_normal((5, nx * 3 // 2))
    assert abs(_re_dot(lam, oadj.r2c(f, nx)) - _re_dot(oadj.r2c_T(lam, nx), f)) < 1e-12


def test_projection_transpose():
    cfg, p = make_pair(nx=16, ny=9, nz=16)
    rng = np.random.default_rng(1)
    shape = (p.nz, p.nxh, 9)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    y = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    assert abs(_re_dot(y, oadj.project_v(x, p)) - _re_dot(oadj.project_v_T(y, p), x)) < 1e-12


def test_helmholtz_transpose_dot():
    """solve_g's map (h, store) -> (f, store') against solve_helmholtz_T."""
    cfg, p = make_pair(nx=8, ny=33, nz=8)
    ops = okmm.make_operators(p)
    d = oadj.dense(ops)
    rng = np.random.default_rng(2)
    kx = np.array([1.0, 2.0, 0.0, 3.0])
    kz = np.array([2.0, -4.0, 2.0, 0.0])
    cz = lambda: rng.standard_normal((p.ny, 4)) + 1j * rng.standard_normal((p.ny, 4))
    for s in (1, 2, 3):
        h, st = cz(), cz()
        f, st2, _ = okmm.solve_scalar_helmholtz(h, st, ops, kx, kz, (p.nu, None), s, 0.01)
        lf, lst = cz(), cz()
        lh, lst0, _ = oadj.solve_helmholtz_T(d, p, lf, lst, kx, kz, s, 0.01, False)
        lhs = _re_dot(lf, f) + _re_dot(lst, st2)
        rhs = _re_dot(lh, h) + _re_dot(lst0, st)
        assert abs(lhs - rhs) <= 1e-10 * abs(lhs), s


@pytest.mark.parametrize("w_tau,w_q", [(1.0, 0.0), (0.0, 1.0)])
def test_gradient_matches_central_differences(w_tau, w_q):
    cfg, p = make_pair(nx=16, ny=33, nz=16, control_amp=-0.5)
    ops = okmm.make_operators(p)
    U = seeded_state(cfg, ops.y)
    RK = okmm.set_initial_data_uvw(U, ops, p)
    w_lo, w_hi = okmm.control_weights(ops, p)
    rng = np.random.default_rng(4)
    gains = 1.0 + 0.05 * rng.standard_normal((p.nz, p.nxh))
    amp, n, eps, dt = -0.5, 3, 1e-4, 0.01
    J, gA, gG = oadj.gradient(U, RK, ops, p, dt, n, (w_lo, w_hi, amp, gains), w_tau, w_q)
    obj = lambda a, g: oadj.objective(U, RK, ops, p, dt, n, (w_lo, w_hi, a, g), w_tau, w_q)
    assert abs(J - obj(amp, gains)) <= 1e-14 * abs(J)
    fd = (obj(amp + eps, gains) - obj(amp - eps, gains)) / (2 * eps)
    assert abs(gA - fd) <= 1e-4 * abs(fd)
    # the gains gradient along a random direction of all per-mode gains: single-gain derivatives
    # (~1e-9) sit at the truncation error of a 1e-4 central difference
    dg = rng.standard_normal(gains.shape)
    fd = (obj(amp, gains + eps * dg) - obj(amp, gains - eps * dg)) / (2 * eps)
    assert abs(float(np.sum(gG * dg)) - fd) <= 1e-4 * abs(fd)
