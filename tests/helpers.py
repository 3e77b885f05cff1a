"""Shared set-up for the parity tests: one configuration expressed both as the C-ABI
Config and as the oracle's Params, seeded initial conditions and error norms."""
from __future__ import annotations

import numpy as np

from channel_passive_b200 import Config, ic
from oracle import kmm as okmm

RE_TAU = 180.0


def make_pair(nx=16, ny=33, nz=16, lmfx=1.0, lmfz=0.5, stretch=0.9, control_amp=0.0,
              control_yplus=15.0, fixed_dt=1, precision=0, **kw):
    cfg = Config(nx=nx, ny=ny, nz=nz, lmfx=lmfx, lmfz=lmfz, stretch=stretch, fixed_dt=fixed_dt,
                 precision=precision, control_amp=control_amp,
                 control_yd=-1.0 + control_yplus / RE_TAU, **kw)
    p = okmm.Params(nx=nx, ny=ny, nz=nz, labs_k=cfg.labs_k, lmfx=lmfx, lmfy=cfg.lmfy, lmfz=lmfz,
                    stretch=stretch, nu=cfg.nu, pr=cfg.pr, bulk_u=cfg.bulk_vel_u,
                    bulk_w=cfg.bulk_vel_w, bulk_t=cfg.bulk_t, u_gal=cfg.u_gal, cfl=cfg.cfl,
                    dt_factor=cfg.dt_factor, dy_factor=cfg.dy_factor, fixed_dt=bool(fixed_dt),
                    control_amp=control_amp, control_yplus=control_yplus, re_tau=RE_TAU,
                    n_scalar=max(1, cfg.n_scalar), pr2=cfg.pr2, bulk_t2=cfg.bulk_t2)
    return cfg, p


def with_scalar2(U, theta2=None):
    """U (10, ...) -> (14, ...) with theta2 in slot 10 (the oracle's two-scalar layout; the C ABI
    reads field 11 of nf >= 11).  theta2 defaults to theta (slot 6)."""
    out = np.zeros((14,) + U.shape[1:], dtype=U.dtype)
    out[:10] = U[:10]
    out[10] = U[6] if theta2 is None else theta2
    return out


def oracle_ctrl(ops, p, gains=None):
    if p.control_amp == 0.0:
        return None
    w_lo, w_hi = okmm.control_weights(ops, p)
    return (w_lo, w_hi, p.control_amp, gains)


def seeded_state(cfg, y, seed=20261203, amplitude=0.1):
    U = ic.seeded_ic(cfg.nx, cfg.ny, cfg.nz, y, cfg.lmfx, cfg.lmfz, seed=seed, amplitude=amplitude)
    return U


def rel_l2(a, b):
    den = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0))


STATE_SLOTS = (0, 1, 2, 6)
STATE_SLOTS2 = (0, 1, 2, 6, 10)
