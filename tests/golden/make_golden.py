"""Regenerates the committed golden fixtures from the FP64 oracle.

    python tests/golden/make_golden.py

* bspline_k7_n32.npz: LABS_fill_full outputs for the reference's own known-answer case
  (tests/test_bspline.cpp:4-26: GSL order 7, n = 32, stretch 0 and 0.99), frozen so the
  C++ builder and the oracle are both checked against the same vectors.
* step_16x33x16.npz: one full RK3 step (fixed dt 0.01, opposition control A = -1 at
  y+ = 15) of a 16x33x16 channel from the seeded initial condition: the state before and
  after, the RK stores after, and the step diagnostics.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from channel_passive_b200 import ic  # noqa: E402
from oracle import bspline, kmm  # noqa: E402


def main():
    out = {}
    for tag, st in (("s0", 0.0), ("s099", 0.99)):
        o = bspline.fill_full(7, 32, st)
        for d in range(5):
            out[f"{tag}_D{d}"] = o["D"][d]
        out[f"{tag}_y"] = o["y"]
        out[f"{tag}_integ"] = o["integ"]
        out[f"{tag}_center"] = o["center"]
    np.savez_compressed(os.path.join(HERE, "bspline_k7_n32.npz"), **out)

    p = kmm.Params(nx=16, ny=33, nz=16, lmfx=1.0, lmfz=0.5, stretch=0.9, fixed_dt=True,
                   control_amp=-1.0, control_yplus=15.0, re_tau=180.0)
    ops = kmm.make_operators(p)
    U = ic.seeded_ic(p.nx, p.ny, p.nz, ops.y, p.lmfx, p.lmfz)
    RK = kmm.set_initial_data_uvw(U.copy(), ops, p)
    U1, RK1 = U.copy(), RK.copy()
    ctrl = (*kmm.control_weights(ops, p), p.control_amp, None)
    dt, sc = kmm.rk3_step(U1, RK1, ops, p, 0.01, None, None, ctrl)
    slots = [0, 1, 2, 6]
    np.savez_compressed(os.path.join(HERE, "step_16x33x16.npz"), U0=U[slots], U1=U1[slots], RK1=RK1,
                        dt=dt, phi_dpdx=np.array(sc.phi_dpdx), phi_dtdx=np.array(sc.phi_dtdx),
                        tau_w=sc.wall_shear_stress, q_w=sc.wall_theta_stress, velmax=sc.velmax)


if __name__ == "__main__":
    main()
