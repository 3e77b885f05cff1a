"""A fixed number of RK3 steps of the benchmark workload on one handle, for profiler captures.

    python -m channel_passive_b200.profile_case --steps 2 [--stats 1] [--precision mixed|fp64] [--nx 192 ...]
    python -m channel_passive_b200.profile_case --adjoint 2


Creates one handle (about 2.5 GB of device memory at 192x129x192 mixed), sets the seeded
random-phase initial condition, runs --warmup steps through the CUDA graph and then --steps
steps kernel by kernel (kmm_profile_step), and prints the per-kernel mean device times; then
--stats statistics-step calls (kmm_get_statistics).  Under a profiler the kernels of interest
are selected by name (k_hvhg, k_helmholtz, k_assemble, k_zinv2, k_xphys2, k_zfwd2, k_mean; for
the statistics k_ydiff, k_mean_vv, k_ppe, k_spectra, k_mom_reduce, k_stat_lines).

--adjoint N instead runs the adjoint configuration (128x97x128 FP64, fixed dt 0.01, A = -0.5 at
y+ = 15, per-mode gains 1 + N(0, 0.05)): kmm_adjoint_forward over N steps and
kmm_adjoint_backward (k_adj_factor, k_adj_modes, k_adj_mean, k_adj_probe, k_xadj2 beside the
recomputed forward substeps), and prints the gradients' norms.
"""
from __future__ import annotations

import argparse
import json
import math

from . import Channel, Config, _lib, ic

RE_TAU = 180.0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nx", type=int, default=192)
    ap.add_argument("--ny", type=int, default=129)
    ap.add_argument("--nz", type=int, default=192)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--precision", choices=("mixed", "fp64"), default="mixed")
    ap.add_argument("--no-control", action="store_true")
    ap.add_argument("--stats", type=int, default=0)
    ap.add_argument("--adjoint", type=int, default=0)
    args = ap.parse_args(argv)
    if args.adjoint:
        return adjoint_case(args.adjoint)
    prec = _lib.KMM_PREC_MIXED if args.precision == "mixed" else _lib.KMM_PREC_FP64
    cfg = Config(nx=args.nx, ny=args.ny, nz=args.nz, lmfx=2.0, lmfz=2.0 / 3.0, stretch=0.9,
                 nu=1.0 / 2800.0, pr=0.71, fixed_dt=1, precision=prec,
                 control_amp=0.0 if args.no_control else -1.0, control_yd=-1.0 + 15.0 / RE_TAU)
    with Channel(cfg) as ch:
        U0 = ic.seeded_ic(args.nx, args.ny, args.nz, ch.y, 2.0, 2.0 / 3.0, seed=20261203)
        ch.set_initial_data_uvw(U0, 0.01)
        if args.warmup:
            ch.step(args.warmup)
        prof = ch.profile_step(args.steps)
        U, _ = ch.download_state()
        st = None
        for _ in range(args.stats):
            st = ch.get_statistics()
    finite = bool(all(math.isfinite(abs(x)) for x in (U[0].sum(), U[1].sum(), U[2].sum(), U[6].sum())))
    if st is not None:
        finite = finite and all(math.isfinite(float(v.sum())) for v in st["lines"].values())
    print(json.dumps({"precision": args.precision, "steps": args.steps, "finite": finite,
                      "kernels_ms": {k: v["ms"] for k, v in prof.items()}}))
    return 0 if finite else 1


def adjoint_case(nsteps: int) -> int:
    import numpy as np

    cfg = Config(nx=128, ny=97, nz=128, lmfx=1.0, lmfz=0.5, stretch=0.9, nu=1.0 / 2800.0, pr=0.71,
                 fixed_dt=1, precision=_lib.KMM_PREC_FP64, control_amp=-0.5,
                 control_yd=-1.0 + 15.0 / RE_TAU)
    rng = np.random.default_rng(20261203)
    gains = (1.0 + 0.05 * rng.standard_normal((cfg.nz, cfg.nxh))).astype(np.float32)
    with Channel(cfg) as ch:
        ch.set_control(-0.5, gains)
        U0 = ic.seeded_ic(128, 97, 128, ch.y, 1.0, 0.5, seed=20261203)
        ch.set_initial_data_uvw(U0, 0.01)
        J = ch.adjoint_forward(nsteps, 1.0, 0.5)
        dA, dg = ch.adjoint_backward()
    finite = bool(math.isfinite(J) and math.isfinite(dA) and np.all(np.isfinite(dg)))
    print(json.dumps({"adjoint_steps": nsteps, "J": J, "dJ_dA": dA, "dJ_dgains_l2": float(np.linalg.norm(dg)),
                      "finite": finite}))
    return 0 if finite else 1


if __name__ == "__main__":
    raise SystemExit(main())
