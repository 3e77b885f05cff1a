#!/usr/bin/env python
"""Benchmark: RK3 steps/s of the KMM channel step at Re_tau 180, 192x129x192.

Headline metric: mixed-precision, graph-captured steps/s on one B200, with the
plain FP64 GPU path timed beside it and the mixed path's relative L2 error against the FP64
path after 100 steps.  Workload: Lx = 4 pi, Lz = 4 pi / 3 (LMFx = 2, LMFz = 2/3),
192 x 129 x 192 modes (288 x 129 x 288 dealiased), order-7 B-splines on the sine map,
nu = 1/2800, Pr = 0.71, opposition control A = -1 at y+ = 15, fixed dt = 0.01, seeded
divergence-free random-phase initial condition (synthetic data).

  python bench.py [--gpus N --steps K --warmup W]          our implementation
  python bench.py --impl reference [...]                    the C/OpenMP FP64 restatement of the
                                                            step (oracle/kmm_cpu.c) on the host threads

Multi-GPU: one independent channel per rank (replicas; the step has no data-path
collective), weak scaling; value = all ranks' steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RK3 steps/s at Re_tau180 192x129x192: mixed vs FP64 GPU at <=1e-5 rel L2 err"
RE_TAU = 180.0
SEED = 20261203


def workload(nx=192, ny=129, nz=192):
    return dict(nx=nx, ny=ny, nz=nz, lmfx=2.0, lmfz=2.0 / 3.0, stretch=0.9, nu=1.0 / 2800.0,
                pr=0.71, fixed_dt=1, control_amp=-1.0, control_yd=-1.0 + 15.0 / RE_TAU)


def workload_name(w):
    return (f"KMM RK3 step {w['nx']}x{w['ny']}x{w['nz']} Re_tau180 (LMFx 2, LMFz 2/3), Pr 0.71 passive "
            f"scalar, opposition control A=-1 at y+=15, fixed dt 0.01, seeded random-phase IC")


# ------------------------------------------------------------------------------------------
# algorithmic bytes per kernel launch (each kernel's own required HBM traffic)
# ------------------------------------------------------------------------------------------
def kernel_bytes(w, s_nl, control=True, scalars=1):
    """Each kernel's required HBM traffic per launch; a second scalar adds one state field, one
    store and three products."""
    nxh = w["nx"] // 2
    nspec = nxh * w["nz"] * w["ny"]
    nmid = nxh * (w["nz"] * 3 // 2) * w["ny"]
    s_st = 16
    nf, npd, nst = 3 + scalars, 5 + 3 * scalars, 2 + scalars
    return {
        "zinv": nf * nspec * s_st + nf * nmid * s_nl,
        "xphys": nf * nmid * s_nl + npd * nmid * s_nl,
        "zfwd": npd * nmid * s_nl + npd * nspec * s_nl,
        "wavespace": npd * nspec * s_nl + (nst + (1 if control else 0)) * nspec * s_st + (nf + nst) * nspec * s_st,
    }


WAVESPACE_PARTS = ("hvhg", "helmholtz", "assemble")


def group_wavespace(prof):
    """Adds the solver group 'wavespace' = hvhg + helmholtz + assemble (one launch each per
    substep): the algorithmic bytes of the per-mode solve belong to the three kernels together."""
    g = dict(prof)
    g["wavespace"] = {"ms": sum(prof[p]["ms"] for p in WAVESPACE_PARTS), "launches": prof["hvhg"]["launches"]}
    return g


def step_bytes(w, s_nl, control=True, scalars=1):
    kb = kernel_bytes(w, s_nl, control, scalars)
    return 3 * sum(kb.values())


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic():
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            return json.load(f)
    except Exception:
        return {}


# ------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", self.gpu_id, f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        except Exception:
            pass
        finally:
            try:
                os.unlink(self.path)
            except Exception:
                pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------------------
# distributed plumbing (replicas)
# ------------------------------------------------------------------------------------------
def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return world, rank, local


def init_dist(world, backend):
    if world <= 1:
        return None
    import datetime

    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=120))
    return dist


def max_over_ranks(value: float, dist, device) -> float:
    """Max of a per-rank float over all ranks (identity without a process group)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(dist, device):
    if dist is None:
        return
    import torch
    t = torch.zeros(1, device=device)
    dist.all_reduce(t)


# ------------------------------------------------------------------------------------------
# CPU reference: the compiled FP64 restatement (oracle/kmm_cpu.c) on every host thread
# ------------------------------------------------------------------------------------------
def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class CpuReference:
    """The workload on the host: the C/OpenMP FP64 restatement of the step (the same algorithm as
    the numpy oracle, checked against it in tests/test_oracle_cpu.py) on all host threads, from
    the same seeded IC with the RK stores built by set_initial_data_uvw.  Every timed step is a
    complete RK3 step (three substeps, all 129 planes and all modes, the mean lines and the CFL
    update) on the state the previous step left."""

    def __init__(self, w, nthreads=0):
        from channel_passive_b200 import ic
        from oracle import cpu as ocpu
        from oracle import kmm as okmm
        ocpu.build()
        p = okmm.Params(nx=w["nx"], ny=w["ny"], nz=w["nz"], lmfx=w["lmfx"], lmfz=w["lmfz"],
                        stretch=w["stretch"], nu=w["nu"], pr=w["pr"], fixed_dt=True,
                        control_amp=w["control_amp"], control_yplus=15.0, re_tau=RE_TAU)
        ops = okmm.make_operators(p)
        ctrl = (*okmm.control_weights(ops, p), p.control_amp, None)
        self.prob = ocpu.Problem(p, ops, ctrl, nthreads=nthreads)
        self.U = ic.seeded_ic(p.nx, p.ny, p.nz, ops.y, p.lmfx, p.lmfz, seed=SEED)
        self.RK = self.prob.set_initial_data_uvw(self.U)
        self.threads = nthreads or ocpu.threads()
        self.w = w

    def step_seconds(self) -> float:
        t0 = time.perf_counter()
        self.prob.rk3(self.U, self.RK, 0.01, 1)
        return time.perf_counter() - t0

    def sample_text(self, nsteps):
        w = self.w
        return (f"C/OpenMP FP64 restatement of the step (oracle/kmm_cpu.c; restatement, not the reference "
                f"binary, which needs gfortran, MPI, FFTW, GSL and HDF5) on {self.threads} host threads: "
                f"{nsteps} complete RK3 steps of {w['nx']}x{w['ny']}x{w['nz']} from the seeded IC, timed "
                f"one by one with the state carried from step to step")


def run_reference(args):
    world, rank, local = dist_env()
    if rank != 0:
        return 0
    w = workload()
    ref = CpuReference(w)
    for _ in range(args.warmup):
        t_w = ref.step_seconds()
    # complete steps only; if the requested count would run past the time cap, fewer are run and
    # "steps" says how many
    k = max(1, min(args.steps, int(args.ref_seconds / max(t_w, 1e-9))))
    times = [ref.step_seconds() for _ in range(k)]
    sec_per_step = float(np.mean(times))
    value = 1.0 / sec_per_step
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": 0,
        "steps": k, "requested_steps": args.steps, "warmup": args.warmup, "ms_per_step": sec_per_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded random-phase IC)",
        "config": {"workload": workload_name(w), "nx": w["nx"], "ny": w["ny"], "nz": w["nz"],
                   "precision": "fp64", "parallelism": f"cpu x{ref.threads} threads"},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": ref.threads, "kind": "port",
                         "sample": ref.sample_text(k)},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_seconds": float(np.sum(times)),
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------
# our implementation
# ------------------------------------------------------------------------------------------
def cpu_baseline_quick(w, seconds=12.0):
    """Rank 0, N = 1: the CPU restatement on every host thread, complete RK3 steps for about
    `seconds` after one warm-up step."""
    ref = CpuReference(w)
    ref.step_seconds()
    times = []
    while sum(times) < seconds and len(times) < 20:
        times.append(ref.step_seconds())
    t = float(np.mean(times))
    return {"value": 1.0 / t, "unit": "steps/s", "cores": ref.threads, "kind": "port",
            "sample": ref.sample_text(len(times)) + "; after one warm-up step"}


# 16 independent channels of uneven sizes, mixed precision, Re_tau 180 (Lx 2 pi, Lz pi), CFL time
# step, each with its own seeded IC, opposition amplitude A ~ U[-1, 0] and detection plane
# y+ ~ U[10, 20].  Amplitudes below -1 give the opposition loop a gain above one: the FP64
# restatement itself diverges from this IC (velmax 40 -> 4455 in 10 steps at A = -1.47,
# y+ = 11.6, even under the CFL time step), so they are not drawn.
ENSEMBLE_A = (-1.0, 0.0)
ENSEMBLE_SHAPES = [(64, 65, 64)] * 6 + [(96, 97, 96)] * 6 + [(128, 97, 128)] * 4


def run_ensemble(args, device, local, rank):
    """Aggregate grid-point-steps/s of the 16-channel ensemble stepped through kmm_ensemble_step
    (every channel's graph launches enqueued on its own stream before any wait) against the same
    channels stepped one by one (kmm_step per channel, in turn).  Both arms are timed by CUDA
    events recorded on an idle device right before and right after the host call."""
    import torch

    from channel_passive_b200 import Channel, Config, ensemble_step, ic
    from channel_passive_b200 import _lib

    rng = np.random.default_rng(SEED + 7 + rank)
    chans, members = [], []
    for i, (nx, ny, nz) in enumerate(ENSEMBLE_SHAPES):
        amp = float(rng.uniform(*ENSEMBLE_A))
        yplus = float(rng.uniform(10.0, 20.0))
        ch = Channel(Config(nx=nx, ny=ny, nz=nz, lmfx=1.0, lmfz=0.5, stretch=0.9, nu=1.0 / 2800.0, pr=0.71,
                            fixed_dt=0, control_amp=amp, control_yd=-1.0 + yplus / RE_TAU,
                            precision=_lib.KMM_PREC_MIXED, device=local))
        U = ic.seeded_ic(nx, ny, nz, ch.y, 1.0, 0.5, seed=SEED + 100 * rank + i)
        chans.append((ch, U))
        members.append({"shape": f"{nx}x{ny}x{nz}", "A": amp, "y_plus": yplus})
    points = sum(nx * ny * nz for nx, ny, nz in ENSEMBLE_SHAPES)
    k = args.ensemble_steps
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def reset():
        for ch, U in chans:
            ch.set_initial_data_uvw(U, 0.01)
        torch.cuda.synchronize()

    def clock(fn):
        torch.cuda.synchronize()
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    hs = [ch for ch, _ in chans]
    reset()
    ensemble_step(hs, args.warmup)                 # graphs captured, clocks up
    for ch in hs:
        ch.step(1)
    reset()
    ms_one = clock(lambda: [ch.step(k) for ch in hs])
    reset()
    ms_ens = clock(lambda: ensemble_step(hs, k))
    for ch in hs:
        ch.close()
    return {"channels": len(hs), "shapes": "6x 64x65x64, 6x 96x97x96, 4x 128x97x128 (Lx 2 pi, Lz pi)",
            "precision": "mixed", "steps_per_channel": k, "dt": "CFL 1.0 per channel",
            "control": "A ~ U[-1, 0], y+ ~ U[10, 20] per channel",
            "grid_point_steps_per_s": points * k / (ms_ens * 1e-3),
            "one_by_one_grid_point_steps_per_s": points * k / (ms_one * 1e-3),
            "speedup_vs_one_by_one": ms_one / ms_ens, "ms": ms_ens, "one_by_one_ms": ms_one,
            "members": members,
            "api": "kmm_ensemble_step over 16 handles (stream-concurrent CUDA graphs); one by one = "
                   "kmm_step(k) per handle in turn"}


# The adjoint configuration: 128x97x128, Lx 2 pi, Lz pi, Pr 0.71, fixed dt 0.01, opposition control
# at y+ = 15 with amplitude A = -0.5 and per-(kx, kz) FP32 gains 1 + N(0, 0.05) (seeded).  A = -0.5:
# the FP64 restatement of the step stays bounded over the 200 steps from this IC (velmax <= 112);
# at A = -1 velmax reaches 167 (a CFL number of 1.7 at dt 0.01).
ADJOINT_AMP = -0.5


def run_adjoint(args, device, local, rank):
    """Gradients of the time-averaged wall shear stress and wall scalar flux over the adjoint
    configuration's steps with respect to the control amplitude and the per-mode gains, through
    kmm_adjoint_forward / kmm_adjoint_backward (FP64, one checkpoint per step, substeps recomputed).
    Timed by CUDA events on the handle's stream around each host call; dJ/dA is checked against a
    central difference (eps 1e-4) of the same GPU step."""
    import torch

    from channel_passive_b200 import Channel, Config, ic
    from channel_passive_b200 import _lib

    w = dict(nx=128, ny=97, nz=128)
    cfg = Config(lmfx=1.0, lmfz=0.5, stretch=0.9, nu=1.0 / 2800.0, pr=0.71, fixed_dt=1,
                 precision=_lib.KMM_PREC_FP64, control_amp=ADJOINT_AMP, control_yd=-1.0 + 15.0 / RE_TAU,
                 device=local, **w)
    n = args.adjoint_steps
    rng = np.random.default_rng(SEED + 4 + rank)
    ch = Channel(cfg)
    gains = (1.0 + 0.05 * rng.standard_normal((cfg.nz, cfg.nxh))).astype(np.float32)
    U0 = ic.seeded_ic(w["nx"], w["ny"], w["nz"], ch.y, cfg.lmfx, cfg.lmfz, seed=SEED + rank)
    stream = torch.cuda.ExternalStream(ch.stream_ptr, device=device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]

    def run(amp, g, w_tau, w_q, backward=True):
        ch.set_control(amp, g)
        ch.set_initial_data_uvw(U0, 0.01)
        torch.cuda.synchronize()
        ev[0].record(stream)
        J = ch.adjoint_forward(n, w_tau, w_q)
        ev[1].record(stream)
        grads = ch.adjoint_backward() if backward else None
        ev[2].record(stream)
        torch.cuda.synchronize()
        return J, grads, ev[0].elapsed_time(ev[1]), (ev[1].elapsed_time(ev[2]) if backward else None)

    run(ADJOINT_AMP, gains, 1.0, 0.0)  # buffers, checkpoints and graph made outside the timing
    Jt, (dAt, dgt), ms_f, ms_b = run(ADJOINT_AMP, gains, 1.0, 0.0)
    Jq, (dAq, dgq), _, _ = run(ADJOINT_AMP, gains, 0.0, 1.0)
    eps = 1e-4
    Jp = run(ADJOINT_AMP + eps, gains, 1.0, 0.0, False)[0]
    Jm = run(ADJOINT_AMP - eps, gains, 1.0, 0.0, False)[0]
    fd_t = (Jp - Jm) / (2 * eps)
    Jp = run(ADJOINT_AMP + eps, gains, 0.0, 1.0, False)[0]
    Jm = run(ADJOINT_AMP - eps, gains, 0.0, 1.0, False)[0]
    fd_q = (Jp - Jm) / (2 * eps)
    ch.close()
    pts = w["nx"] * w["ny"] * w["nz"]
    return {"workload": "128x97x128 Re_tau 180 (Lx 2 pi, Lz pi), Pr 0.71, fixed dt 0.01, opposition control "
                        f"A = {ADJOINT_AMP} at y+ = 15 with per-mode gains 1 + N(0, 0.05)",
            "steps": n, "precision": "fp64",
            "forward_ms": ms_f, "backward_ms": ms_b, "backward_over_forward": ms_b / ms_f,
            "forward_grid_point_steps_per_s": pts * n / (ms_f * 1e-3),
            "tau_w": {"J": Jt, "dJ_dA": dAt, "fd_dJ_dA": fd_t, "rel_err_vs_fd": abs(dAt - fd_t) / abs(fd_t),
                      "gains_grad_l2": float(np.linalg.norm(dgt))},
            "q_w": {"J": Jq, "dJ_dA": dAq, "fd_dJ_dA": fd_q, "rel_err_vs_fd": abs(dAq - fd_q) / abs(fd_q),
                    "gains_grad_l2": float(np.linalg.norm(dgq))},
            "api": "kmm_adjoint_forward (one checkpoint per step) + kmm_adjoint_backward (substeps recomputed); "
                   "FD: central, eps 1e-4, same GPU step"}


def run_production(args, device, local, rank, dist):
    """The Re_tau 590 production grid: 384x257x384, Lx 2 pi, Lz pi, tanh-mapped y, nu 1/10850,
    CFL 0.8, opposition control A = -1 at y+ = 15 of Re_tau 590, two passive scalars (Pr 0.71 and
    Pr 0.2; the second in field 11, started from the first's profile).  Mixed-precision and FP64
    RK3 steps/s through the CUDA graph, each timed by CUDA events on the handle's stream, the
    step's HBM roofline fraction, and mixed vs FP64 after the timed steps."""
    import torch

    from channel_passive_b200 import Channel, Config, ic
    from channel_passive_b200 import _lib

    w = dict(nx=384, ny=257, nz=384)
    common = dict(lmfx=1.0, lmfz=0.5, stretch=2.0, grid=_lib.KMM_GRID_TANH, nu=1.0 / 10850.0, pr=0.71,
                  cfl=0.8, fixed_dt=0, control_amp=-1.0, control_yd=-1.0 + 15.0 / 590.0, device=local,
                  n_scalar=2, pr2=0.2, bulk_t2=1.0, **w)
    k = args.production_steps
    res, states = {}, {}
    U0 = None
    for name, prec in (("mixed", _lib.KMM_PREC_MIXED), ("fp64", _lib.KMM_PREC_FP64)):
        ch = Channel(Config(precision=prec, **common))
        if U0 is None:
            U10 = ic.seeded_ic(w["nx"], w["ny"], w["nz"], ch.y, 1.0, 0.5, seed=SEED + rank)
            U0 = np.zeros((11,) + U10.shape[1:], dtype=np.complex128)
            U0[:10] = U10
            U0[10] = U10[6]
        ch.set_initial_data_uvw(U0, 1e-3)
        # tuned on the started state (the CFL rule needs a velocity field for its whole-step
        # comparisons); the tuner puts the state back
        tuning = ch.autotune()
        ch.step(args.warmup)
        ch.set_initial_data_uvw(U0, 1e-3)
        stream = torch.cuda.ExternalStream(ch.stream_ptr, device=device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier(dist, device)
        torch.cuda.synchronize()
        e0.record(stream)
        ch.step_async(k)
        e1.record(stream)
        out = ch.sync()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), dist, device)
        states[name], _ = ch.download_state(11)
        prof = ch.profile_step(2)
        ch.close()
        s_nl = 8 if name == "mixed" else 16
        peak, _kind = measured_peaks()
        sb = step_bytes(w, s_nl, scalars=2)
        res[name] = {"steps_per_s": k / (ms * 1e-3), "ms_per_step": ms / k, "last_dt": out["dt"],
                     "step_algorithmic_bytes": sb,
                     "step_frac": sb / (ms / k * 1e-3) / 1e9 / peak,
                     "q_w": [out["wall_theta_stress"], out["wall_theta_stress2"]],
                     "kernels_ms": {kn: v["ms"] for kn, v in prof.items()},
                     "tuning": {kt: v for kt, v in tuning.items()
                                if not kt.startswith("ms_") or kt in ("ms_step", "ms_x", "ms_helm")}}
    names = {0: "u", 1: "v", 2: "w", 6: "theta", 10: "theta2"}
    Um, Ud = states["mixed"], states["fp64"]
    rel = {names[f]: float(np.linalg.norm(Um[f] - Ud[f]) / np.linalg.norm(Ud[f])) for f in names}
    return {"workload": "384x257x384 Re_tau 590 (Lx 2 pi, Lz pi, tanh y map), nu 1/10850, CFL 0.8, "
                        "opposition control A=-1 at y+=15, two passive scalars Pr 0.71 and Pr 0.2",
            "steps": k, "warmup": args.warmup, "mixed": res["mixed"], "fp64": res["fp64"],
            "mixed_over_fp64": res["mixed"]["steps_per_s"] / res["fp64"]["steps_per_s"],
            "grid_point_steps_per_s": res["mixed"]["steps_per_s"] * w["nx"] * w["ny"] * w["nz"],
            "rel_l2_mixed_vs_fp64": rel,
            "roofline_peak": "of measured HBM copy bandwidth",
            "scalars": "Pr 0.71 and Pr 0.2 (the reference carries one; the second is checked against the "
                       "build's own FP64 oracle)"}


def run_kmm(args):
    import torch

    from channel_passive_b200 import Channel, Config, ic
    from channel_passive_b200 import _lib

    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    dist = init_dist(world, "nccl")
    w = workload(args.nx, args.ny, args.nz)
    common = dict(nx=w["nx"], ny=w["ny"], nz=w["nz"], lmfx=w["lmfx"], lmfz=w["lmfz"], stretch=w["stretch"],
                  nu=w["nu"], pr=w["pr"], fixed_dt=1, control_amp=w["control_amp"],
                  control_yd=w["control_yd"], device=local)
    # both handles run the autotuner at creation (kmm_autotune: launch shapes timed on this grid)
    mixed = Channel(Config(precision=_lib.KMM_PREC_MIXED, autotune=1, **common))
    fp64 = Channel(Config(precision=_lib.KMM_PREC_FP64, autotune=1, **common))
    U0 = ic.seeded_ic(w["nx"], w["ny"], w["nz"], mixed.y, w["lmfx"], w["lmfz"], seed=SEED + rank)
    dt = 0.01
    # accuracy: 100 steps from the same IC, mixed vs FP64 (the FP64 GPU path matches the oracle
    # to 1e-10 in the parity tests)
    for ch in (mixed, fp64):
        ch.set_initial_data_uvw(U0, dt)
        ch.step(args.acc_steps)
    Um, _ = mixed.download_state()
    Ud, _ = fp64.download_state()
    names = {0: "u", 1: "v", 2: "w", 6: "theta"}
    rel = {names[s]: float(np.linalg.norm(Um[s] - Ud[s]) / np.linalg.norm(Ud[s])) for s in names}

    def timed(ch, k, wmup):
        ch.step(wmup)
        stream = torch.cuda.ExternalStream(ch.stream_ptr, device=device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier(dist, device)
        torch.cuda.synchronize()
        e0.record(stream)
        ch.step_async(k)
        e1.record(stream)
        out = ch.sync()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        return max_over_ranks(ms, dist, device), out

    gpu_id = local
    try:
        props = torch.cuda.get_device_properties(local)
        uuid = str(getattr(props, "uuid", "") or "")
        gpu_id = ("GPU-" + uuid) if uuid and not uuid.startswith("GPU-") else (uuid or str(local))
    except Exception:
        gpu_id = str(local)
    with ClockSampler(str(gpu_id)) as clk:
        ms_mixed, out_m = timed(mixed, args.steps, args.warmup)
    clocks = clk.summary()
    ms_fp64, _ = timed(fp64, args.steps, args.warmup)
    per_rank_sps = args.steps / (ms_mixed / 1e3)
    value = world * args.steps / (ms_mixed / 1e3)
    fp64_value = world * args.steps / (ms_fp64 / 1e3)

    # per-kernel device time (event pairs around every launch) for the roofline
    prof = group_wavespace(mixed.profile_step(args.prof_steps))
    prof64 = group_wavespace(fp64.profile_step(args.prof_steps))
    kb = kernel_bytes(w, 8)
    kb64 = kernel_bytes(w, 16)
    totals = {k: prof[k]["ms"] * prof[k]["launches"] for k in kb}
    dom = max(totals, key=totals.get)
    peak, peak_kind = measured_peaks()
    achieved = kb[dom] / (prof[dom]["ms"] * 1e-3) / 1e9
    traffic = profile_traffic().get(dom)
    kernels = {k: {"ms": prof[k]["ms"], "GB_s": kb[k] / (prof[k]["ms"] * 1e-3) / 1e9,
                   "frac": kb[k] / (prof[k]["ms"] * 1e-3) / 1e9 / peak} for k in kb}
    kernels64 = {k: {"ms": prof64[k]["ms"], "GB_s": kb64[k] / (prof64[k]["ms"] * 1e-3) / 1e9,
                     "frac": kb64[k] / (prof64[k]["ms"] * 1e-3) / 1e9 / peak} for k in kb64}
    kernels["wavespace"]["parts_ms"] = {p: prof[p]["ms"] for p in WAVESPACE_PARTS}
    kernels64["wavespace"]["parts_ms"] = {p: prof64[p]["ms"] for p in WAVESPACE_PARTS}

    # end to end: host-resident state in pinned memory, full upload + step + download per step
    nxh = w["nx"] // 2
    nspec = nxh * w["nz"] * w["ny"]
    U_h = torch.zeros((7, w["nz"], nxh, w["ny"]), dtype=torch.complex128).pin_memory()
    Uc, _ = mixed.download_state(7)
    U_h.copy_(torch.from_numpy(Uc))
    stream = torch.cuda.ExternalStream(mixed.stream_ptr, device=device)
    # restart option 1 per call: only u, v, w, theta cross the bus, RK_STORE is rebuilt from U
    mixed.step_host_ptr(U_h.data_ptr(), 7, None, 1)
    barrier(dist, device)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        mixed.step_host_ptr(U_h.data_ptr(), 7, None, 1)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), dist, device)
    e2e_value = world * args.e2e_steps / (ms_e2e / 1e3)
    io_bytes = 4 * nspec * 16

    # a statistics step (kmm_get_statistics: statistics, spectra, moments, pressure) of the
    # current state, outputs left on the device; timed outside the step region
    mixed.get_statistics(download=False)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.stat_calls):
        mixed.get_statistics(download=False)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_stat = max_over_ranks(e0.elapsed_time(e1), dist, device) / args.stat_calls

    ens = run_ensemble(args, device, local, rank) if args.ensemble_steps > 0 else None
    prod = run_production(args, device, local, rank, dist) if args.production_steps > 0 else None
    adj = run_adjoint(args, device, local, rank) if args.adjoint_steps > 0 else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_quick(w)

    # per substep: begin, zinv, xphys, zfwd, mean lines, hvhg (which also takes the control
    # probes), helmholtz, assemble; plus the dt update of substep 1
    launches_per_step = 3 * 8 + 1
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_mixed / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic (seeded divergence-free random-phase IC, seed 20261203 + rank)",
        "config": {"workload": workload_name(w), "nx": w["nx"], "ny": w["ny"], "nz": w["nz"],
                   "precision": "mixed (FP32 transforms/products, FP64 state, solves, mean modes)",
                   "graph": True, "parallelism": f"replicas x{world}",
                   "l2": "no flush: the resident state and slabs (>1 GB) exceed the 126 MB L2 every step"},
        "grid_point_steps_per_s": value * w["nx"] * w["ny"] * w["nz"],
        "fp64": {"value": fp64_value, "ms_per_step": ms_fp64 / args.steps, "kernels": kernels64,
                 "tuning": fp64.tuning},
        "tuning": mixed.tuning,
        "mixed_over_fp64": value / fp64_value,
        "rel_l2_mixed_vs_fp64": rel,
        "rel_l2_steps": args.acc_steps,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "algorithmic_bytes": kb[dom],
                     "step_algorithmic_bytes": step_bytes(w, 8),
                     "step_frac": step_bytes(w, 8) / (ms_mixed / args.steps * 1e-3) / 1e9 / peak,
                     "kernels": kernels},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "steps/s", "h2d_bytes_per_step": io_bytes,
                "d2h_bytes_per_step": io_bytes,
                "api": "kmm_step_host(rk = NULL): pinned host U (reference layout; u, v, w, theta) uploaded, RK_STORE rebuilt on the device as restart option 1 does, one RK3 step, U downloaded"},
        "statistics": {"ms_per_call": ms_stat, "per_step_time": ms_stat / (ms_mixed / args.steps),
                       "api": "kmm_get_statistics: the 58 stat-file lines, 2 x 18 spectra, U_c, T_c "
                              "and the pressure of the current state (statistics step), on the device"},
        "ensemble": ens,
        "production": prod,
        "adjoint": adj,
        "gpu_launches": launches_per_step * args.steps,
        "clocks": clocks,
        "last_step": {"dt": out_m["dt"], "dpdx": out_m["phi_dpdx"][3], "tau_w": out_m["wall_shear_stress"],
                      "dTdx": out_m["phi_dtdx"][3], "q_w": out_m["wall_theta_stress"]},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    mixed.close()
    fp64.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


def free_port() -> int:
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch_ranks(n: int, argv) -> int:
    """`bench.py --gpus N` started without a launcher: run the same command as N ranks (one
    process per GPU) under torch.distributed.run on this node, so N independent channels are
    stepped and timed as max over ranks.  Rank 0's JSON line is the output."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={free_port()}", os.path.abspath(__file__)] + list(argv)
    return subprocess.call(cmd)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="kmm", choices=["kmm", "reference"])
    ap.add_argument("--nx", type=int, default=192)
    ap.add_argument("--ny", type=int, default=129)
    ap.add_argument("--nz", type=int, default=192)
    ap.add_argument("--acc-steps", type=int, default=100)
    ap.add_argument("--prof-steps", type=int, default=5)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--stat-calls", type=int, default=5, help="statistics-step calls timed")
    ap.add_argument("--production-steps", type=int, default=20,
                    help="RK3 steps timed on the 384x257x384 production grid (0: skip)")
    ap.add_argument("--adjoint-steps", type=int, default=200,
                    help="RK3 steps of the adjoint configuration's gradient (0: skip)")
    ap.add_argument("--ensemble-steps", type=int, default=50,
                    help="RK3 steps per channel of the 16-channel ensemble (0: skip)")
    ap.add_argument("--ref-seconds", type=float, default=150.0,
                    help="cap on the reference arm's timed seconds (complete steps only)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return relaunch_ranks(args.gpus, sys.argv[1:] if argv is None else list(argv))
    if args.impl == "reference":
        return run_reference(args)
    return run_kmm(args)


if __name__ == "__main__":
    sys.exit(main())
