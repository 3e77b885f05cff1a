"""ctypes binding of the compiled oracle (oracle/kmm_cpu.c; TEST INFRASTRUCTURE ONLY).

The C restatement runs the same FP64 algorithm as ``oracle.kmm`` with OpenMP over wall-normal
planes and over (kx, kz) modes.  Tests use it for trajectories that the numpy oracle would take
minutes over (the 192x129x192 grid, 100-step runs), and bench.py times it as the CPU baseline.
It is checked against ``oracle.kmm`` on the CPU (tests/test_oracle_cpu.py).

``build()`` compiles ``oracle/lib/libkmm_oracle.so`` with gcc (x86-64-v3, OpenMP); the shared
library travels with the repository like the product library.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess
from pathlib import Path

import numpy as np

from . import kmm as okmm

HERE = Path(__file__).resolve().parent
SRC = HERE / "kmm_cpu.c"
LIB = HERE / "lib" / "libkmm_oracle.so"
CFLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-std=gnu11"]


def build(force: bool = False) -> Path:
    if not force and LIB.exists() and LIB.stat().st_mtime >= SRC.stat().st_mtime:
        return LIB
    LIB.parent.mkdir(exist_ok=True)
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [shutil.which("gcc") or os.environ.get("CC", "gcc")] + CFLAGS + [str(SRC), "-o", str(tmp), "-lm"]
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode:
        raise RuntimeError("oracle build failed:\n" + " ".join(cmd) + "\n" + r.stdout)
    os.replace(tmp, LIB)
    return LIB


class Params(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("bw", C.c_int32),
                ("lmfx", C.c_double), ("lmfz", C.c_double), ("nu", C.c_double), ("pr", C.c_double),
                ("bulk_u", C.c_double), ("bulk_w", C.c_double), ("bulk_t", C.c_double),
                ("u_gal", C.c_double), ("cflx", C.c_double), ("dt_factor", C.c_double),
                ("dxr", C.c_double), ("dzr", C.c_double), ("fixed_dt", C.c_int32),
                ("nthreads", C.c_int32), ("control_amp", C.c_double)]


class Ops(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("d0", "d1", "d2", "d0lu", "integ", "dyr", "wlo", "whi", "gains")]


class Scalars(C.Structure):
    _fields_ = [("dt", C.c_double), ("velmax", C.c_double), ("phi_dpdx", C.c_double * 4),
                ("phi_dtdx", C.c_double * 4), ("wall_shear_stress", C.c_double),
                ("wall_theta_stress", C.c_double)]

    def as_dict(self):
        return {"dt": self.dt, "velmax": self.velmax, "phi_dpdx": list(self.phi_dpdx),
                "phi_dtdx": list(self.phi_dtdx), "wall_shear_stress": self.wall_shear_stress,
                "wall_theta_stress": self.wall_theta_stress}


_lib = None


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        for name in ("kmm_oracle_rk3",):
            fn = getattr(lib, name)
            fn.restype = C.c_int
            fn.argtypes = [C.POINTER(Params), C.POINTER(Ops), C.c_void_p, C.c_void_p, C.POINTER(C.c_double),
                           C.c_int, C.POINTER(Scalars)]
        lib.kmm_oracle_substep.restype = C.c_int
        lib.kmm_oracle_substep.argtypes = [C.POINTER(Params), C.POINTER(Ops), C.c_void_p, C.c_void_p,
                                           C.POINTER(C.c_double), C.c_int, C.POINTER(Scalars)]
        lib.kmm_oracle_threads.restype = C.c_int
        lib.kmm_oracle_set_initial_data_uvw.restype = C.c_int
        lib.kmm_oracle_set_initial_data_uvw.argtypes = [C.POINTER(Params), C.POINTER(Ops), C.c_void_p, C.c_void_p]
        _lib = lib
    return _lib


def threads() -> int:
    return load().kmm_oracle_threads()


class Problem:
    """The C oracle's view of one channel: parameters and operators in its layouts (the arrays
    are kept alive here)."""

    def __init__(self, p: okmm.Params, ops: okmm.Operators, ctrl=None, nthreads: int = 0):
        self.p, self.ops = p, ops
        f = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).T)  # (ld, ny) -> Fortran order
        self._keep = [f(ops.D0), f(ops.D1), f(ops.D2), f(ops.D0_lu), np.ascontiguousarray(ops.integ),
                      okmm.dyr_vector(ops.y, p.dy_factor)]
        amp = 0.0
        wlo = whi = np.zeros(p.ny)
        gains = None
        if ctrl is not None:
            wlo, whi, amp, gains = ctrl
        self._keep += [np.ascontiguousarray(wlo, dtype=np.float64), np.ascontiguousarray(whi, dtype=np.float64)]
        g = None if gains is None else np.ascontiguousarray(np.asarray(gains, dtype=np.float64).reshape(-1))
        self._keep.append(g)
        ptr = lambda a: None if a is None else a.ctypes.data
        self.ops_c = Ops(*[ptr(a) for a in self._keep])
        self.params = Params(nx=p.nx, ny=p.ny, nz=p.nz, bw=ops.bw, lmfx=p.lmfx, lmfz=p.lmfz, nu=p.nu, pr=p.pr,
                             bulk_u=p.bulk_u, bulk_w=p.bulk_w, bulk_t=p.bulk_t, u_gal=p.u_gal, cflx=p.cflx,
                             dt_factor=p.dt_factor, dxr=p.dxr, dzr=p.dzr, fixed_dt=int(bool(p.fixed_dt)),
                             nthreads=int(nthreads), control_amp=float(amp))

    @staticmethod
    def _check(U, RK, p):
        for a, nf in ((U, 10), (RK, 3)):
            if a.dtype != np.complex128 or not a.flags.c_contiguous or a.shape != (nf, p.nz, p.nx // 2, p.ny):
                raise ValueError("U (10, nz, nxh, ny) and RK (3, nz, nxh, ny) must be C-contiguous complex128")

    def set_initial_data_uvw(self, U):
        """initial_step.f90:139-179: the RK stores (3, nz, nxh, ny) from u, v, w, theta."""
        RK = np.zeros((3,) + U.shape[1:], dtype=np.complex128)
        self._check(U, RK, self.p)
        rc = load().kmm_oracle_set_initial_data_uvw(C.byref(self.params), C.byref(self.ops_c), U.ctypes.data,
                                                    RK.ctypes.data)
        if rc:
            raise RuntimeError(f"kmm_oracle_set_initial_data_uvw failed ({rc})")
        return RK

    def rk3(self, U, RK, dt: float, nsteps: int = 1):
        """nsteps RK3 steps in place (like oracle.kmm.rk3_step repeated); returns (dt, [scalars])."""
        self._check(U, RK, self.p)
        d = C.c_double(dt)
        sc = (Scalars * max(nsteps, 1))()
        rc = load().kmm_oracle_rk3(C.byref(self.params), C.byref(self.ops_c), U.ctypes.data, RK.ctypes.data,
                                   C.byref(d), int(nsteps), sc)
        if rc == 3:
            raise okmm.DtError(f"ABORT due to timestep dt = {d.value}")
        if rc:
            raise RuntimeError(f"kmm_oracle_rk3 failed ({rc})")
        return d.value, [sc[i].as_dict() for i in range(nsteps)]

    def substep(self, U, RK, s: int, dt: float):
        """One time_march substep in place; returns (dt, scalars)."""
        self._check(U, RK, self.p)
        d = C.c_double(dt)
        sc = Scalars()
        rc = load().kmm_oracle_substep(C.byref(self.params), C.byref(self.ops_c), U.ctypes.data, RK.ctypes.data,
                                       C.byref(d), int(s), C.byref(sc))
        if rc == 3:
            raise okmm.DtError(f"ABORT due to timestep dt = {d.value}")
        if rc:
            raise RuntimeError(f"kmm_oracle_substep failed ({rc})")
        return d.value, sc.as_dict()
