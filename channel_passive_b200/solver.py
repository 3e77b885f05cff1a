"""Host-side mirror of the reference's time-step interface over libkmm's C ABI.

The names follow the reference routines they stand in for:

* ``read_input_file``  -> read_input_file.f90:38-89 (positional ``input`` file)
* ``labs_fill_full``   -> LABS_fill_full (labs_fill_full.cpp:35-195)
* ``Channel``          -> the module state set up by LABS_initialize / RK3_initialize /
  ppdfftw_initialize, with ``time_march`` (time_march.f90:36-128),
  ``set_initial_data_uvw`` (initial_step.f90:139-179) and the main-loop step
  (main.f90:134-193) as methods.

Arrays use the reference layout: complex128 numpy arrays of shape (nf, nz, nxh, ny)
(= Fortran U(ny, nxh, nz, nf)); RK stores (3, nz, nxh, ny).  Errors raise
``KmmError`` where the reference would call mpi_abort.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field, fields

import numpy as np

from . import _lib
from ._lib import KmmConfig, KmmError, KmmInfo, KmmScalars, KmmTuning, check

NFIELD = 10


@dataclass
class Config:
    nx: int = 64
    ny: int = 65
    nz: int = 64
    no_of_field: int = 10
    rk_scheme: int = 3
    labs_k: int = 6
    lmfx: float = 1.0
    lmfy: float = 1.0
    lmfz: float = 0.5
    stretch: float = 0.9
    grid: int = _lib.KMM_GRID_SINE
    nu: float = 1.0 / 2800.0
    pr: float = 0.71
    bulk_vel_u: float = 1.0
    bulk_vel_w: float = 0.0
    bulk_t: float = 1.0
    u_gal: float = 0.0
    cfl: float = 1.0
    dt_factor: float = 0.0
    dy_factor: float = 1.0
    fixed_dt: int = 0
    precision: int = _lib.KMM_PREC_FP64
    control_amp: float = 0.0
    control_yd: float = -1.0 + 15.0 / 180.0
    device: int = 0
    n_scalar: int = 1
    pr2: float = 0.2
    bulk_t2: float = 1.0
    autotune: int = 0

    def to_c(self) -> KmmConfig:
        c = KmmConfig()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c

    @classmethod
    def from_c(cls, c: KmmConfig) -> "Config":
        return cls(**{f.name: getattr(c, f.name) for f in fields(cls)})

    @property
    def nxh(self):
        return self.nx // 2

    @property
    def nx32(self):
        return self.nx * 3 // 2

    @property
    def nz32(self):
        return self.nz * 3 // 2


def read_input_file(path: str) -> Config:
    """Parse the reference's positional ``input`` file (read_input_file.f90:38-89)."""
    lib = _lib.load()
    c = KmmConfig()
    check(lib.kmm_read_input_file(str(path).encode(), C.byref(c)))
    return Config.from_c(c)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def labs_fill_full(k: int, n: int, stretch: float, ly: float = 2.0) -> dict:
    """B-spline operators exactly as LABS_fill_full returns them (K = GSL order = labs_k+1).

    M[d] is returned as (n, n) arrays indexed [point, basis] (the C array M_d[basis + point*n]).
    """
    lib = _lib.load()
    M = [np.zeros((n, n)) for _ in range(5)]
    y = np.zeros(n)
    yknot = np.zeros(n - k + 2)
    integ = np.zeros(n)
    center = np.zeros(n)
    kk, nn = C.c_int(k), C.c_int(n)
    st, l = C.c_double(stretch), C.c_double(ly)
    lib.kmm_labs_fill_full(*[_dptr(m) for m in M], _dptr(y), _dptr(yknot), _dptr(integ),
                           _dptr(center), C.byref(kk), C.byref(nn), C.byref(st), C.byref(l))
    return {"D": np.stack(M), "y": y, "breakpoints": yknot, "integ": integ, "center": center}


def _as_state(U: np.ndarray, cfg: Config, what="U") -> np.ndarray:
    if U.dtype != np.complex128 or not U.flags.c_contiguous:
        raise ValueError(f"{what} must be a C-contiguous complex128 array")
    if U.shape[1:] != (cfg.nz, cfg.nxh, cfg.ny):
        raise ValueError(f"{what} has shape {U.shape}, expected (nf, {cfg.nz}, {cfg.nxh}, {cfg.ny})")
    return U


class Channel:
    """One channel resident in HBM on one GPU (the GPU half of the drop-in boundary)."""

    def __init__(self, config: Config | None = None, **overrides):
        cfg = config or Config()
        for k, v in overrides.items():
            setattr(cfg, k, v)
        self.config = cfg
        self._lib = _lib.load()
        h = C.c_void_p()
        c = cfg.to_c()
        check(self._lib.kmm_create(C.byref(c), C.byref(h)))
        self._h = h
        info = KmmInfo()
        check(self._lib.kmm_get_info(self._h, C.byref(info)))
        self.info = info
        self.bw = info.bw
        n = cfg.ny
        ld = 2 * self.bw + 1
        self.y = np.zeros(n)
        self.integ = np.zeros(n)
        self.D0, self.D1, self.D2, self.D0_lu = (np.zeros((n, ld)) for _ in range(4))
        check(self._lib.kmm_get_operators(self._h, _dptr(self.y), _dptr(self.integ), _dptr(self.D0),
                                          _dptr(self.D1), _dptr(self.D2), _dptr(self.D0_lu)))
        # (ny, ld) C order = Fortran (ld, ny): present as [r, j] like the reference's A(r, j)
        self.D0, self.D1, self.D2, self.D0_lu = (a.T.copy() for a in (self.D0, self.D1, self.D2, self.D0_lu))

    # -- lifetime ---------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            self._lib.kmm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- state ------------------------------------------------------------------------
    def set_initial_data_uvw(self, U: np.ndarray, dt: float = 0.0):
        U = _as_state(U, self.config)
        check(self._lib.kmm_set_initial_data_uvw(self._h, _dptr(U), U.shape[0], dt))

    def upload_state(self, U: np.ndarray, RK: np.ndarray, dt: float):
        U = _as_state(U, self.config)
        RK = _as_state(RK, self.config, "RK")
        check(self._lib.kmm_upload_state(self._h, _dptr(U), U.shape[0], _dptr(RK), dt))

    @property
    def nstores(self) -> int:
        """RK stores: 3, plus one for a second passive scalar."""
        return 3 + (1 if self.config.n_scalar == 2 else 0)

    def download_state(self, nf: int | None = None):
        cfg = self.config
        if nf is None:
            nf = NFIELD if cfg.n_scalar != 2 else 11
        U = np.zeros((nf, cfg.nz, cfg.nxh, cfg.ny), dtype=np.complex128)
        RK = np.zeros((self.nstores, cfg.nz, cfg.nxh, cfg.ny), dtype=np.complex128)
        check(self._lib.kmm_download_state(self._h, _dptr(U), nf, _dptr(RK)))
        return U, RK

    def get_pressure(self) -> np.ndarray:
        """get_pressure.f90:1-137 for the current state: the pressure U(:,:,:,6) of the
        reference, (nz, nxh, ny) complex128 (kmm_get_pressure)."""
        cfg = self.config
        P = np.zeros((cfg.nz, cfg.nxh, cfg.ny), dtype=np.complex128)
        check(self._lib.kmm_get_pressure(self._h, _dptr(P)))
        return P

    def get_statistics(self, pressure: bool = False, download: bool = True) -> dict | None:
        """The statistics of a statistics step of the current state (kmm_get_statistics:
        get_statistics_1, write_spectra, the physical moments of dft_x_realspace and
        get_statistics_2).  Returns {"lines": {name: (ny,)}, "spec_kx": {name: (nxh, ny)},
        "spec_kz": {name: (nz, ny)}, "U_c", "T_c"} with the reference's dataset names (spectrum
        "uu" is "Euu_kx" / "Euu_kz" there), plus "P" (nz, nxh, ny) when pressure is set.
        With download=False the numbers are computed and left on the device (None returned)."""
        if not download:
            check(self._lib.kmm_get_statistics(self._h, None, None, None, None, None))
            return None
        cfg = self.config
        nl, nsp = _lib.KMM_STAT_NLINES, _lib.KMM_STAT_NSPEC
        lines = np.zeros((nl, cfg.ny))
        skx = np.zeros((nsp, cfg.nxh, cfg.ny))
        skz = np.zeros((nsp, cfg.nz, cfg.ny))
        centre = np.zeros(2)
        P = np.zeros((cfg.nz, cfg.nxh, cfg.ny), dtype=np.complex128) if pressure else None
        check(self._lib.kmm_get_statistics(self._h, _dptr(lines), _dptr(skx), _dptr(skz), _dptr(centre),
                                           _dptr(P) if pressure else None))
        lnames = [self._lib.kmm_stat_line_name(i).decode() for i in range(nl)]
        snames = [self._lib.kmm_stat_spec_name(i).decode() for i in range(nsp)]
        out = {"lines": dict(zip(lnames, lines)), "spec_kx": dict(zip(snames, skx)),
               "spec_kz": dict(zip(snames, skz)), "U_c": float(centre[0]), "T_c": float(centre[1])}
        if pressure:
            out["P"] = P
        return out

    @property
    def dt(self) -> float:
        d = C.c_double()
        check(self._lib.kmm_get_dt(self._h, C.byref(d)))
        return d.value

    @dt.setter
    def dt(self, value: float):
        check(self._lib.kmm_set_dt(self._h, float(value)))

    def set_control_gains(self, gains: np.ndarray | None):
        if gains is None:
            check(self._lib.kmm_set_control_gains(self._h, None))
            return
        g = np.ascontiguousarray(gains, dtype=np.float32)
        if g.shape != (self.config.nz, self.config.nxh):
            raise ValueError("gains must have shape (nz, nxh)")
        check(self._lib.kmm_set_control_gains(self._h, g.ctypes.data_as(C.POINTER(C.c_float))))

    def set_control(self, amp: float, gains: np.ndarray | None = None, y_d: float | None = None):
        """kmm_set_control: opposition amplitude, per-mode gains (nz, nxh) or None (= 1), and the
        detection plane y_d (default: the configured one)."""
        yd = self.config.control_yd if y_d is None else float(y_d)
        gp = None
        if gains is not None:
            g = np.ascontiguousarray(gains, dtype=np.float32)
            if g.shape != (self.config.nz, self.config.nxh):
                raise ValueError("gains must have shape (nz, nxh)")
            gp = g.ctypes.data_as(C.POINTER(C.c_float))
        check(self._lib.kmm_set_control(self._h, float(amp), gp, yd))
        self.config.control_amp = float(amp)
        if amp != 0.0:
            self.config.control_yd = yd

    # -- launch shapes ------------------------------------------------------------------
    def autotune(self) -> dict:
        """kmm_autotune: time the candidate launch shapes on this grid, keep the fastest."""
        t = KmmTuning()
        check(self._lib.kmm_autotune(self._h, C.byref(t)))
        return t.as_dict()

    @property
    def tuning(self) -> dict:
        t = KmmTuning()
        check(self._lib.kmm_get_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **shapes):
        """kmm_set_tuning: pin launch shapes (z_lines_per_block, x_rows_per_block, x_threads,
        modes_per_block, u_layout, assemble_threads, tables_shared, helm_modes_per_block,
        helm_tables_shared, helm_stage_ahead, z_tma, hvhg_stage_ahead, factor_cache); unnamed ones
        keep their current values."""
        t = KmmTuning()
        check(self._lib.kmm_get_tuning(self._h, C.byref(t)))
        for k, v in shapes.items():
            setattr(t, k, int(v))
        check(self._lib.kmm_set_tuning(self._h, C.byref(t)))

    # -- discrete adjoint of the control objective -------------------------------------
    def adjoint_forward(self, nsteps: int, w_tau: float = 1.0, w_q: float = 0.0) -> float:
        """kmm_adjoint_forward: nsteps RK3 steps from the current state with one checkpoint per
        step; returns J = (w_tau tau_w + w_q q_w) averaged over the steps."""
        J = C.c_double()
        check(self._lib.kmm_adjoint_forward(self._h, int(nsteps), float(w_tau), float(w_q), C.byref(J)))
        return J.value

    def adjoint_backward(self):
        """kmm_adjoint_backward: (dJ/dA, dJ/dgains of shape (nz, nxh)) for the recorded steps."""
        dA = C.c_double()
        dg = np.zeros((self.config.nz, self.config.nxh))
        check(self._lib.kmm_adjoint_backward(self._h, C.byref(dA), _dptr(dg)))
        return dA.value, dg

    def data_store(self, path: str, timestep: int = 0, time: float = 0.0, fields: int = _lib.KMM_STORE_ALL):
        """kmm_data_store (data_store.f90:11-173): the state and the problem definition as a restart
        file in the reference's HDF5 layout; timestep and time are the driver's counters."""
        check(self._lib.kmm_data_store(self._h, str(path).encode(), int(timestep), float(time), int(fields)))

    def restart(self, path: str, option: int = 1) -> dict:
        """kmm_restart (initial_step.f90:15-56, 184-513): the state from a restart file with
        restart_option 1 (u, v, w, theta), 2 (g, phi, theta + mean profiles) or 3 (v, g, theta +
        mean profiles); returns the file's timestep, time and dt (the handle's dt becomes it)."""
        info = _lib.KmmRestartInfo()
        check(self._lib.kmm_restart(self._h, str(path).encode(), int(option), C.byref(info)))
        return {"timestep": info.timestep, "time": info.time, "dt": info.dt}

    def adjoint_release(self):
        check(self._lib.kmm_adjoint_release(self._h))

    # -- time stepping ----------------------------------------------------------------
    def time_march(self, rk_substep: int) -> dict:
        s = KmmScalars()
        check(self._lib.kmm_time_march(self._h, int(rk_substep), C.byref(s)))
        return s.as_dict()

    def step(self, nsteps: int = 1) -> dict:
        s = KmmScalars()
        check(self._lib.kmm_step(self._h, int(nsteps), C.byref(s)))
        return s.as_dict()

    def step_async(self, nsteps: int = 1):
        check(self._lib.kmm_step_async(self._h, int(nsteps)))

    def sync(self) -> dict:
        s = KmmScalars()
        check(self._lib.kmm_sync(self._h, C.byref(s)))
        return s.as_dict()

    def step_host_ptr(self, u_ptr: int, nf: int, rk_ptr: int | None, nsteps: int = 1) -> dict:
        """kmm_step_host on raw host pointers (e.g. pinned torch tensors).  rk_ptr None (or 0):
        RK_STORE is rebuilt from U on the device (restart option 1) and only U is transferred."""
        s = KmmScalars()
        rk = C.cast(rk_ptr, C.POINTER(C.c_double)) if rk_ptr else None
        check(self._lib.kmm_step_host(self._h, C.cast(u_ptr, C.POINTER(C.c_double)), nf, rk,
                                      int(nsteps), C.byref(s)))
        return s.as_dict()

    def step_host(self, U: np.ndarray, RK: np.ndarray | None, nsteps: int = 1) -> dict:
        U = _as_state(U, self.config)
        if RK is None:
            return self.step_host_ptr(U.ctypes.data, U.shape[0], None, nsteps)
        RK = _as_state(RK, self.config, "RK")
        return self.step_host_ptr(U.ctypes.data, U.shape[0], RK.ctypes.data, nsteps)

    @property
    def stream_ptr(self) -> int:
        """cudaStream_t of the handle (all its launches go there)."""
        st = C.c_void_p()
        check(self._lib.kmm_get_stream(self._h, C.byref(st)))
        return st.value or 0

    def profile_step(self, nsteps: int = 1) -> dict:
        """Per-kernel mean device time (ms) and launch counts over nsteps unfused steps."""
        ms = (C.c_double * _lib.KMM_NKERNEL)()
        cnt = (C.c_int * _lib.KMM_NKERNEL)()
        check(self._lib.kmm_profile_step(self._h, int(nsteps), ms, cnt))
        return {name: {"ms": ms[i], "launches": cnt[i]} for i, name in enumerate(_lib.KERNEL_NAMES)}

    # -- device building blocks (torch CUDA tensors, reference layouts) ------------------
    @staticmethod
    def _stream():
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def y_to_x(self, u, xp):
        """y_to_x.f90:21-50 for one field: u (nz, nxh, ny) complex128 -> xp (ny, nz32, nxh)."""
        check(self._lib.kmm_dev_y_to_x(self._h, C.c_void_p(u.data_ptr()), C.c_void_p(xp.data_ptr()),
                                       self._stream()))

    def x_to_y(self, xp, u, rescale: bool = True):
        """x_to_y.f90:21-46 (+ rescale_data) for one field."""
        check(self._lib.kmm_dev_x_to_y(self._h, C.c_void_p(xp.data_ptr()), C.c_void_p(u.data_ptr()),
                                       int(bool(rescale)), self._stream()))

    def dft_x_realspace(self, xp10, rk_substep: int, velmax=None):
        """dft_x_realspace.f90:68-213 on a 10-slot X-pencil tensor (10, ny, nz32, nxh)."""
        vp = C.c_void_p(velmax.data_ptr()) if velmax is not None else C.c_void_p()
        check(self._lib.kmm_dev_dft_x_realspace(self._h, C.c_void_p(xp10.data_ptr()), int(rk_substep),
                                                vp, self._stream()))

    def wavespace(self, U10, RK, rk_substep: int, dt: float) -> dict:
        """wavespace.f90:22-113 on device tensors U (10, nz, nxh, ny) and RK (3, nz, nxh, ny)."""
        s = KmmScalars()
        check(self._lib.kmm_dev_wavespace(self._h, C.c_void_p(U10.data_ptr()), C.c_void_p(RK.data_ptr()),
                                          int(rk_substep), float(dt), C.byref(s), self._stream()))
        return s.as_dict()

    def labs_lu(self, a_modes):
        check(self._lib.kmm_dev_labs_lu(self._h, C.c_void_p(a_modes.data_ptr()), a_modes.shape[-1],
                                        self._stream()))

    def labs_bs(self, a_modes, b):
        check(self._lib.kmm_dev_labs_bs(self._h, C.c_void_p(a_modes.data_ptr()), C.c_void_p(b.data_ptr()),
                                        b.shape[-1], self._stream()))

    def labs_mat_mul(self, which: int, x, b):
        check(self._lib.kmm_dev_labs_mat_mul(self._h, int(which), C.c_void_p(x.data_ptr()),
                                             C.c_void_p(b.data_ptr()), x.shape[-1], self._stream()))


def ensemble_step(channels, nsteps: int = 1) -> list[dict]:
    """kmm_ensemble_step: nsteps RK3 steps of every channel, each channel's graph launches
    enqueued on its own stream before any is waited on, so independent channels of any sizes
    run side by side on the GPU.  Returns each channel's diagnostics of its last step."""
    chans = list(channels)
    if len({id(c) for c in chans}) != len(chans):
        raise ValueError("ensemble_step: a channel appears twice")
    n = len(chans)
    hs = (C.c_void_p * max(n, 1))(*[c._h for c in chans])
    outs = (KmmScalars * max(n, 1))()
    check(chans[0]._lib.kmm_ensemble_step(hs, n, int(nsteps), outs) if n else 0)
    return [outs[i].as_dict() for i in range(n)]


__all__ = ["Config", "Channel", "KmmError", "read_input_file", "labs_fill_full", "NFIELD", "ensemble_step"]
