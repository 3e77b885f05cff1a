"""ctypes binding of libkmm.so (include/kmm.h).

The shared library is built in tree (``channel_passive_b200/lib/libkmm.so``) by
``channel_passive_b200.build``.  There is no Python or CPU fallback for any
compute entry point: loading fails loudly when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libkmm.so"

KMM_OK = 0
KMM_ERR_CONFIG = 1
KMM_ERR_CUDA = 2
KMM_ERR_DT = 3
KMM_ERR_NONFINITE = 4
KMM_ERR_ARG = 5
KMM_ERR_TIMEOUT = 6
KMM_ERR_IO = 7
KMM_STORE_U, KMM_STORE_V, KMM_STORE_W, KMM_STORE_G, KMM_STORE_PHI, KMM_STORE_THETA = 1, 2, 4, 8, 16, 32
KMM_STORE_ALL = 63

KMM_PREC_FP64 = 0
KMM_PREC_MIXED = 1
KMM_NOALLOC_MAX_DOUBLES = 2097152
KMM_STAT_NLINES = 58
KMM_STAT_NSPEC = 18
KMM_NKERNEL = 8
KERNEL_NAMES = ("begin_substep", "zinv", "xphys", "update_dt", "zfwd", "hvhg", "helmholtz", "assemble")
KMM_GRID_SINE = 0
KMM_GRID_TANH = 1


class KmmConfig(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("no_of_field", C.c_int32), ("rk_scheme", C.c_int32), ("labs_k", C.c_int32),
        ("lmfx", C.c_double), ("lmfy", C.c_double), ("lmfz", C.c_double),
        ("stretch", C.c_double), ("grid", C.c_int32),
        ("nu", C.c_double), ("pr", C.c_double),
        ("bulk_vel_u", C.c_double), ("bulk_vel_w", C.c_double), ("bulk_t", C.c_double),
        ("u_gal", C.c_double), ("cfl", C.c_double), ("dt_factor", C.c_double),
        ("dy_factor", C.c_double), ("fixed_dt", C.c_int32), ("precision", C.c_int32),
        ("control_amp", C.c_double), ("control_yd", C.c_double), ("device", C.c_int32),
        ("n_scalar", C.c_int32), ("pr2", C.c_double), ("bulk_t2", C.c_double),
        ("autotune", C.c_int32), ("reserved", C.c_int32),
    ]


class KmmScalars(C.Structure):
    _fields_ = [
        ("dt", C.c_double), ("velmax", C.c_double),
        ("phi_dpdx", C.c_double * 4), ("phi_dtdx", C.c_double * 4),
        ("wall_shear_stress", C.c_double), ("wall_theta_stress", C.c_double),
        ("phi_dtdx2", C.c_double * 4), ("wall_theta_stress2", C.c_double),
    ]

    def as_dict(self):
        return {"dt": self.dt, "velmax": self.velmax, "phi_dpdx": list(self.phi_dpdx),
                "phi_dtdx": list(self.phi_dtdx), "wall_shear_stress": self.wall_shear_stress,
                "wall_theta_stress": self.wall_theta_stress, "phi_dtdx2": list(self.phi_dtdx2),
                "wall_theta_stress2": self.wall_theta_stress2}


class KmmInfo(C.Structure):
    _fields_ = [
        ("bw", C.c_int32), ("nxh", C.c_int32), ("nx32", C.c_int32), ("nz32", C.c_int32),
        ("nmodes", C.c_int64), ("device_bytes", C.c_int64),
        ("fft_radix_x", C.c_int32 * 8), ("fft_radix_z", C.c_int32 * 8),
    ]


class KmmTuning(C.Structure):
    _fields_ = [
        ("z_lines_per_block", C.c_int32), ("x_rows_per_block", C.c_int32), ("x_threads", C.c_int32),
        ("modes_per_block", C.c_int32), ("u_layout", C.c_int32), ("assemble_threads", C.c_int32),
        ("tuned", C.c_int32), ("tables_shared", C.c_int32),
        ("helm_modes_per_block", C.c_int32), ("helm_tables_shared", C.c_int32), ("helm_stage_ahead", C.c_int32),
        ("z_tma", C.c_int32), ("hvhg_stage_ahead", C.c_int32), ("factor_cache", C.c_int32),
        ("ms_z", C.c_double * 3), ("ms_x", C.c_double * 3), ("ms_modes", C.c_double * 2),
        ("ms_layout", C.c_double * 2), ("ms_assemble", C.c_double * 3), ("ms_tables", C.c_double * 2),
        ("ms_helm", C.c_double * 12), ("ms_z_tma", C.c_double * 3), ("ms_hvhg", C.c_double * 12),
        ("ms_step", C.c_double * 2),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_}
        for k, v in d.items():
            if not isinstance(v, (int, float)):
                d[k] = list(v)
        return d


class KmmRestartInfo(C.Structure):
    _fields_ = [("timestep", C.c_int32), ("reserved", C.c_int32), ("time", C.c_double), ("dt", C.c_double)]


# every symbol include/kmm.h declares, with its ctypes signature
_P = C.c_void_p
_D = C.POINTER(C.c_double)
SIGNATURES = {
    "kmm_last_error": (C.c_char_p, []),
    "kmm_config_default": (C.c_int, [C.POINTER(KmmConfig)]),
    "kmm_read_input_file": (C.c_int, [C.c_char_p, C.POINTER(KmmConfig)]),
    "kmm_create": (C.c_int, [C.POINTER(KmmConfig), C.POINTER(_P)]),
    "kmm_destroy": (C.c_int, [_P]),
    "kmm_get_info": (C.c_int, [_P, C.POINTER(KmmInfo)]),
    "kmm_get_operators": (C.c_int, [_P, _D, _D, _D, _D, _D, _D]),
    "kmm_labs_fill_full": (None, [_D, _D, _D, _D, _D, _D, _D, _D, _D, C.POINTER(C.c_int),
                                  C.POINTER(C.c_int), _D, _D]),
    "kmm_upload_state": (C.c_int, [_P, _D, C.c_int, _D, C.c_double]),
    "kmm_download_state": (C.c_int, [_P, _D, C.c_int, _D]),
    "kmm_set_initial_data_uvw": (C.c_int, [_P, _D, C.c_int, C.c_double]),
    "kmm_time_march": (C.c_int, [_P, C.c_int, C.POINTER(KmmScalars)]),
    "kmm_step": (C.c_int, [_P, C.c_int, C.POINTER(KmmScalars)]),
    "kmm_step_async": (C.c_int, [_P, C.c_int]),
    "kmm_sync": (C.c_int, [_P, C.POINTER(KmmScalars)]),
    "kmm_step_host": (C.c_int, [_P, _D, C.c_int, _D, C.c_int, C.POINTER(KmmScalars)]),
    "kmm_get_stream": (C.c_int, [_P, C.POINTER(_P)]),
    "kmm_get_pressure": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "kmm_ensemble_step": (C.c_int, [C.POINTER(_P), C.c_int, C.c_int, C.POINTER(KmmScalars)]),
    "kmm_get_statistics": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double), C.POINTER(C.c_double),
                                     C.POINTER(C.c_double)]),
    "kmm_stat_line_name": (C.c_char_p, [C.c_int]),
    "kmm_stat_spec_name": (C.c_char_p, [C.c_int]),
    "kmm_profile_step": (C.c_int, [_P, C.c_int, _D, C.POINTER(C.c_int)]),
    "kmm_get_dt": (C.c_int, [_P, _D]),
    "kmm_set_dt": (C.c_int, [_P, C.c_double]),
    "kmm_set_control_gains": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "kmm_set_control": (C.c_int, [_P, C.c_double, C.POINTER(C.c_float), C.c_double]),
    "kmm_dev_y_to_x": (C.c_int, [_P, _P, _P, _P]),
    "kmm_dev_x_to_y": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "kmm_dev_dft_x_realspace": (C.c_int, [_P, _P, C.c_int, _P, _P]),
    "kmm_dev_wavespace": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, C.POINTER(KmmScalars), _P]),
    "kmm_dev_labs_lu": (C.c_int, [_P, _P, C.c_int, _P]),
    "kmm_dev_labs_bs": (C.c_int, [_P, _P, _P, C.c_int, _P]),
    "kmm_dev_labs_mat_mul": (C.c_int, [_P, C.c_int, _P, _P, C.c_int, _P]),
    "kmm_dev_hvhg": (C.c_int, [_P] + [_P] * 8 + [_P] * 3 + [_P, _P, C.c_int64, C.c_int64, C.c_int, _P]),
    "kmm_dev_solve_g": (C.c_int, [_P] + [_P] * 4 + [_P] * 4 + [_P, _P, C.c_double, C.c_int, C.c_int,
                                                             C.c_double, C.c_int, _P]),
    "kmm_dev_solve_t": (C.c_int, [_P] + [_P] * 4 + [_P] * 4 + [_P, _P, C.c_double, C.c_double, C.c_int,
                                                             C.c_int, C.c_double, C.c_int, _P]),
    "kmm_dev_solve_v_f": (C.c_int, [_P] + [_P] * 8 + [_P] * 5 + [_P, _P, C.c_double, C.c_int, C.c_int,
                                                               C.c_double, _P, C.c_int, _P]),
    "kmm_dev_solve_u_w": (C.c_int, [_P, _P, _P, _P, _P, C.c_int, _P]),
    "kmm_adjoint_forward": (C.c_int, [_P, C.c_int, C.c_double, C.c_double, _D]),
    "kmm_adjoint_backward": (C.c_int, [_P, _D, _D]),
    "kmm_adjoint_release": (C.c_int, [_P]),
    "kmm_autotune": (C.c_int, [_P, C.POINTER(KmmTuning)]),
    "kmm_get_tuning": (C.c_int, [_P, C.POINTER(KmmTuning)]),
    "kmm_set_tuning": (C.c_int, [_P, C.POINTER(KmmTuning)]),
    "kmm_helmholtz_solve_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, _P, _P, _P, _P, _P, _P]),
    "kmm_io_create": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(_P)]),
    "kmm_io_open": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(_P)]),
    "kmm_io_close": (C.c_int, [_P]),
    "kmm_io_string_set": (C.c_int, [_P, C.c_char_p, C.c_char_p]),
    "kmm_io_string_get": (C.c_int, [_P, C.c_char_p, C.c_char_p, C.c_int64]),
    "kmm_io_exists": (C.c_int, [_P, C.c_char_p]),
    "kmm_io_line_write_double": (C.c_int, [_P, C.c_char_p, C.c_int64, _D, C.c_char_p]),
    "kmm_io_line_write_integer": (C.c_int, [_P, C.c_char_p, C.c_int64, C.POINTER(C.c_int32), C.c_char_p]),
    "kmm_io_line_read_double": (C.c_int, [_P, C.c_char_p, C.c_int64, C.c_int64, C.c_int64, _D]),
    "kmm_io_line_read_integer": (C.c_int, [_P, C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.POINTER(C.c_int32)]),
    "kmm_io_plane_write_double": (C.c_int, [_P, C.c_char_p, C.c_int64, C.c_int64, _D, C.c_char_p]),
    "kmm_io_plane_read_double": (C.c_int, [_P, C.c_char_p, C.c_int64, C.c_int64, _D]),
    "kmm_io_field_writev_double": (C.c_int, [_P, C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.c_int32, _D]),
    "kmm_io_field_readv_double": (C.c_int, [_P, C.c_char_p, C.c_int64, C.c_int64, C.c_int64, C.c_int32,
                                            C.c_int64, C.c_int64, C.c_int64, C.c_int64, _D]),
    "kmm_io_dataset_write_raw": (C.c_int, [_P, C.c_char_p, C.c_int32, C.POINTER(C.c_int64), C.c_int32, C.c_int32,
                                           _P]),
    "kmm_io_attr_write_integer": (C.c_int, [_P, C.c_char_p, C.c_char_p, C.c_int64, C.POINTER(C.c_int32)]),
    "kmm_io_delete": (C.c_int, [_P, C.c_char_p]),
    "kmm_data_store": (C.c_int, [_P, C.c_char_p, C.c_int32, C.c_double, C.c_int32]),
    "kmm_restart": (C.c_int, [_P, C.c_char_p, C.c_int32, C.POINTER(KmmRestartInfo)]),
}

_lib = None


class KmmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libkmm error {code}: {msg}")
        self.code = code


def load(path: str | os.PathLike | None = None):
    """Load libkmm.so (once).  Raises if the CUDA library has not been built.  The environment
    variable KMM_LIBRARY selects another build of the same ABI (for example one compiled with
    different tuning macros)."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else Path(os.environ.get("KMM_LIBRARY") or LIB_PATH)
    if not p.exists():
        raise RuntimeError(f"libkmm.so not found at {p}; build it with "
                           "`python -m channel_passive_b200.build` (nvcc, sm_100a)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int):
    if rc != KMM_OK:
        raise KmmError(rc, load().kmm_last_error().decode())
    return rc
