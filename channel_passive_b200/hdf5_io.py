"""Checkpoint files in the reference's HDF5 layout (kmm_io_* of libkmm), the one-process
counterpart of channel_hdf5_io's io_handle (module_hdf5_io.f90:6-456).

    with IoFile(path, "w") as f:            # io_file_create (overwrite)
        f.string_set("Readme", "...")        # io_string_set on "/"
        f.line_write("time", [0.25], "Simulation time")
        f.field_write("u", U[0])             # U[f] is (nz, nxh, ny) complex, the package's layout
    with IoFile(path) as f:                  # io_file_open, read-only
        t = f.line_read("time", 1)[0]
        u = f.field_read("u", ny, nxh, nz)

Modes: "r" read-only, "r+" read and update (written again on close), "w" create or overwrite,
"x" create, refusing an existing file.  Reads check rank, shape and element type the way the
reference's transfer() does and raise KmmError(KMM_ERR_IO) with its message.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check


def _b(s: str) -> bytes:
    return s.encode()


class IoFile:
    def __init__(self, path: str, mode: str = "r"):
        self._lib = _lib.load()
        self._io = C.c_void_p()
        p = _b(str(path))
        if mode in ("w", "x"):
            check(self._lib.kmm_io_create(p, 1 if mode == "w" else 0, C.byref(self._io)))
        elif mode in ("r", "r+"):
            check(self._lib.kmm_io_open(p, 1 if mode == "r+" else 0, C.byref(self._io)))
        else:
            raise ValueError(f"mode {mode!r}: expected r, r+, w or x")

    def close(self):
        if self._io:
            io, self._io = self._io, C.c_void_p()
            check(self._lib.kmm_io_close(io))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # attributes and names
    def string_set(self, name: str, value: str):
        check(self._lib.kmm_io_string_set(self._io, _b(name), _b(value)))

    def string_get(self, name: str, maxlen: int = 4096) -> str:
        buf = C.create_string_buffer(maxlen)
        check(self._lib.kmm_io_string_get(self._io, _b(name), buf, maxlen))
        return buf.value.decode()

    def exists(self, name: str) -> bool:
        return self._lib.kmm_io_exists(self._io, _b(name)) == 1

    def delete(self, name: str):
        check(self._lib.kmm_io_delete(self._io, _b(name)))

    # lines
    def line_write(self, name: str, values, comment: str | None = None):
        v = np.ascontiguousarray(values)
        cm = _b(comment) if comment else None
        if np.issubdtype(v.dtype, np.integer):
            v = np.ascontiguousarray(v, dtype=np.int32)
            check(self._lib.kmm_io_line_write_integer(self._io, _b(name), v.size,
                                                      v.ctypes.data_as(C.POINTER(C.c_int32)), cm))
        else:
            v = np.ascontiguousarray(v, dtype=np.float64)
            check(self._lib.kmm_io_line_write_double(self._io, _b(name), v.size,
                                                     v.ctypes.data_as(C.POINTER(C.c_double)), cm))

    def line_read(self, name: str, n: int, dtype=np.float64, start: int = 0, count: int | None = None):
        count = n - start if count is None else count
        out = np.zeros(max(count, 1), dtype=np.int32 if np.issubdtype(np.dtype(dtype), np.integer) else np.float64)
        if out.dtype == np.int32:
            check(self._lib.kmm_io_line_read_integer(self._io, _b(name), n, start, count,
                                                     out.ctypes.data_as(C.POINTER(C.c_int32))))
        else:
            check(self._lib.kmm_io_line_read_double(self._io, _b(name), n, start, count,
                                                    out.ctypes.data_as(C.POINTER(C.c_double))))
        return out[:count]

    # planes: Fortran (na, nb), i.e. numpy (nb, na)
    def plane_write(self, name: str, plane, comment: str | None = None):
        p = np.ascontiguousarray(plane, dtype=np.float64)
        nb, na = p.shape
        check(self._lib.kmm_io_plane_write_double(self._io, _b(name), na, nb, p.ctypes.data_as(C.POINTER(C.c_double)),
                                                  _b(comment) if comment else None))

    def plane_read(self, name: str, na: int, nb: int):
        out = np.zeros((nb, na))
        check(self._lib.kmm_io_plane_read_double(self._io, _b(name), na, nb, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    # fields: (nz, nxh, ny) complex, the memory order of Fortran (2, ny, nxh, nz)
    def field_write(self, name: str, field):
        f = np.ascontiguousarray(field, dtype=np.complex128)
        nz, nxh, ny = f.shape
        check(self._lib.kmm_io_field_writev_double(self._io, _b(name), ny, nxh, nz, 2,
                                                   f.ctypes.data_as(C.POINTER(C.c_double))))

    def field_read(self, name: str, ny: int, nxh: int, nz: int, x=(0, None), z=(0, None)):
        x0, xn = x[0], (nxh - x[0] if x[1] is None else x[1])
        z0, zn = z[0], (nz - z[0] if z[1] is None else z[1])
        out = np.zeros((zn, xn, ny), dtype=np.complex128)
        ptr = out.ctypes.data_as(C.POINTER(C.c_double)) if out.size else None
        check(self._lib.kmm_io_field_readv_double(self._io, _b(name), ny, nxh, nz, 2, x0, xn, z0, zn, ptr))
        return out

    # anything else: a C-order array of float64 (ncomp > 1: the last axis becomes an HDF5 array)
    # or int32, and int32 dataset attributes
    def write_raw(self, name: str, data, ncomp: int = 1):
        a = np.ascontiguousarray(data)
        kind = 1 if np.issubdtype(a.dtype, np.integer) else 0
        a = np.ascontiguousarray(a, dtype=np.int32 if kind else np.float64)
        dims = a.shape[:-1] if ncomp > 1 else a.shape
        if ncomp > 1 and a.shape[-1] != ncomp:
            raise ValueError("the last axis must hold the ncomp components")
        cd = (C.c_int64 * max(len(dims), 1))(*dims)
        check(self._lib.kmm_io_dataset_write_raw(self._io, _b(name), len(dims), cd, kind, ncomp,
                                                 a.ctypes.data_as(C.c_void_p)))

    def attr_write_int(self, dataset: str, name: str, values):
        v = np.ascontiguousarray(values, dtype=np.int32)
        check(self._lib.kmm_io_attr_write_integer(self._io, _b(dataset), _b(name), v.size,
                                                  v.ctypes.data_as(C.POINTER(C.c_int32))))
