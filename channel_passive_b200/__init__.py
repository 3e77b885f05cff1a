"""B200 (sm_100a) implementation of the PoongBack KMM channel RK3 time step with a passive
scalar (yaojieuh/CHANNEL_PASSIVE), behind a C ABI (include/kmm.h) that mirrors the
reference's Fortran routines.

The compute path is libkmm.so (CUDA kernels + C++ operator builder); this package holds
the build recipe, the ctypes binding and a thin host-side mirror of the reference
interface.
"""
from .solver import Channel, Config, KmmError, NFIELD, ensemble_step, labs_fill_full, read_input_file  # noqa: F401
from . import ic  # noqa: F401
from .hdf5_io import IoFile  # noqa: F401
