"""The allocation-free Helmholtz solve (kmm_helmholtz_solve_noalloc) against the existing
handle-based path (kmm_dev_labs_lu + kmm_dev_labs_bs on a caller-built band) and against the
oracle's packed-band LU and substitution, through the C ABI.

The new entry point serves callers that may not allocate device memory (stream capture in
progress, device memory reserved by another allocator, no tolerance for cudaMalloc's
synchronisation); its scratch is a fixed array inside the library.  Two calls in a row must
each match the existing path, and an oversize request must be refused before any launch.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from channel_passive_b200 import Channel, Config
from channel_passive_b200 import _lib

pytestmark = pytest.mark.gpu
DEV = "cuda:0"


def _dirichlet_bands(ch, a, b):
    """(ld, ny, nm) bands a*D0 - b*D2 with the Dirichlet first/last rows (numpy, host)."""
    bw = ch.bw
    A = a[None, None] * ch.D0[..., None] - b[None, None] * ch.D2[..., None]
    for col in (0, -1):
        diag = a * ch.D0[bw, col] - b * ch.D2[bw, col]
        A[:, col] = 0.0
        A[bw, col] = diag
    return A


def _existing_path(ch, a, b, rhs):
    A = _dirichlet_bands(ch, a, b)
    a_dev = torch.from_numpy(np.ascontiguousarray(np.transpose(A, (1, 0, 2)))).to(DEV)
    x = torch.from_numpy(rhs.copy()).to(DEV)
    ch.labs_lu(a_dev)
    ch.labs_bs(a_dev, x)
    torch.cuda.synchronize()
    return x.cpu().numpy()


def test_noalloc_matches_existing_path_two_calls():
    lib = _lib.load()
    cfg = Config(nx=8, ny=65, nz=8)
    with Channel(cfg) as ch:
        ny, bw = cfg.ny, ch.bw
        nm = 300
        d0 = torch.from_numpy(np.ascontiguousarray(ch.D0.T)).to(DEV)  # (ny, ld) = Fortran (ld, ny)
        d2 = torch.from_numpy(np.ascontiguousarray(ch.D2.T)).to(DEV)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rng = np.random.default_rng(42)
        for call in range(2):
            a = 1.0 + rng.random(nm)
            b = 0.05 * rng.random(nm) * (call + 1)
            rhs = rng.standard_normal((ny, nm)) + 1j * rng.standard_normal((ny, nm))
            ref = _existing_path(ch, a, b, rhs)
            a_d = torch.from_numpy(a).to(DEV)
            b_d = torch.from_numpy(b).to(DEV)
            x = torch.from_numpy(rhs.copy()).to(DEV)
            rc = lib.kmm_helmholtz_solve_noalloc(ny, bw, nm, C.c_void_p(d0.data_ptr()),
                                                 C.c_void_p(d2.data_ptr()), C.c_void_p(a_d.data_ptr()),
                                                 C.c_void_p(b_d.data_ptr()), C.c_void_p(x.data_ptr()), stream)
            assert rc == 0, lib.kmm_last_error().decode()
            torch.cuda.synchronize()
            got = x.cpu().numpy()
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err < 1e-13, (call, err)


def test_noalloc_matches_oracle():
    """Against the oracle directly: per mode the band a D0 - b D2 with the Dirichlet first and last
    rows, factored and solved by oracle/labs.py (fixed_bandec / fixed_banbks in the reference's
    loop order, module_labs.f90:3487-3636, 4252-4318), on the oracle's own operators."""
    from oracle import kmm as okmm
    from oracle import labs as olabs
    from tests.helpers import make_pair

    lib = _lib.load()
    cfg, p = make_pair(nx=8, ny=65, nz=8)
    ops = okmm.make_operators(p)
    with Channel(cfg) as ch:
        ny, bw = cfg.ny, ch.bw
        assert bw == ops.bw and np.array_equal(ch.D0, ops.D0) and np.array_equal(ch.D2, ops.D2)
        nm = 64
        rng = np.random.default_rng(7)
        a = 1.0 + rng.random(nm)
        b = 0.02 * rng.random(nm)
        rhs = rng.standard_normal((ny, nm)) + 1j * rng.standard_normal((ny, nm))
        want = np.empty_like(rhs)
        for m in range(nm):
            A = a[m] * ops.D0 - b[m] * ops.D2
            for col in (0, ny - 1):
                diag = A[bw, col]
                A[:, col] = 0.0
                A[bw, col] = diag
            want[:, m] = olabs.bs(olabs.lu(A), rhs[:, m])
        d0 = torch.from_numpy(np.ascontiguousarray(ch.D0.T)).to(DEV)
        d2 = torch.from_numpy(np.ascontiguousarray(ch.D2.T)).to(DEV)
        a_d, b_d = torch.from_numpy(a).to(DEV), torch.from_numpy(b).to(DEV)
        x = torch.from_numpy(rhs.copy()).to(DEV)
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = lib.kmm_helmholtz_solve_noalloc(ny, bw, nm, C.c_void_p(d0.data_ptr()), C.c_void_p(d2.data_ptr()),
                                             C.c_void_p(a_d.data_ptr()), C.c_void_p(b_d.data_ptr()),
                                             C.c_void_p(x.data_ptr()), stream)
        assert rc == 0, lib.kmm_last_error().decode()
        torch.cuda.synchronize()
        got = x.cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < 1e-13


def test_noalloc_rejects_oversize_request():
    lib = _lib.load()
    ny, bw = 129, 4
    nm = _lib.KMM_NOALLOC_MAX_DOUBLES // ((2 * bw + 1) * ny) + 1
    dummy = torch.zeros(1, dtype=torch.float64, device=DEV)
    p = C.c_void_p(dummy.data_ptr())
    rc = lib.kmm_helmholtz_solve_noalloc(ny, bw, nm, p, p, p, p, p, C.c_void_p(0))
    assert rc == _lib.KMM_ERR_ARG
    assert "exceeds" in lib.kmm_last_error().decode()
