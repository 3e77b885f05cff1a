"""The reference's per-mode routines as batched device entry points (kmm_dev_hvhg,
kmm_dev_solve_g, kmm_dev_solve_t, kmm_dev_solve_v_f, kmm_dev_solve_u_w) against the oracle's
restatements of hvhg.f90, solve_g.f90, solve_t.f90, solve_v_f.f90 and solve_u_w.f90, through the
C ABI, on random lines of many modes at every substep.  Both sides run the routines in the
reference's statement order in FP64, so they agree to rounding (1e-13 relative L2)."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from channel_passive_b200 import Channel, Config
from channel_passive_b200 import _lib
from oracle import kmm as okmm
from tests.helpers import make_pair, rel_l2

pytestmark = pytest.mark.gpu
DEV = "cuda:0"
NM = 500


def _p(t):
    return C.c_void_p(t.data_ptr())


def _lines(a):
    """numpy (ny, nm) complex -> device, mode fastest (value y of mode m at y * nm + m)."""
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _setup(seed):
    cfg, p = make_pair(nx=16, ny=33, nz=16)
    ops = okmm.make_operators(p)
    rng = np.random.default_rng(seed)
    kx = rng.integers(0, 8, NM) / p.lmfx
    kz = rng.integers(-8, 9, NM) / p.lmfz
    kx[kx == 0] += 1.0  # no (0, 0) mode: its k^2 is zero

    def rl():
        return rng.standard_normal((p.ny, NM)) + 1j * rng.standard_normal((p.ny, NM))

    return cfg, p, ops, kx, kz, rl


def _bands(ch):
    # (ld, ny) numpy [r, j] -> Fortran (2bw+1, ny): C-order (ny, ld)
    return [torch.from_numpy(np.ascontiguousarray(b.T)).to(DEV) for b in (ch.D0_lu, ch.D0, ch.D1, ch.D2)]


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_hvhg_matches_oracle():
    cfg, p, ops, kx, kz, rl = _setup(1)
    lib = _lib.load()
    u = [rl() for _ in range(8)]
    ref = okmm.hvhg(*u, ops, kx, kz)
    with Channel(cfg) as ch:
        d0lu, d0, d1, d2 = _bands(ch)
        du = [_lines(a) for a in u]
        kxd, kzd = torch.from_numpy(kx).to(DEV), torch.from_numpy(kz).to(DEV)
        _lib.check(lib.kmm_dev_hvhg(ch._h, *[_p(t) for t in du], _p(d0lu), _p(d1), _p(d2), _p(kxd), _p(kzd),
                                    cfg.nx32, cfg.nz32, NM, _stream()))
        torch.cuda.synchronize()
        got = [t.cpu().numpy() for t in du]
    for name, g, r in (("hg", got[0], ref[0]), ("hv", got[4], ref[1]), ("ht", got[5], ref[2])):
        assert rel_l2(g, r) < 1e-13, name


@pytest.mark.parametrize("substep", [1, 2, 3])
@pytest.mark.parametrize("scalar", [False, True])
def test_solve_g_and_t_match_oracle(substep, scalar):
    cfg, p, ops, kx, kz, rl = _setup(10 + substep)
    lib = _lib.load()
    h, store = rl(), rl()
    dt = 0.013
    diff = (p.nu, p.pr) if scalar else (p.nu, None)
    u_ref, store_ref, dbuf_ref = okmm.solve_scalar_helmholtz(h, store.copy(), ops, kx, kz, diff, substep, dt)
    with Channel(cfg) as ch:
        d0lu, d0, d1, d2 = _bands(ch)
        du, ds = _lines(h), _lines(store)
        b1, b2 = torch.zeros_like(du), torch.zeros_like(du)
        dbuf = torch.zeros((p.ny, 2 * ch.bw + 1, NM), dtype=torch.float64, device=DEV)
        kxd, kzd = torch.from_numpy(kx).to(DEV), torch.from_numpy(kz).to(DEV)
        if scalar:
            rc = lib.kmm_dev_solve_t(ch._h, _p(du), _p(ds), _p(b1), _p(b2), _p(d0lu), _p(d0), _p(d2), _p(dbuf),
                                     _p(kxd), _p(kzd), p.nu, p.pr, p.ny, substep, dt, NM, _stream())
        else:
            rc = lib.kmm_dev_solve_g(ch._h, _p(du), _p(ds), _p(b1), _p(b2), _p(d0lu), _p(d0), _p(d2), _p(dbuf),
                                     _p(kxd), _p(kzd), p.nu, p.ny, substep, dt, NM, _stream())
        _lib.check(rc)
        torch.cuda.synchronize()
        assert rel_l2(du.cpu().numpy(), u_ref) < 1e-13
        assert rel_l2(ds.cpu().numpy(), store_ref) < 1e-13
        # D_buf: (ld, ny, nm) per the oracle, [j][r][m] here
        assert rel_l2(np.transpose(dbuf.cpu().numpy(), (1, 0, 2)), dbuf_ref) < 1e-14


@pytest.mark.parametrize("substep", [1, 2, 3])
@pytest.mark.parametrize("with_wall", [False, True])
def test_solve_v_f_and_u_w_match_oracle(substep, with_wall):
    cfg, p, ops, kx, kz, rl = _setup(20 + substep)
    lib = _lib.load()
    hv, sp, g = rl(), rl(), rl()
    dt = 0.011
    rng = np.random.default_rng(3)
    vwall = (rng.standard_normal((2, NM)) + 1j * rng.standard_normal((2, NM))) if with_wall else None
    # solve_g first: its factors are solve_v_f's input
    _, _, dbuf_g = okmm.solve_scalar_helmholtz(rl(), rl(), ops, kx, kz, (p.nu, None), substep, dt)
    v_ref, dv_ref, sp_ref = okmm.solve_v_f(hv, sp.copy(), None, ops, dbuf_g, kx, kz, p.nu, substep, dt, vwall)
    u_ref, w_ref = okmm.solve_u_w(g, dv_ref, kx, kz)
    with Channel(cfg) as ch:
        d0lu, d0, d1, d2 = _bands(ch)
        dhv, dsp = _lines(hv), _lines(sp)
        v, dv, b1, b2, b3 = (torch.zeros_like(dhv) for _ in range(5))
        dbuf = torch.from_numpy(np.ascontiguousarray(np.transpose(dbuf_g, (1, 0, 2)))).to(DEV)
        kxd, kzd = torch.from_numpy(kx).to(DEV), torch.from_numpy(kz).to(DEV)
        vw = _lines(vwall) if with_wall else None
        _lib.check(lib.kmm_dev_solve_v_f(ch._h, _p(v), _p(dv), _p(dhv), _p(dsp), _p(b1), _p(b2), _p(b3), None,
                                         _p(d0lu), _p(d0), _p(d1), _p(d2), _p(dbuf), _p(kxd), _p(kzd), p.nu,
                                         p.ny, substep, dt, _p(vw) if with_wall else None, NM, _stream()))
        dg = _lines(g)
        _lib.check(lib.kmm_dev_solve_u_w(ch._h, _p(dg), _p(dv), _p(kxd), _p(kzd), NM, _stream()))
        torch.cuda.synchronize()
        assert rel_l2(v.cpu().numpy(), v_ref) < 1e-12
        assert rel_l2(dsp.cpu().numpy(), sp_ref) < 1e-12
        assert rel_l2(dg.cpu().numpy(), u_ref) < 1e-12
        assert rel_l2(dv.cpu().numpy(), w_ref) < 1e-12


def test_routines_reject_bad_arguments():
    lib = _lib.load()
    with Channel(Config(nx=8, ny=33, nz=8)) as ch:
        x = torch.zeros((33, 4), dtype=torch.complex128, device=DEV)
        k = torch.ones(4, dtype=torch.float64, device=DEV)
        bd = torch.zeros((33, 2 * ch.bw + 1), dtype=torch.float64, device=DEV)
        db = torch.zeros((33, 2 * ch.bw + 1, 4), dtype=torch.float64, device=DEV)
        args = [_p(x), _p(x), _p(x), _p(x), _p(bd), _p(bd), _p(bd), _p(db), _p(k), _p(k), 1e-3]
        assert lib.kmm_dev_solve_g(ch._h, *args, 34, 1, 0.01, 4, None) == _lib.KMM_ERR_ARG      # ny mismatch
        assert lib.kmm_dev_solve_g(ch._h, *args, 33, 4, 0.01, 4, None) == _lib.KMM_ERR_ARG      # bad substep
        assert lib.kmm_dev_solve_g(ch._h, *args, 33, 1, 0.01, 0, None) == _lib.KMM_ERR_ARG      # no modes
        odd = C.c_void_p(x.data_ptr() + 8)
        assert lib.kmm_dev_solve_u_w(ch._h, odd, _p(x), _p(k), _p(k), 4, None) == _lib.KMM_ERR_ARG
