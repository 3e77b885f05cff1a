"""The C-ABI library: loads, exports every symbol include/kmm.h declares, host-side entry
points (operator builder, input parser, configuration checks).  No GPU compute here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from channel_passive_b200 import Config, KmmError, labs_fill_full, read_input_file
from channel_passive_b200 import _lib
from oracle import bspline

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    txt = open(os.path.join(ROOT, "include", "kmm.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(kmm_\w+)\s*\(", txt)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
        assert n in _lib.SIGNATURES, f"{n} has no ctypes signature"


def test_config_struct_layout():
    c = _lib.KmmConfig()
    assert C.sizeof(c) == 192
    assert _lib.KmmConfig.control_yd.offset == 152
    lib = _lib.load()
    assert lib.kmm_config_default(C.byref(c)) == 0
    assert (c.nx, c.ny, c.nz, c.no_of_field, c.rk_scheme, c.labs_k) == (64, 65, 64, 10, 3, 6)


@pytest.mark.parametrize("k,n,stretch", [(7, 32, 0.0), (7, 32, 0.99), (7, 129, 0.9), (5, 33, 0.5)])
def test_labs_fill_full_matches_oracle(k, n, stretch):
    a = labs_fill_full(k, n, stretch)
    b = bspline.fill_full(k, n, stretch)
    for d in range(5):
        np.testing.assert_array_equal(a["D"][d], b["D"][d])
    np.testing.assert_array_equal(a["y"], b["y"])
    np.testing.assert_allclose(a["integ"], b["integ"], rtol=0, atol=1e-15)
    np.testing.assert_array_equal(a["center"], b["center"])
    np.testing.assert_array_equal(a["breakpoints"], b["breakpoints"])


def test_labs_fill_full_reference_known_answer():
    for stretch in (0.0, 0.99):
        o = labs_fill_full(7, 32, stretch)
        assert abs(o["integ"].sum() - 2.0) <= 1e-12
        for d in range(5):
            M = o["D"][d]
            scale = 1.0 + np.abs(M).sum(axis=1)
            assert np.all(np.abs(M.sum(axis=1) - (1.0 if d == 0 else 0.0)) <= 1e-11 * scale)


def test_read_input_file():
    cfg = read_input_file(os.path.join(ROOT, "tests", "golden", "input_192x129x192"))
    assert (cfg.nx, cfg.ny, cfg.nz, cfg.no_of_field, cfg.labs_k) == (192, 129, 192, 10, 6)
    assert cfg.lmfx == 2.0 and abs(cfg.lmfz - 2.0 / 3.0) < 1e-15
    assert cfg.nu == pytest.approx(1.0 / 2800.0, rel=1e-15)
    assert cfg.pr == 0.71 and cfg.stretch == 0.9 and cfg.cfl == 1.0


def test_read_input_file_rejects_malformed(tmp_path):
    bad = tmp_path / "input"
    bad.write_text(" nx ny nz no_of_field\n192 129\n")
    with pytest.raises(KmmError) as e:
        read_input_file(str(bad))
    assert e.value.code == _lib.KMM_ERR_CONFIG
    with pytest.raises(KmmError):
        read_input_file(str(tmp_path / "missing"))


@pytest.mark.parametrize("override,msg", [
    (dict(ny=9), "too large"),
    (dict(rk_scheme=4), "Runge-Kutta"),
    (dict(no_of_field=6), "no_of_field"),
    (dict(nx=7), "even"),
    (dict(nx=14), "factor"),
    (dict(nu=-1.0), "positive"),
    (dict(control_amp=-1.0, control_yd=0.5), "y_d"),
    # the per-mode kernels' 32-bit line offsets: 2*bw*nxh*nz*ny must stay below 2^31
    (dict(nx=2048, ny=129, nz=2048), "2^31"),
])
def test_create_rejects_bad_config(override, msg):
    from channel_passive_b200 import Channel
    cfg = Config(nx=16, ny=33, nz=16)
    for k, v in override.items():
        setattr(cfg, k, v)
    with pytest.raises(KmmError) as e:
        Channel(cfg)
    assert e.value.code == _lib.KMM_ERR_CONFIG
    assert msg in str(e.value)


def test_null_arguments_return_status():
    lib = _lib.load()
    assert lib.kmm_create(None, None) == _lib.KMM_ERR_ARG
    assert lib.kmm_time_march(None, 1, None) == _lib.KMM_ERR_ARG
    assert lib.kmm_step_host(None, None, 10, None, 1, None) == _lib.KMM_ERR_ARG
    assert lib.kmm_ensemble_step(None, 1, 1, None) == _lib.KMM_ERR_ARG
    hs = (C.c_void_p * 2)(None, None)
    assert lib.kmm_ensemble_step(hs, 2, 1, None) == _lib.KMM_ERR_ARG
    assert lib.kmm_ensemble_step(hs, 0, 1, None) == 0
    assert lib.kmm_destroy(None) == 0
