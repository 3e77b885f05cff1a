"""Checkpoint files (kmm_io_*, channel_passive_b200.hdf5_io): the library's HDF5 reader and writer
against the reference's own I/O test (tests/io/run_io_tests.py, io_roundtrip.f90 of the
reference).

* Known answers of the legacy fixtures (written by the HDF5 library through ESIO, layouts 0, 1
  and 2): timestep 17, time 0.25, dt 0.125, U_mean = W_mean = (11, 22, 33), the Euu_kx plane
  i + 100 x, the fields c + 10 y + 100 x + 1000 z + 10000 f, read whole and with the reader
  decompositions of the reference test (1, 2, 4, 6 readers over kz, empty ones included).
* The writer against the HDF5 library: for the same datasets, the dataspace, datatype and fill
  value message bodies and the message flags equal the fixtures' byte for byte
  (tests/golden/h5_legacy_messages.json, made from the fixtures by tests/golden/make_h5_golden.py
  with the independent walker tests/h5walk.py), and the walker reads back the written data.
* The native round trip and the rank-0 append of the reference test, and its four rejections
  with their messages (rank, type, shape, legacy metadata length).
"""
import json
import os

import numpy as np
import pytest

from channel_passive_b200 import IoFile, KmmError
from channel_passive_b200 import _lib
from tests.h5walk import H5Walk

HERE = os.path.dirname(__file__)
GOLDEN = json.load(open(os.path.join(HERE, "golden", "h5_legacy_messages.json")))
FIXTURES = "/root/reference/SOURCE_PASSOPB/tests/io/fixtures"
NY, NX, NZ = 3, 5, 4
NAMES = ["u", "v", "w", "g", "phi", "theta"]


def _want(f):
    """io_roundtrip.f90: component c + 10 y + 100 x + 1000 z + 10000 f (1-based), as (nz, nx, ny)."""
    z, x, y = np.indices((NZ, NX, NY))
    base = 10 * (y + 1) + 100 * (x + 1) + 1000 * (z + 1) + 10000 * f
    return (base + 1) + 1j * (base + 2)


def _write_native(path):
    """The 'write' branch of io_roundtrip.f90 with one writer."""
    with IoFile(path, "w") as f:
        f.string_set("Readme", "Channel I/O compatibility test")
        f.line_write("timestep", np.array([17], np.int32), "Current step in time")
        f.line_write("time", [0.25], "Simulation time")
        f.line_write("dt", [0.125])
        for n in ("U_mean", "W_mean", "T_mean"):
            f.line_write(n, [11.0, 22.0, 33.0])
        i, x = np.indices((NY, NX))
        f.plane_write("Euu_kx", ((i + 1) + 100 * (x + 1)).T, "Spectrum plane")
        for k, n in enumerate(NAMES):
            f.field_write(n, _want(k + 1))
    with IoFile(path, "r+") as f:  # rank-0 statistics: reopen for update without truncation
        f.line_write("appended", [42.0])
        f.line_write("appended", [43.0])
        assert f.line_read("time", 1)[0] == 0.25


def _check_read(path, legacy):
    with IoFile(path) as f:
        assert f.line_read("timestep", 1, np.int32)[0] == 17
        assert f.line_read("time", 1)[0] == 0.25
        assert f.line_read("dt", 1)[0] == 0.125
        assert np.array_equal(f.line_read("U_mean", NY), [11, 22, 33])
        assert np.array_equal(f.line_read("W_mean", NY), [11, 22, 33])
        if not legacy:
            assert np.array_equal(f.line_read("T_mean", NY), [11, 22, 33])
        assert f.line_read("appended", 1)[0] == 43
        i, x = np.indices((NY, NX))
        assert np.array_equal(f.plane_read("Euu_kx", NY, NX), ((i + 1) + 100 * (x + 1)).T)
        for k, n in enumerate(NAMES[:5] if legacy else NAMES):
            assert np.array_equal(f.field_read(n, NY, NX, NZ), _want(k + 1)), n
            for np_ in (1, 2, 4, 6):  # the reference's readers: kz split, some ranks empty
                for rank in range(np_):
                    zs, zn = rank * NZ // np_, (rank + 1) * NZ // np_ - rank * NZ // np_
                    got = f.field_read(n, NY, NX, NZ, z=(zs, zn))
                    assert np.array_equal(got, _want(k + 1)[zs:zs + zn]), (n, np_, rank)
        if legacy:
            with pytest.raises(KmmError) as e:
                f.field_read("theta", NY, NX, NZ)
            assert e.value.code == _lib.KMM_ERR_IO and "missing restart dataset theta" in str(e.value)


@pytest.mark.skipif(not os.path.isdir(FIXTURES), reason="the reference checkout is not here")
@pytest.mark.parametrize("name", ["legacy.h5", "legacy-layout-1.h5", "legacy-layout-2.h5"])
def test_reference_fixtures_known_answers(name):
    _check_read(os.path.join(FIXTURES, name), legacy=True)
    with IoFile(os.path.join(FIXTURES, name)) as f:
        assert f.string_get("Readme") == "TBL legacy compatibility fixture"


def test_golden_matches_the_known_answers():
    """The golden summary holds what the fixtures hold (so the writer comparison below compares
    with the HDF5 library's bytes of these same values)."""
    for fn, g in GOLDEN.items():
        sets = g["datasets"]
        for k, n in enumerate(NAMES[:5]):
            # every layout stores the elements in the same order (layout 2 only flattens the shape)
            data = np.frombuffer(bytes.fromhex(sets[n]["data"]), dtype="<f8").view(np.complex128)
            assert np.array_equal(data, _want(k + 1).reshape(-1)), (fn, n)
        assert np.frombuffer(bytes.fromhex(sets["timestep"]["data"]), "<i4")[0] == 17


def test_native_roundtrip_and_append(tmp_path):
    p = str(tmp_path / "native.h5")
    _write_native(p)
    _check_read(p, legacy=False)
    with IoFile(p) as f:
        assert f.string_get("Native_IO") == "POONGBACK channel native parallel HDF5 v1"
        assert f.string_get("Readme") == "Channel I/O compatibility test"


def test_writer_messages_match_the_hdf5_library(tmp_path):
    """Every dataset the legacy fixture and a native file share: identical dataspace, datatype
    and fill-value message bodies, identical flags per message type, identical comments and data
    (the fixture is layout 0 without ESIO metadata)."""
    p = str(tmp_path / "native.h5")
    _write_native(p)
    w = H5Walk(p)
    ref = GOLDEN["legacy.h5"]
    assert (w.leaf_k, w.node_k) == (ref["leaf_k"], ref["node_k"])
    common = sorted(set(ref["datasets"]) & set(w.links))
    assert len(common) == 12, common
    for name in common:
        r, m = ref["datasets"][name], w.dataset(name)
        assert m[0x01][1].hex() == r["dataspace"], name
        assert m[0x03][1].hex() == r["datatype"], name
        assert m[0x05][1].hex() == r["fill"], name
        for t in (0x01, 0x03, 0x05, 0x08, 0x12):
            assert m[t][0] == r["flags"][hex(t)], (name, hex(t))
        assert (m[0x0D][1].split(b"\0")[0].decode() if 0x0D in m else "") == r["comment"], name
        assert w.data(name).hex() == r["data"], name
    # links sorted by name in the B-tree: every key is the last name of its node, ascending
    keys = w.btree_keys[0]
    assert keys[0] == "" and keys[1:] == sorted(keys[1:])
    # the local heap's free list ends with the library's sentinel 1
    assert w.heap_free < w.heap_size
    nxt, size = np.frombuffer(w.b[w.heap_data + w.heap_free:w.heap_data + w.heap_free + 16], "<u8")
    assert nxt == 1 and w.heap_free + size <= w.heap_size


@pytest.mark.parametrize("case,message", [
    ("rank", "unexpected dataset rank"),
    ("type", "expected array-valued field"),
    ("shape", "restart dimensions do not match input"),
    ("metadata", "malformed legacy metadata length"),
])
def test_rejections(tmp_path, case, message):
    """run_io_tests.py: ambiguous layouts and types are refused, not read as complex data."""
    p = str(tmp_path / "bad.h5")
    _write_native(p)
    with IoFile(p, "r+") as f:
        data = f.field_read("u", NY, NX, NZ)
        pairs = np.stack([data.real, data.imag], axis=-1)  # (nz, nx, ny, 2)
        if case == "metadata":
            f.attr_write_int("u", "esio_field_metadata", np.zeros(7, np.int32))
        elif case == "rank":
            f.write_raw("u", pairs)  # a 4-D scalar dataset
        elif case == "type":
            f.write_raw("u", pairs[..., 0])  # 3-D scalar dataset
        else:
            f.write_raw("u", np.zeros((NZ, NX + 1, NY, 2)), ncomp=2)
    with IoFile(p) as f:
        with pytest.raises(KmmError) as e:
            f.field_read("u", NY, NX, NZ)
    assert e.value.code == _lib.KMM_ERR_IO and message in str(e.value)


def test_legacy_layouts_through_metadata(tmp_path):
    """ESIO layouts 1 (3-D) and 2 (flattened (nz * nx, ny)), announced by esio_field_metadata,
    read like layout 0; metadata naming other dimensions is refused."""
    p = str(tmp_path / "legacy2.h5")
    _write_native(p)
    with IoFile(p, "r+") as f:
        for k, n in enumerate(NAMES):
            d = _want(k + 1)
            pairs = np.stack([d.real, d.imag], axis=-1)
            if k % 2:
                f.write_raw(n, pairs.reshape(NZ * NX, NY, 2), ncomp=2)
                f.attr_write_int(n, "esio_field_metadata", [0, 1, 8, 2, NZ, NX, NY, 2])
            else:
                f.write_raw(n, pairs, ncomp=2)
                f.attr_write_int(n, "esio_field_metadata", [0, 1, 8, 1, NZ, NX, NY, 2])
    _check_read(p, legacy=False)
    with IoFile(p, "r+") as f:
        f.attr_write_int("v", "esio_field_metadata", [0, 1, 8, 2, NZ, NX, NY + 1, 2])
    with IoFile(p) as f:
        with pytest.raises(KmmError) as e:
            f.field_read("v", NY, NX, NZ)
    assert "legacy field metadata does not match input" in str(e.value)


def test_missing_and_malformed_files(tmp_path):
    with pytest.raises(KmmError) as e:
        IoFile(str(tmp_path / "absent.h5"))
    assert e.value.code == _lib.KMM_ERR_IO
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"\x89HDF\r\n\x1a\n" + b"\0" * 40)
    with pytest.raises(KmmError) as e:
        IoFile(str(bad))
    assert e.value.code == _lib.KMM_ERR_IO
    p = str(tmp_path / "x.h5")
    _write_native(p)
    with pytest.raises(KmmError):  # io_file_create without overwrite refuses an existing file
        IoFile(p, "x")
    # a truncated file is refused, not read past its end
    raw = open(p, "rb").read()
    t = tmp_path / "t.h5"
    t.write_bytes(raw[:len(raw) // 2])
    with pytest.raises(KmmError) as e:
        with IoFile(str(t)) as f:
            f.field_read("theta", NY, NX, NZ)
    assert e.value.code == _lib.KMM_ERR_IO
