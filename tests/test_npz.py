"""The checkpoint container (disco_b200/host/disco_npz.c) against NumPy's own
.npz reader and writer, on the CPU: what the C writer produces numpy.load
reads back (and zipfile's CRC check passes), what numpy.savez produces the C
reader reads, pieces appended through begin/append/end equal one put, and
malformed use is refused."""
import ctypes as C
import zipfile

import numpy as np
import pytest

import disco_b200 as db


def _create(path):
    z = C.c_void_p()
    assert db.library().disco_npz_create(str(path).encode(), C.byref(z)) == 0
    return z


def _put(z, name, a):
    a = np.ascontiguousarray(a)
    shape = (C.c_int64 * max(a.ndim, 1))(*a.shape)
    return db.library().disco_npz_put(z, name.encode(), a.dtype.str.encode(), a.ndim, shape,
                                      a.ctypes.data_as(C.c_void_p))


def _open(path):
    z = C.c_void_p()
    s = db.library().disco_npz_open(str(path).encode(), C.byref(z))
    return s, z


def _read(z, name):
    lib = db.library()
    descr = C.create_string_buffer(16)
    nd = C.c_int()
    sh = (C.c_int64 * 8)()
    s = lib.disco_npz_info(z, name.encode(), descr, C.byref(nd), sh)
    if s:
        return s, None
    a = np.zeros(tuple(sh[:nd.value]), np.dtype(descr.value.decode()))
    s = lib.disco_npz_read(z, name.encode(), 0, a.ctypes.data_as(C.c_void_p), a.nbytes)
    return s, a


ARRAYS = {
    "Grid/T": np.array([12.5]),
    "Grid/Index": np.arange(12, dtype=np.int32).reshape(3, 4),
    "Data/Cells": np.random.default_rng(1).standard_normal((37, 9)),
    "Data/Diagnostics": np.zeros((3, 4, 0)),
    "Opts/HYDRO": np.array([b"mhd"]),
    "Grid/r_jph": np.linspace(0.5, 3.0, 11),
}


def test_c_writes_numpy_reads(tmp_path):
    p = tmp_path / "c.npz"
    z = _create(p)
    for k, a in ARRAYS.items():
        assert _put(z, k, a) == 0, k
    assert db.library().disco_npz_close(z) == 0
    with zipfile.ZipFile(p) as zf:
        assert zf.testzip() is None                    # every member's CRC-32
    got = np.load(p)
    assert sorted(got.files) == sorted(ARRAYS)
    for k, a in ARRAYS.items():
        assert got[k].dtype == a.dtype and got[k].shape == a.shape, k
        assert np.array_equal(got[k], a), k


def test_numpy_writes_c_reads(tmp_path):
    p = tmp_path / "np.npz"
    np.savez(p, **ARRAYS)
    s, z = _open(p)
    assert s == 0
    for k, a in ARRAYS.items():
        s, b = _read(z, k)
        assert s == 0, k
        assert b.dtype == a.dtype and b.shape == a.shape and np.array_equal(a, b), k
    s, _ = _read(z, "Data/Missing")
    assert s == 9
    assert db.library().disco_npz_close(z) == 0


def test_pieces_equal_put(tmp_path):
    lib = db.library()
    a = np.random.default_rng(2).standard_normal((1000, 15))
    p1, p2 = tmp_path / "one.npz", tmp_path / "pieces.npz"
    z = _create(p1)
    assert _put(z, "Data/Cells", a) == 0
    assert lib.disco_npz_close(z) == 0
    z = _create(p2)
    shape = (C.c_int64 * 2)(*a.shape)
    assert lib.disco_npz_begin(z, b"Data/Cells", b"<f8", 2, shape) == 0
    for r0 in range(0, 1000, 333):
        piece = np.ascontiguousarray(a[r0:r0 + 333])
        assert lib.disco_npz_append(z, piece.ctypes.data_as(C.c_void_p), piece.nbytes) == 0
    assert lib.disco_npz_end(z) == 0
    assert lib.disco_npz_close(z) == 0
    assert p1.read_bytes() == p2.read_bytes()
    # a byte range of the data, as restart reads one annulus at a time
    s, z = _open(p2)
    row = np.zeros(15)
    assert lib.disco_npz_read(z, b"Data/Cells", 17 * 15 * 8, row.ctypes.data_as(C.c_void_p), row.nbytes) == 0
    assert np.array_equal(row, a[17])
    assert lib.disco_npz_read(z, b"Data/Cells", 999 * 15 * 8, row.ctypes.data_as(C.c_void_p),
                              row.nbytes + 8) == 1                # past the end
    assert lib.disco_npz_close(z) == 0


def test_refusals(tmp_path):
    lib = db.library()
    z = _create(tmp_path / "bad.npz")
    shape = (C.c_int64 * 1)(4)
    assert lib.disco_npz_begin(z, b"x", b"<f8", 1, shape) == 0
    four = np.zeros(5)
    assert lib.disco_npz_append(z, four.ctypes.data_as(C.c_void_p), four.nbytes) == 1   # too many bytes
    assert lib.disco_npz_end(z) == 1                                                 # too few
    assert lib.disco_npz_close(z) == 0
    p = tmp_path / "comp.npz"
    np.savez_compressed(p, a=np.arange(100.0))
    s, z = _open(p)
    assert s == 0
    assert _read(z, "a")[0] == 3                       # compressed member: not supported
    lib.disco_npz_close(z)
    (tmp_path / "junk.npz").write_bytes(b"not a zip file at all" * 3)
    assert _open(tmp_path / "junk.npz")[0] == 9
    assert _open(tmp_path / "absent.npz")[0] == 9


@pytest.mark.parametrize("n", [0, 1])
def test_empty_and_tiny(tmp_path, n):
    p = tmp_path / "e.npz"
    z = _create(p)
    a = np.zeros((n, 7))
    assert _put(z, "Data/Planets", a) == 0
    assert db.library().disco_npz_close(z) == 0
    assert np.load(p)["Data/Planets"].shape == (n, 7)
