"""disco_mindt_noalloc: getmindt on caller-owned device arrays, with no
device allocation inside the library.

It serves callers that may not call cudaMalloc -- a host code that owns all
device memory through its own pool, or a run loop during which allocation is
forbidden.  Each test feeds it the state of a disk (kept in tensors the test
allocates, i.e. the caller's memory) and checks it against the allocating
entry point, disco_batch_mindt, on two calls in a row (the first call also
sets up the static scratch's device address).  The cases cover a 2D disk, a
3D disk with z ghost layers (z edges and the k index of the annulus table),
a grid of more than 1024 annuli (the table is uploaded in 1024-entry
chunks), and the viscous limit with constant nu and with alpha.  This file
is collected last on purpose.
"""
import ctypes as C
import os

import numpy as np
import pytest

import disco_b200 as db
from helpers import case_disk, par_with

pytestmark = pytest.mark.gpu


def _bind():
    lib = db.library()
    f = lib.disco_mindt_noalloc
    D = C.POINTER(C.c_double)
    I = C.POINTER(C.c_int)
    f.restype = C.c_int
    f.argtypes = [C.POINTER(db.Params), C.c_int, C.c_int, C.c_int, I, I, D, D,
                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, D]
    return f


def _noalloc_twice(disk, st):
    """Two calls of the entry point on the state st (host arrays), from
    device tensors the caller owns."""
    import torch
    f = _bind()
    dev = torch.device("cuda", 0)
    prim = torch.tensor(np.ascontiguousarray(st["prim"].T), dtype=torch.float64, device=dev)
    piph = torch.tensor(st["piph"], dtype=torch.float64, device=dev)
    dphi = torch.tensor(st["dphi"], dtype=torch.float64, device=dev)
    wiph = torch.tensor(st["wiph"], dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    Ng = np.ascontiguousarray(disk.Ng, np.int32)
    Np = np.ascontiguousarray(disk.Np, np.int32)
    rj = np.ascontiguousarray(disk.r_jph)
    zk = np.ascontiguousarray(disk.z_kph)
    torch.cuda.synchronize()
    out = []
    for _ in range(2):
        dt = C.c_double(0.0)
        s = f(C.byref(disk.params), 0, disk.Nr, disk.Nz, Ng.ctypes.data_as(C.POINTER(C.c_int)),
              Np.ctypes.data_as(C.POINTER(C.c_int)), rj.ctypes.data_as(C.POINTER(C.c_double)),
              zk.ctypes.data_as(C.POINTER(C.c_double)), prim.data_ptr(), piph.data_ptr(),
              dphi.data_ptr(), wiph.data_ptr(), stream, C.byref(dt))
        assert s == 0, db.STATUS.get(s, s)
        out.append(dt.value)
    return out


def test_mindt_noalloc_matches_batch_mindt():
    disk = db.Disk.from_files(*db.template_paths("c0_kepler2d"))
    b = db.Batch([disk])
    b.run(3)                                   # a state with moved, uneven cells
    b.sync()
    st = b.get_cells()
    dt_ref = b.mindt()[0]
    b.close()
    out = _noalloc_twice(disk, st)
    # the minimum is order independent, so the two paths agree bit for bit
    # (well inside the 1e-12 relative tolerance of the other parity tests)
    assert out[0] == dt_ref and out[1] == dt_ref, (out, dt_ref)


@pytest.mark.parametrize("case", ["c0_outflow3d", "c0_visc", "c0_visc_alpha"])
def test_mindt_noalloc_golden_states(case):
    """3D with z ghosts, and both forms of the viscous limit (the constant-nu
    case is set up so that the viscous limit decides dt)."""
    disk, g = case_disk(case)
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    dt_ref = b.mindt()[0]
    b.close()
    st = {"prim": g["s0_prim"], "piph": g["s0_piph"], "dphi": g["s0_dphi"], "wiph": g["s0_wiph"]}
    out = _noalloc_twice(disk, st)
    assert out[0] == dt_ref and out[1] == dt_ref, (case, out, dt_ref)


def test_mindt_noalloc_more_than_1024_annuli():
    p = par_with({"Num_R": 1100})               # 1104 annuli with the ghosts
    try:
        disk = db.Disk.from_files(p, os.path.join(db.TEMPLATES, "c0_kepler2d.in"))
    finally:
        os.unlink(p)
    assert disk.Nr * disk.Nz > 1024
    b = db.Batch([disk])
    b.run(3)
    b.sync()
    st = b.get_cells()
    dt_ref = b.mindt()[0]
    b.close()
    out = _noalloc_twice(disk, st)
    assert out[0] == dt_ref and out[1] == dt_ref, (out, dt_ref)


def test_mindt_noalloc_rejects_oversized_grid():
    f = _bind()
    disk = db.Disk.from_files(*db.template_paths("c0_kepler2d"))
    Nz = 1000                                  # 132 x 1000 annuli > 65536
    Ng = np.ascontiguousarray(disk.Ng, np.int32)
    Np = np.full(disk.Nr * Nz, 8, np.int32)
    rj = np.ascontiguousarray(disk.r_jph)
    zk = np.linspace(-0.5, 0.5, Nz + 1)
    dt = C.c_double(0.0)
    import torch
    tiny = torch.zeros(8, dtype=torch.float64, device="cuda")   # rejected before any use
    p = tiny.data_ptr()
    s = f(C.byref(disk.params), 0, disk.Nr, Nz, Ng.ctypes.data_as(C.POINTER(C.c_int)),
          Np.ctypes.data_as(C.POINTER(C.c_int)), rj.ctypes.data_as(C.POINTER(C.c_double)),
          zk.ctypes.data_as(C.POINTER(C.c_double)), p, p, p, p, None, C.byref(dt))
    assert s == 1
