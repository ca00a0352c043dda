"""disco_mindt_noalloc: getmindt on caller-owned device arrays, with no
device allocation inside the library.

It serves callers that may not call cudaMalloc -- a host code that owns all
device memory through its own pool, or a run loop during which allocation is
forbidden.  The test feeds it the state of a config-0 disk (kept in tensors
the test allocates, i.e. the caller's memory) and checks it against the
allocating entry point, disco_batch_mindt, on two calls in a row (the first
call also sets up the static scratch's device address).  This file is
collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

import disco_b200 as db

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


def test_mindt_noalloc_matches_batch_mindt():
    import torch
    f = _bind()
    disk = db.Disk.from_files(*db.template_paths("c0_kepler2d"))
    b = db.Batch([disk])
    b.run(3)                                   # a state with moved, uneven cells
    b.sync()
    st = b.get_cells()
    dt_ref = b.mindt()[0]

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
    # the minimum is order independent, so the two paths agree bit for bit
    # (well inside the 1e-12 relative tolerance of the other parity tests)
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
