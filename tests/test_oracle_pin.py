"""The CPU oracle (oracle/oracle.c) is pinned bit-for-bit to the reference.

Golden fixtures come from running the reference itself
(tests/golden/make_golden.py); when the reference binary built by
oracle/Makefile is present, a full-size config-0 run is compared live too.
"""
import os

import numpy as np
import pytest

import pyoracle
from helpers import CASES, case_disk, golden, oracle_for


@pytest.mark.parametrize("case", CASES)
def test_oracle_matches_reference_golden(case):
    disk, g = case_disk(case)
    o = oracle_for(disk)
    o.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    assert o.mindt() == g["s0_dt_next"]
    dts = []
    for _ in range(int(g["nsteps"])):
        dt = o.mindt()
        dts.append(dt)
        o.timestep(dt)
    assert np.array_equal(np.array(dts), g["dt"])
    st = o.get_cells()
    real = g["real"] == 1
    for k in ("prim", "piph", "dphi", "wiph"):
        assert np.array_equal(st[k], g["sN_" + k]), k
    assert np.array_equal(st["cons"][real], g["sN_cons"][real])
    assert o.mindt() == g["sN_dt_next"]
    f = o.faces(1)
    for k in ("fIndex", "iL", "iR", "LRtype"):
        assert np.array_equal(f[k], g[k]), k
    assert np.array_equal(f["geom"], g["fgeom"])
    Q, _ = o.diagnostics()
    assert np.array_equal(Q, g["Qrz"])
    assert o.time() == g["t"]


def test_oracle_matches_reference_full_config0():
    """Config 0 at full size (Nr=128, 57,856 cells), 3 steps, live reference."""
    binary = pyoracle.ref_binary("c0_kepler2d")
    if not os.path.exists(binary) and not os.path.isdir(pyoracle.REF_SRC):
        pytest.skip("reference binary not built here")
    import disco_b200 as db
    par, opt = db.template_paths("c0_kepler2d")
    d0 = pyoracle.run_ref("c0_kepler2d", par, 0)
    d3 = pyoracle.run_ref("c0_kepler2d", par, 3)
    disk = db.Disk.from_files(par, opt)
    o = oracle_for(disk)
    o.set_cells(d0["prim"], d0["cons"], d0["piph"], d0["dphi"], d0["wiph"], d0["real"])
    for s in range(3):
        dt = o.mindt()
        assert dt == d3["dt"][s]
        o.timestep(dt)
    st = o.get_cells()
    assert np.array_equal(st["prim"], d3["prim"])
    assert np.array_equal(st["piph"], d3["piph"])
    f = o.faces(1)
    assert np.array_equal(f["iL"], d3["faces_1"]["iL"])
    assert np.array_equal(f["LRtype"], d3["faces_1"]["LRtype"])
