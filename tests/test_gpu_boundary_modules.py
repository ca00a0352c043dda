"""Boundary modules beyond fixed / fixed3d / zerograd, against the reference
binary built with the same module (rigid rotation without gravity, so the
fixtures depend on no libm call except where noted):

- polar (Boundary/polar.c) on grids down to the axis (NoBC_Rmin 1, R_Min 0):
  no inner ghosts, the first annulus's r slopes fixed by plm_geom_boundary ->
  geom_grad (plm.c:184-185, cylindrical.c:141-173), the polar source terms
  (euler.c, mhd.c, planet.c with NoBC_Rmin; they call sin(dphi/2), whose
  CUDA and glibc values may differ in the last bit), and the outer r and z
  ghosts re-evaluated from the Initial module each substep.  2D hydro, 2D
  MHD with CT, 3D MHD with CT.
- outflow3d: zero-gradient copies with the outflow diode on every side
  (boundary_functions.c:269-440), 3D hydro.
- zerograd_omk: the same with Omega of the r ghosts from the Initial module
  (boundary_fixed_q_rinn / _rout), 3D MHD.
- accrete3d: outflow inner r, fixed outer r and z (set_cell_init), 3D MHD
  with CT.
- polar3d: fixed outer r and z (set_cell_init) on an axis grid, 3D MHD with
  CT.
- fixRrefZ, tube, surfaceGravBox, fixed_gap, flowthrough: composed per side from fixed
  (set_cell_init), zero-gradient (with or without the outflow diode) and
  mirror copies (boundary_reflect_*: the annulus as far inside as the ghost
  is outside, normal velocity negated; no-slip: all three), r sides before z
  sides (flowthrough's outer r fixed again on an azimuthal window after its
  copy); 3D hydro.
- horizon_bin: outer r and z ghosts at the midpoint, and every cell inside
  one of two spheres of radius 0.8 at x = +-5 re-initialised there each
  substep, out of the dt minimum from its first excision on (the
  reference's real flag is never set back); 2D and 3D hydro.  The test is
  per cell with sin and cos of the cell's phi (libm).
- horizon3d: polar3d's ghosts plus boundary_fixed_horizon
  (boundary_functions.c:622-656): every annulus whose outer corner lies
  inside R = 1 is re-initialised by set_cell_init each substep and left out
  of the dt minimum, 3D hydro on an axis grid.

State compared at 1e-12 relative L1 (in practice far below), face lists bit
for bit, ghost cells included at set-up."""
import os

import numpy as np
import pytest

import disco_b200 as db
from helpers import case_disk, observed_slots, par_with, rel_l1, rel_l1_cols

pytestmark = pytest.mark.gpu

POLAR = ["c0_polar", "c1_polar_ct", "c1_polar3d", "c1_polar3dbc", "c0_horizon3d"]
COMPOSED = ["c0_bc_fixRrefZ", "c0_bc_tube", "c0_bc_surfaceGravBox", "c0_bc_fixed_gap",
            "c0_bc_flowthrough"]
CASES = POLAR + ["c0_outflow3d", "c1_omk3d", "c1_accrete3d", "c0_hbin", "c0_hbin3d"] + COMPOSED
TOL = 1e-12


@pytest.mark.parametrize("case", CASES)
def test_module_setup(case):
    """setupCells and the module's ghost values on the device."""
    disk, g = case_disk(case)
    if case in POLAR:
        assert disk.Ng[0] == 0 and disk.r_jph[0] == 0.0
    b = db.Batch([disk])
    st = b.get_cells()
    r = disk.real == 1
    assert np.array_equal(st["piph"], g["s0_piph"])
    assert max(rel_l1_cols(st["prim"][r], g["s0_prim"][r])) <= TOL
    # ghosts: the outer r layers and the z layers, set from the Initial module
    gh = ~r
    if gh.any():
        assert max(rel_l1_cols(st["prim"][gh], g["s0_prim"][gh])) <= TOL
    assert abs(b.mindt()[0] / g["s0_dt_next"] - 1) <= TOL


@pytest.mark.parametrize("case", CASES)
def test_module_steps(case):
    disk, g = case_disk(case)
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"],
                Phi=g.get("s0_Phi"))
    dts = []
    for _ in range(int(g["nsteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    b.sync()
    st = b.get_cells()
    F = b.faces(0, 1)
    for k in ("fIndex", "iL", "iR", "LRtype"):
        assert np.array_equal(F[k], g[k]), k
    r = disk.real == 1
    assert np.max(np.abs(np.array(dts) / g["dt"] - 1)) <= TOL
    ep = rel_l1_cols(st["prim"][r], g["sN_prim"][r])
    ec = rel_l1_cols(st["cons"][r], g["sN_cons"][r])
    print("%s: prim %.2e cons %.2e" % (case, max(ep), max(ec)))
    assert max(ep) <= TOL and max(ec) <= TOL
    # the axis annulus itself (its slopes are the geometric ones); the ghosts
    if case in POLAR:
        a0 = slice(0, int(disk.Np[0]))
        assert max(rel_l1_cols(st["prim"][a0], g["sN_prim"][a0])) <= TOL
    gh = ~r
    assert max(rel_l1_cols(st["prim"][gh], g["sN_prim"][gh])) <= TOL
    if "sN_Phi" in g:
        m = observed_slots(disk, b.num_faces)
        for s in range(m.shape[1]):
            if m[:, s].any():
                assert rel_l1(st["Phi"][m[:, s], s], g["sN_Phi"][m[:, s], s]) <= TOL, s


def test_polar_needs_the_axis():
    """The polar module leaves inner ghosts unset: refused on a grid that
    has them (NoBC_Rmin 0)."""
    p = par_with({"Num_R": 12}, base="c0_kepler2d")
    disk = db.Disk.from_files(p, os.path.join(db.TEMPLATES, "c0_polar.in"))
    os.unlink(p)
    with pytest.raises(db.DiscoError) as e:
        db.Batch([disk])
    assert e.value.status == 3


@pytest.mark.parametrize("module", ["polar3d", "horizon3d"])
def test_axis_modules_need_no_inner_ghosts(module):
    """polar3d and horizon3d set no inner r ghosts (Boundary/polar3d.c,
    horizon3d.c): refused on a grid that has them."""
    p = par_with({"Num_R": 12, "Num_Z": 4}, base="c1_mhd3d")
    cfg = {"polar3d": "c1_polar3dbc", "horizon3d": "c0_horizon3d"}[module]
    disk = db.Disk.from_files(p, os.path.join(db.TEMPLATES, cfg + ".in"))
    os.unlink(p)
    assert disk.modules.boundary == db.BOUNDARY[module]
    with pytest.raises(db.DiscoError) as e:
        db.Batch([disk])
    assert e.value.status == 3


def test_horizon3d_excises():
    """The fixture's excised annuli (the reference marks them not real) are
    inside R = 1, and after the steps their prims are the set_cell_init values
    the device left there too."""
    disk, g = case_disk("c0_horizon3d")
    geo = disk.real == 1
    ex = geo & (g["real"] == 0)
    assert ex.sum() > 0 and (g["real"][~geo] == 0).all()
    b = db.Batch([disk])
    st = b.get_cells()
    assert max(rel_l1_cols(st["prim"][ex], g["s0_prim"][ex])) <= TOL
    b.close()


def test_host_initial_module():
    """The same reference Initial module through the Python API: the disk
    reads as DISCO_IC_HOST, the device set-up refuses it, and from the
    reference's uploaded step-0 state the steps match the reference bit for
    bit (zero-gradient boundaries)."""
    disk, g = case_disk("c0_rigid_zg")
    assert disk.modules.initial == db.INITIAL["host"]
    with pytest.raises(db.DiscoError) as e:
        db.Batch([disk])
    assert e.value.status == 3
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    dts = []
    for _ in range(int(g["nsteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    b.sync()
    st = b.get_cells()
    r = disk.real == 1
    assert np.array_equal(np.array(dts), g["dt"])
    assert np.array_equal(st["prim"][r], g["sN_prim"][r])
