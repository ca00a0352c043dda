"""Viscosity of the Euler module (in.par Use_Viscosity, Viscosity,
Use_As_Alpha) against the reference binary: visc_flux added to the Riemann
flux at phi, r and z faces from the averaged face state and gradients
(riemann.c:295-310, euler.c:217-259), visc_source (euler.c:261-295) and the
viscous limit of mindt (euler.c:357-375).

- c0_visc: constant nu large enough that the viscous dt limit sets every
  step's dt; rigid rotation without gravity, no libm call: bit for bit.
- c0_visc_alpha: alpha viscosity (nu = alpha c^2 r^1.5, a pow) on the
  Keplerian disk with point-mass gravity: 1e-11 relative L1, as the other
  gravity fixtures.
"""
import os

import numpy as np
import pytest

import disco_b200 as db
from helpers import case_disk, par_with, rel_l1, rel_l1_cols

pytestmark = pytest.mark.gpu


def _steps(b, n):
    dts = []
    for _ in range(n):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    b.sync()
    return np.array(dts)


@pytest.mark.parametrize("case", ["c0_visc", "c0_visc_alpha"])
def test_viscosity_matches_reference(case):
    disk, g = case_disk(case)
    assert disk.params.visc_flag == 1
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    dts = _steps(b, int(g["nsteps"]))
    st = b.get_cells()
    r = disk.real == 1
    if case == "c0_visc":
        assert np.array_equal(dts, g["dt"])
        assert np.array_equal(st["prim"][r], g["sN_prim"][r])
        assert np.array_equal(st["cons"][r], g["sN_cons"][r])
    else:
        assert np.max(np.abs(dts / g["dt"] - 1)) < 1e-11
        assert max(rel_l1_cols(st["prim"][r], g["sN_prim"][r])) < 1e-11


def test_viscosity_device_setup_and_mixed():
    """The device set-up of the viscous disk equals the reference's step 0,
    and the mixed form follows FP64 within its 1e-5."""
    disk, g = case_disk("c0_visc_alpha")
    a = db.Batch([disk])
    m = db.Batch([disk], precision=db.PREC_MIXED)
    assert abs(a.mindt()[0] / g["s0_dt_next"] - 1) < 1e-13
    _steps(a, 20)
    _steps(m, 20)
    sa, sm = a.get_cells(), m.get_cells()
    r = disk.real == 1
    err = max(rel_l1(sm["prim"][r, q], sa["prim"][r, q]) for q in (0, 1, 3))
    print("mixed vs FP64 with alpha viscosity, 20 steps: %.2e" % err)
    assert err < 1e-5


def test_viscosity_refused_with_mhd():
    """Hydro/mhd.c has no visc_flux: viscous MHD is refused."""
    _, opt = db.template_paths("c1_mhd2d")
    p = par_with({"Num_R": 8, "Use_Viscosity": 1, "Viscosity": 0.01}, base="c1_mhd2d")
    disk = db.Disk.from_files(p, opt)
    os.unlink(p)
    with pytest.raises(db.DiscoError) as e:
        db.Batch([disk])
    assert e.value.status == 3
