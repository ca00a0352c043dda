"""Host-side logic (no GPU): in.par / Makefile_opt.in parsing, grid and phi
set-up against the reference, and the C ABI surface of the library."""
import ctypes as C
import math
import os
import re

import numpy as np
import pytest

import disco_b200 as db
from helpers import CASES, case_disk, par_with

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_read_par_template():
    par, opt = db.template_paths("c0_kepler2d")
    p = db.read_par(par)
    assert p.Num_R == 128 and p.Num_Z == 1
    assert p.rmin == 0.5 and p.rmax == 3.0
    assert p.phimax == 2.0 * math.pi           # P_Times_2pi (readpar.c:166)
    assert p.CFL == 0.5 and p.PLM == 1.5 and p.Riemann_Solver == 1
    assert p.Adiabatic_Index == 1.6666666666667
    assert p.initPar0 == 314159 and p.initPar[1] == 1e-3
    m = db.read_opt(opt)
    assert (m.hydro, m.boundary, m.planets, m.num_c, m.num_n, m.ct_mode) == (0, 0, 1, 5, 1, 0)


def test_read_par_separators_and_first_match():
    path = par_with({"CFL": "=> 0.25  // comment", "PLM": ":1.0"})
    with open(path, "a") as f:
        f.write("CFL 0.9\n")                     # later duplicate is ignored (readpar.c:14-19)
    p = db.read_par(path)
    os.unlink(path)
    assert p.CFL == 0.25 and p.PLM == 1.0


def test_read_opt_unknown_module(tmp_path):
    f = tmp_path / "opt.in"
    f.write_text("INITIAL = kepler_noise\nHYDRO = greuler\nGEOMETRY = cylindrical\n")
    with pytest.raises(db.DiscoError) as e:
        db.read_opt(str(f))
    assert e.value.status == 3


@pytest.mark.parametrize("case", CASES)
def test_grid_and_phi_match_reference(case):
    disk, g = case_disk(case)
    assert np.array_equal(disk.Np, g["Np"])
    assert np.array_equal(disk.r_jph, g["r_jph"])
    assert np.array_equal(disk.z_kph, g["z_kph"])
    assert np.array_equal(disk.piph, g["s0_piph"])
    assert np.array_equal(disk.dphi, g["s0_dphi"])
    assert np.array_equal(disk.real, g["real"])


@pytest.mark.parametrize("case,module", [("c0_horizon3d", "horizon3d"), ("c1_polar3dbc", "polar3d"),
                                         ("c3_grhorizon", "horizon"), ("c0_hbin", "horizon_bin"),
                                         ("c0_hbin3d", "horizon_bin")])
def test_axis_and_horizon_modules_parse(case, module):
    """The excising boundary modules read from Makefile_opt.in; the grid
    matches the reference, whose real flag also drops the excised annuli."""
    disk, g = case_disk(case)
    assert disk.modules.boundary == db.BOUNDARY[module]
    assert disk.Ng[0] == 0
    assert np.array_equal(disk.Np, g["Np"]) and np.array_equal(disk.r_jph, g["r_jph"])
    r = disk.real == 1
    assert (g["real"][~r] == 0).all()
    excised = r & (g["real"] == 0)
    assert excised.any() == module.startswith("horizon")


def test_np_floor_minimum_four():
    path = par_with({"Num_R": 4, "aspect": 100.0})
    disk = db.Disk(db.read_par(path), db.read_opt(db.template_paths("c0_kepler2d")[1]))
    os.unlink(path)
    assert disk.Np.min() == 4                    # gridsetup.c:137-138


def test_struct_layouts_match_library():
    lib = db.library()
    assert lib.disco_sizeof(0) == C.sizeof(db.Params)
    assert lib.disco_sizeof(1) == C.sizeof(db.Modules)
    assert lib.disco_abi_version() == 3


def test_library_exports_every_declared_symbol():
    names = set()
    for h in os.listdir(os.path.join(REPO, "include")):
        text = open(os.path.join(REPO, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(disco_\w+)\s*\(", text))
    assert len(names) >= 20
    lib = C.CDLL(db.LIBPATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_no_device_is_a_clean_error():
    """Without a GPU every device entry point fails loudly (no CPU fallback)."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    disk = db.Disk.from_files(*db.template_paths("c0_kepler2d"))
    with pytest.raises(db.DiscoError) as e:
        db.Batch([disk])
    assert e.value.status == 6
    assert db.library().disco_strerror(6) == b"no CUDA device"


@pytest.mark.parametrize("case,module", [("c0_bc_fixRrefZ", "fixRrefZ"), ("c0_bc_tube", "tube"),
                                         ("c0_bc_surfaceGravBox", "surfaceGravBox"),
                                         ("c0_bc_fixed_gap", "fixed_gap"),
                                         ("c0_bc_flowthrough", "flowthrough")])
def test_composed_boundary_modules_parse(case, module):
    disk, g = case_disk(case)
    assert disk.modules.boundary == db.BOUNDARY[module]
    assert np.array_equal(disk.Np, g["Np"]) and np.array_equal(disk.real, g["real"])
