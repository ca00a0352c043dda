"""setupCells' options against the reference binary: addNoise (noise.c:15-50,
in.par Noise_Type 1 / 2 / 3 with Noise_Abs / Noise_Rel), whose draws come
from glibc's rand() in the reference's cell order (made on the host by
disco_setup_noise and applied on the device after the Initial module), and
Include_Atmos (adjust_gas, planet.c:76-96, with the binary's potential).
The noise fixtures are libm-free (rigid rotation, no gravity): set-up state,
getmindt and the steps bit for bit.  adjust_gas calls cos, sin and pow, so
the atmosphere case is held to 1e-13 at set-up and 1e-11 after the steps."""
import numpy as np
import pytest

import disco_b200 as db
from helpers import case_disk, rel_l1_cols

pytestmark = pytest.mark.gpu

CASES = ["c0_noise1", "c0_noise2", "c1_noise3", "c0_atmos"]
EXACT = {"c0_noise1", "c0_noise2", "c1_noise3"}


@pytest.mark.parametrize("case", CASES)
def test_setup_options(case):
    disk, g = case_disk(case)
    b = db.Batch([disk])
    st = b.get_cells()
    r = disk.real == 1
    if case in EXACT:
        assert disk.noise is not None
        assert np.array_equal(st["prim"][r], g["s0_prim"][r])
        assert np.array_equal(st["cons"][r], g["s0_cons"][r])
        assert b.mindt()[0] == g["s0_dt_next"]
    else:
        assert max(rel_l1_cols(st["prim"][r], g["s0_prim"][r])) < 1e-13
        assert abs(b.mindt()[0] / g["s0_dt_next"] - 1) < 1e-13


@pytest.mark.parametrize("case", CASES)
def test_setup_options_steps(case):
    disk, g = case_disk(case)
    b = db.Batch([disk])
    dts = []
    for _ in range(int(g["nsteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    b.sync()
    st = b.get_cells()
    r = disk.real == 1
    if case in EXACT:
        assert np.array_equal(np.array(dts), g["dt"])
        assert np.array_equal(st["prim"][r], g["sN_prim"][r])
    else:
        assert np.max(np.abs(np.array(dts) / g["dt"] - 1)) < 1e-11
        assert max(rel_l1_cols(st["prim"][r], g["sN_prim"][r])) < 1e-11


def test_noise_needs_draws():
    """A batch whose disk has Noise_Type set refuses to set up without the
    draws (the C ABI order: disco_batch_set_noise first)."""
    disk, g = case_disk("c0_noise1")
    b = db.Batch([disk], setup=False)
    b.set_cells(None, None, disk.piph, disk.dphi, None, disk.real)
    assert db.library().disco_batch_setup_cells(b.h) == 7     # DISCO_ERR_STATE
