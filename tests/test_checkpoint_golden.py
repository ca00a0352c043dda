"""The checkpoint fixtures (tests/golden/ck_*.npz, made by make_golden.py
from the reference binary with oracle/ref_checkpoint.c standing in for its
HDF5 modules) checked on the CPU against what the reference's layout code
(Output/h5out.c:349-598, Output/ascii.c:7-77, Restart/h5in.c:72-77) says
they must hold: Index is the running cell count, Id_phi0 the first cell of
largest cos(phi), the Cells rows prim / Phi / piph, the ascii lines the same
cells' centres and prims, and the state right after a restart the
checkpoint's piph and face fluxes."""
import os

import numpy as np
import pytest

from helpers import CKPT_CASES, GOLDEN, golden


@pytest.mark.parametrize("case", CKPT_CASES)
def test_layout(case):
    g = golden(case)
    Np = g["ck_Np"]
    assert np.array_equal(Np.ravel(), g["Np"])
    idx = np.concatenate([[0], np.cumsum(Np.ravel())[:-1]])
    assert np.array_equal(g["ck_Index"].ravel(), idx)
    assert np.array_equal(g["ck_r_jph"], g["r_jph"]) and np.array_equal(g["ck_z_kph"], g["z_kph"])
    cells = g["ck_Cells"]
    q = g["s0_prim"].shape[1]
    nf = cells.shape[1] - q - 1
    assert nf in (0, 3, 5)
    assert cells.shape[0] == g["Np"].sum()
    assert np.all(np.isfinite(cells))
    assert g["ck_T"][0] == g["sN_t"]
    assert np.array_equal(g["ck_Planets"], g["sN_planets"])
    # Id_phi0: within each annulus, the first cell of largest cos(phi)
    phi = cells[:, -1] - .5 * g["sN_dphi"]
    c = np.cos(phi)
    for jk, (o, n) in enumerate(zip(idx, Np.ravel())):
        best = o + int(np.argmax(c[o:o + n]))
        got = g["ck_Id_phi0"].ravel()[jk]
        # numpy's cos may differ from libm's in the last bit: accept a tie
        assert got == best or abs(c[got] - c[best]) <= 4e-16, (jk, got, best)
    # Diagnostics: the window's sums divided by its length
    nt = g["ck_Diagnostics"].shape[2]
    if nt:
        want = g["sN_Qrz"].reshape(g["ck_Diagnostics"].shape) / g["sN_t_avg"]
        assert np.array_equal(g["ck_Diagnostics"], want)


@pytest.mark.parametrize("case", CKPT_CASES)
def test_ascii_lines(case):
    g = golden(case)
    rows = np.array([[float(x) for x in line.split()] for line in
                     bytes(g["ascii"]).decode().splitlines()])
    cells = g["ck_Cells"]
    q = g["s0_prim"].shape[1]
    Nz, Nr = g["ck_Np"].shape
    rj, zk = g["r_jph"], g["z_kph"]
    order, jrow, krow = [], [], []
    idx = g["ck_Index"]
    for j in range(Nr):                      # ascii.c: j outer, k inner
        for k in range(Nz):
            n = g["ck_Np"][k, j]
            order.extend(range(idx[k, j], idx[k, j] + n))
            jrow += [j] * n
            krow += [k] * n
    order, jrow, krow = np.array(order), np.array(jrow), np.array(krow)
    assert rows.shape == (len(order), 6 + q)
    piph, dphi = cells[order, -1], g["sN_dphi"][order]
    close = lambda a, b: np.testing.assert_allclose(a, b, rtol=6e-6, atol=1e-300)
    close(rows[:, 0], .5 * (rj[jrow + 1] + rj[jrow]))       # r_jph[j], r_jph[j-1]
    close(rows[:, 1], piph - .5 * dphi)
    close(rows[:, 2], .5 * (zk[krow + 1] + zk[krow]))
    close(rows[:, 3], rj[jrow + 1] - rj[jrow])
    close(rows[:, 4], dphi)
    close(rows[:, 5], zk[krow + 1] - zk[krow])
    close(rows[:, 6:], cells[order, :q])


@pytest.mark.parametrize("case", CKPT_CASES)
def test_restart_state(case):
    """setupCells after restart (domain.c:139-240): piph and Phi as stored,
    dphi from calc_dp, prim within round-off of the stored prim (prim2cons
    then cons2prim), the checkpoint's planets and time."""
    g = golden(case)
    cells = g["ck_Cells"]
    q = g["s0_prim"].shape[1]
    assert np.array_equal(g["r0_piph"], cells[:, -1])
    if "r0_Phi" in g:
        assert np.array_equal(g["r0_Phi"], cells[:, q:-1])
    assert np.array_equal(g["r0_dphi"], g["sN_dphi"])
    r = g["real"] == 1
    err = np.abs(g["r0_prim"][r] - cells[r, :q]) / np.maximum(np.abs(cells[r, :q]), 1e-300)
    with open(os.path.join(GOLDEN, case + ".par")) as f:
        noisy = any(line.split()[:2] not in (["Noise_Type", "0"], []) and line.split()[0] == "Noise_Type"
                    for line in f if line.split())
    if noisy:
        assert err.max() > 1e-6         # setupCells adds the noise again on restart
    else:
        assert err.max() < 1e-11        # pressure from E - kinetic energy: cancellation
    assert np.array_equal(g["r0_planets"], g["ck_Planets"])
    assert g["r0_t"] == g["ck_T"][0]
