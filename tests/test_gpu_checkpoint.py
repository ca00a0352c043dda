"""Checkpoint, ascii output and restart of the device state
(disco_batch_write_checkpoint / _write_ascii / _restart) against the
reference's own output and restart, from the ck_* fixtures of
tests/golden/make_golden.py:

- the writer on the reference's step-N state: every dataset of the
  reference's checkpoint (Grid/*, Data/Cells, Data/Planets) bit for bit, and
  the ascii file byte for byte;
- the writer after N steps on the GPU from the same start: bit for bit for
  the libm-free cases, within the point-mass gravity tolerance for ck_cm2,
  diagnostics averaged and then zeroed as output() does;
- restart from the reference's checkpoint (written by numpy into the .npz
  container): the set-up state and getmindt, then M steps, against the
  reference restarted from the same checkpoint;
- at full size, the properties a checkpoint exists for: write, restart into
  a fresh batch, write again -- piph, face fluxes, time and planets
  unchanged, prims to round-off -- and restarts from either file continue
  alike; a batch of several disks restarts disk by disk; files of another
  grid, missing, compressed or with another planet type are refused.
"""
import os

import numpy as np
import pytest

import disco_b200 as db
from helpers import (CKPT_CASES, CK_NAMES, GOLDEN, TEMPLATES, ck_to_npz, golden, observed_slots,
                     par_with, rel_l1, rel_l1_cols)

pytestmark = pytest.mark.gpu

EXACT = {"ck_rigid", "ck_ct_rigid", "ck_ct3d_rigid", "ck_noise"}
TOL = 1e-11            # point-mass force: CUDA's libm against glibc's, as the other fixtures


def _disk(case):
    g = golden(case)
    return db.Disk.from_files(os.path.join(GOLDEN, case + ".par"),
                              os.path.join(TEMPLATES, str(g["cfg"]) + ".in")), g


def _at_step_n(disk, g):
    """A batch holding the reference's step-N state, planets and time."""
    b = db.Batch([disk], setup=False)
    q = disk.q
    cells = g["ck_Cells"]
    Phi = cells[:, q:-1] if cells.shape[1] > q + 1 and b.ct else None
    b.set_cells(cells[:, :q], None, cells[:, -1], g["sN_dphi"], g["sN_wiph"], g["real"], Phi=Phi)
    b.set_planets(g["sN_planets"])
    b.set_time(float(g["sN_t"]))
    return b


def _from_start(disk, g):
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"],
                Phi=g.get("s0_Phi"))
    return b


@pytest.mark.parametrize("case", CKPT_CASES)
def test_writer_matches_reference(case, tmp_path):
    disk, g = _disk(case)
    b = _at_step_n(disk, g)
    f = np.load(b.write_checkpoint(str(tmp_path / "checkpoint_0001")))
    for k in ("T", "r_jph", "z_kph", "Index", "Np", "Id_phi0", "Cells", "Planets"):
        a, want = f[CK_NAMES[k]], g["ck_" + k]
        assert a.dtype == want.dtype and a.shape == want.shape, k
        assert np.array_equal(a, want), k
    assert f["Data/Diagnostics"].shape == g["ck_Diagnostics"].shape
    assert int(f["Opts/CT_MODE"][0]) == disk.modules.ct_mode
    assert f["Pars/Num_R"][0] == disk.params.Num_R


@pytest.mark.parametrize("case", CKPT_CASES)
def test_ascii_matches_reference(case, tmp_path):
    disk, g = _disk(case)
    b = _at_step_n(disk, g)
    with open(b.write_ascii(str(tmp_path / "output")), "rb") as fh:
        text = fh.read()
    assert text == bytes(g["ascii"])


@pytest.mark.parametrize("case", CKPT_CASES)
def test_writer_after_gpu_steps(case, tmp_path):
    disk, g = _disk(case)
    b = _from_start(disk, g)
    for _ in range(int(g["nsteps"])):
        b.timestep(b.mindt()[0])
    b.sync()
    f = np.load(b.write_checkpoint(str(tmp_path / "ck")))
    for k in ("r_jph", "z_kph", "Index", "Np"):
        assert np.array_equal(f[CK_NAMES[k]], g["ck_" + k]), k
    cells, want = f["Data/Cells"], g["ck_Cells"]
    if case in EXACT:
        for k in ("T", "Id_phi0", "Planets"):
            assert np.array_equal(f[CK_NAMES[k]], g["ck_" + k]), k
        q = disk.q
        nf = cells.shape[1] - q - 1
        assert np.array_equal(cells[:, :q], want[:, :q])           # prim
        assert np.array_equal(cells[:, -1], want[:, -1])           # piph
        if nf:                                                     # the face fluxes cells read
            m = observed_slots(disk, nf)
            assert np.array_equal(cells[:, q:-1][m], want[:, q:-1][m])
    else:
        assert abs(f["Grid/T"][0] / g["ck_T"][0] - 1) < TOL
        r = g["real"] == 1
        assert max(rel_l1_cols(cells[r], want[r])) < TOL
        assert np.abs(f["Data/Planets"] - g["ck_Planets"]).max() < TOL
        assert np.mean(f["Grid/Id_phi0"] == g["ck_Id_phi0"]) > 0.99
    D, Dw = f["Data/Diagnostics"], g["ck_Diagnostics"]
    if Dw.size:
        assert rel_l1(D, Dw) < (1e-12 if case in EXACT else TOL)
        Qrz, tavg = b.diagnostics()
        assert tavg == 0.0 and not np.any(Qrz)          # zero_diagnostics


@pytest.mark.parametrize("case", CKPT_CASES)
def test_restart_matches_reference(case, tmp_path):
    disk, g = _disk(case)
    path = ck_to_npz(g, str(tmp_path / "input.npz"))
    b = db.Batch([disk], setup=False)
    b.restart(path)
    b.sync()
    st = b.get_cells()
    r = g["real"] == 1
    t, cnt = b.time()
    assert t == g["r0_t"] and cnt == 0
    assert np.array_equal(b.planets(), g["r0_planets"])
    for k in ("piph", "dphi", "wiph"):
        assert np.array_equal(st[k], g["r0_" + k]), k
    if "r0_Phi" in g:
        assert np.array_equal(st["Phi"], g["r0_Phi"])
    if case in EXACT:
        assert np.array_equal(st["prim"], g["r0_prim"])
        assert np.array_equal(st["cons"][r], g["r0_cons"][r])
        assert b.mindt()[0] == g["r0_dt_next"]
    else:
        assert max(rel_l1_cols(st["prim"][r], g["r0_prim"][r])) < 1e-13
        assert abs(b.mindt()[0] / g["r0_dt_next"] - 1) < TOL
    dts = []
    for _ in range(int(g["msteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    b.sync()
    st = b.get_cells()
    t, cnt = b.time()
    assert cnt == int(g["msteps"])
    if case in EXACT:
        assert np.array_equal(np.array(dts), g["rM_dt"])
        assert t == g["rM_t"]
        for k in ("prim", "piph"):
            assert np.array_equal(st[k], g["rM_" + k]), k
        assert np.array_equal(st["cons"][r], g["rM_cons"][r])
        if "rM_Phi" in g:
            m = observed_slots(disk, g["rM_Phi"].shape[1])
            assert np.array_equal(st["Phi"][m], g["rM_Phi"][m])
        assert np.array_equal(b.planets(), g["rM_planets"])
    else:
        assert np.max(np.abs(np.array(dts) / g["rM_dt"] - 1)) < TOL
        assert max(rel_l1_cols(st["prim"][r], g["rM_prim"][r])) < TOL
        assert max(rel_l1_cols(st["cons"][r], g["rM_cons"][r])) < TOL
        assert np.abs(b.planets() - g["rM_planets"]).max() < TOL


def _mhd3d_ct(nr=24, nz=16):
    _, opt = db.template_paths("c1_mhd3d")
    p = par_with({"Num_R": nr, "Num_Z": nz, "Constrained_Transport": 1, "Init_Par5": 20.0,
                  "Init_Par6": 0.05, "Init_Par1": 0.05}, base="c1_mhd3d")
    disk = db.Disk.from_files(p, opt)
    os.unlink(p)
    return disk


@pytest.mark.parametrize("precision", [db.PREC_FP64, db.PREC_MIXED])
def test_roundtrip_full_size(tmp_path, precision):
    """3D MHD with constrained transport (24 x 16 annuli, ~110k cells): write
    A after 10 steps, restart a fresh batch from A and write B: piph, face
    fluxes, time, planets and the grid datasets identical, prims to the
    round-off of prim2cons / cons2prim.  Restarting from B and from A then
    gives the same run (10 steps) to round-off growth.

    Against the run that was never interrupted the restart differs by more
    than round-off, as the reference's does: setupCells recomputes the mesh
    velocities from the restored prims (set_wcell, domain.c:239), while the
    running job's getmindt still sees those set at the start of its last
    step, so the next dt and everything after it move by about one step's
    change of the mesh velocity."""
    disk = _mhd3d_ct()
    a = db.Batch([disk], precision=precision)
    a.run(10)
    a.sync()
    pa = a.write_checkpoint(str(tmp_path / "a"))
    b = db.Batch([disk], precision=precision, setup=False)
    b.restart(pa)
    pb = b.write_checkpoint(str(tmp_path / "b"))
    fa, fb = np.load(pa), np.load(pb)
    q = disk.q
    for k in ("Grid/T", "Grid/r_jph", "Grid/z_kph", "Grid/Index", "Grid/Np", "Grid/Id_phi0",
              "Data/Planets"):
        assert np.array_equal(fa[k], fb[k]), k
    ca, cb = fa["Data/Cells"], fb["Data/Cells"]
    assert np.array_equal(ca[:, q:], cb[:, q:])           # Phi and piph
    r = disk.real == 1
    tol = 1e-13 if precision == db.PREC_FP64 else 1e-6
    assert max(rel_l1_cols(cb[r, :q], ca[r, :q])) < tol
    c = db.Batch([disk], precision=precision, setup=False)
    c.restart(pb)
    b.restart(pa)
    b.run(10)
    c.run(10)
    a.run(10)
    for x in (a, b, c):
        x.sync()
    sa, sb, sc = a.get_cells(), b.get_cells(), c.get_cells()
    e_bc = max(rel_l1_cols(sc["prim"][r], sb["prim"][r]))
    e_ab = max(rel_l1_cols(sb["prim"][r], sa["prim"][r]))
    print("after 10 more steps: restart(B) vs restart(A) %.2e, restart(A) vs uninterrupted %.2e"
          % (e_bc, e_ab))
    assert e_bc < (1e-11 if precision == db.PREC_FP64 else 1e-5)
    assert abs(b.time()[0] / c.time()[0] - 1) < (1e-13 if precision == db.PREC_FP64 else 1e-6)
    assert e_ab < 1e-3


def test_multi_disk_restart(tmp_path):
    """A batch of three disks of different sizes restarts from one file per
    disk exactly as each disk restarts alone."""
    disks = []
    for nr, mach in ((16, 20.0), (24, 15.0), (12, 25.0)):
        p = par_with({"Num_R": nr, "Mach_Number": mach}, base="c0_kepler2d")
        disks.append(db.Disk.from_files(p, db.template_paths("c0_kepler2d")[1]))
        os.unlink(p)
    a = db.Batch(disks)
    a.run(6)
    a.sync()
    paths = [a.write_checkpoint(str(tmp_path / ("d%d" % d)), disk=d) for d in range(3)]
    b = db.Batch(disks, setup=False)
    b.restart(paths)
    sb = b.get_cells()
    dts = b.mindt()
    for d in range(3):
        one = db.Batch([disks[d]], setup=False)
        one.restart(paths[d])
        s1 = one.get_cells()
        lo, hi = b.offsets[d], b.offsets[d + 1]
        for k in ("prim", "piph", "dphi", "wiph"):
            assert np.array_equal(sb[k][lo:hi], s1[k]), (d, k)
        assert b.time(d) == one.time(0)
        assert np.array_equal(b.planets(d), one.planets(0))
        assert dts[d] == one.mindt()[0]


def test_restart_refusals(tmp_path):
    disk, g = _disk("ck_rigid")
    b = db.Batch([disk], setup=False)
    # another grid: the fixture's checkpoint into a disk of other Num_R
    p = par_with({"Num_R": 22, "Log_Zoning": 0, "Init_Par2": 1, "Energy_Omega": 0,
                  "Mach_Number": 5.0}, base="c0_kepler2d")
    other = db.Disk.from_files(p, os.path.join(TEMPLATES, "c0_nograv.in"))
    os.unlink(p)
    path = ck_to_npz(g, str(tmp_path / "in.npz"))
    with pytest.raises(db.DiscoError) as e:
        db.Batch([other], setup=False).restart(path)
    assert e.value.status == 1
    with pytest.raises(db.DiscoError) as e:
        b.restart(str(tmp_path / "absent.npz"))
    assert e.value.status == 9
    np.savez_compressed(tmp_path / "z.npz", **{CK_NAMES[k]: g["ck_" + k] for k in CK_NAMES})
    with pytest.raises(db.DiscoError) as e:
        b.restart(str(tmp_path / "z.npz"))
    assert e.value.status == 3
    # a planet type other than the point mass
    bad = dict(g)
    bad["ck_Planets"] = g["ck_Planets"].copy()
    bad["ck_Planets"][0, 6] = 1.0
    with pytest.raises(db.DiscoError) as e:
        b.restart(ck_to_npz(bad, str(tmp_path / "pl.npz")))
    assert e.value.status == 3
    # the state is unchanged by the refusals and a good file still restarts
    b.restart(path)
    assert b.time()[0] == g["ck_T"][0]


def test_run_cli_checkpoint_and_restart(tmp_path):
    """python -m disco_b200.run writes a checkpoint after its steps and a
    second run restarts from it: the time carries over, the step count
    starts again, and the ascii file has one line per cell."""
    import json
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    ck = str(tmp_path / "checkpoint_0001")
    base = [sys.executable, "-m", "disco_b200.run", "--template", "c0_kepler2d", "--set", "Num_R=32"]
    r1 = subprocess.run(base + ["--steps", "4", "--warmup", "1", "--checkpoint", ck,
                                "--ascii", str(tmp_path / "out")],
                        cwd=repo, check=True, capture_output=True, text=True, timeout=600)
    a = json.loads(r1.stdout.strip().splitlines()[-1])
    assert a["count_steps"] == 5 and os.path.exists(ck + ".npz")
    with open(str(tmp_path / "out.dat")) as f:
        assert sum(1 for _ in f) == a["cells"]
    r2 = subprocess.run(base + ["--steps", "4", "--warmup", "1", "--restart", ck + ".npz"],
                        cwd=repo, check=True, capture_output=True, text=True, timeout=600)
    b = json.loads(r2.stdout.strip().splitlines()[-1])
    assert b["count_steps"] == 5 and b["t"] > a["t"]
    assert np.load(ck + ".npz")["Grid/T"][0] == a["t"]
