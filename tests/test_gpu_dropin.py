"""The drop-in: the reference's own host code (read_par_file, setupGrid,
setupDomain, setupCells, boundary_trans -- everything but timestep() and
getmindt()) linked with disco_b200/shim, i.e. the link-time substitution
a Disco maintainer makes, against the unmodified reference binary.  The
driver calls the shim's disco_gpu_init after set-up, as a host would.

Both binaries are built from the reference sources by oracle/Makefile
(targets disco_ref and hybrid) wherever the reference tree is available."""
import os
import shutil
import subprocess
import tempfile

import numpy as np
import pytest

import pyoracle
from helpers import GOLDEN, ck_to_raw, golden, rel_l1_cols

pytestmark = pytest.mark.gpu


def _run(binary, par, nsteps, report=False, env_extra=None, par_over=None):
    work = tempfile.mkdtemp(prefix="dropin_")
    try:
        with open(par) as f:
            text = f.read()
        for k, v in (par_over or {}).items():     # e.g. Restart 1
            text = "".join("%s\t\t%s\n" % (k, v) if line.split()[:1] == [k] else line
                           for line in text.splitlines(True))
        with open(os.path.join(work, "in.par"), "w") as f:
            f.write(text)
        dump = os.path.join(work, "dump")
        env = dict(os.environ, **(env_extra or {}))
        if report:
            env["DISCO_REF_REPORT"] = "1"
        subprocess.run([binary, work, str(nsteps), dump], check=True,
                       stdout=subprocess.DEVNULL, timeout=600, env=env)
        out = pyoracle.load_dump(dump)
        if report:
            with open(os.path.join(work, "report.dat")) as f:
                out["report"] = np.array([float(x) for x in f.read().split()])
        return out
    finally:
        shutil.rmtree(work, ignore_errors=True)


def _binaries(cfg):
    ref = pyoracle.ref_binary(cfg)
    hyb = os.path.join(os.path.dirname(ref), "disco_hybrid")
    if not (os.path.exists(ref) and os.path.exists(hyb)):
        pytest.skip("reference / hybrid binaries for %s not built" % cfg)
    return ref, hyb


def test_dropin_bitexact_libm_free():
    ref, hyb = _binaries("c0_nograv")
    par = os.path.join(GOLDEN, "c0_rigid.par")
    a, b = _run(ref, par, 10), _run(hyb, par, 10)
    assert np.array_equal(a["dt"], b["dt"])
    for k in ("prim", "piph", "dphi", "wiph"):
        assert np.array_equal(a[k], b[k]), k
    r = a["real"] == 1
    assert np.array_equal(a["cons"][r], b["cons"][r])
    for k in ("iL", "iR", "LRtype"):
        assert np.array_equal(a["faces_1"][k], b["faces_1"][k]), k
    assert a["dt_next"] == b["dt_next"]
    # the shim's own exports: the device's face lists (disco_gpu_get_faces)
    # equal the reference's, and disco_gpu_last_error / disco_gpu_free ran
    for k in ("iL", "iR"):
        assert np.array_equal(b["gpu_faces_1"][k], a["faces_1"][k]), k


def test_dropin_grmhd_bitexact():
    """The GRMHD module selection (grmhd2, schw_ks_rpz, normal frame, HLL,
    fixed3d, the gr_torus_noise torus) through the drop-in: the reference's
    own setupCells and boundaries on the host, every step on the device."""
    ref, hyb = _binaries("c3_grtorus")
    par = os.path.join(GOLDEN, "c3_grtorus.par")
    a, b = _run(ref, par, 5), _run(hyb, par, 5)
    assert np.array_equal(a["dt"], b["dt"])
    r = a["real"] == 1
    for k in ("prim", "cons"):
        assert np.array_equal(a[k][r], b[k][r]), k
    for k in ("piph", "dphi"):
        assert np.array_equal(a[k], b[k]), k
    for k in ("iL", "iR", "LRtype"):
        assert np.array_equal(a["faces_1"][k], b["faces_1"][k]), k
    assert a["dt_next"] == b["dt_next"]


def test_dropin_config0_20_steps():
    ref, hyb = _binaries("c0_kepler2d")
    import disco_b200 as db
    par, _ = db.template_paths("c0_kepler2d")
    a, b = _run(ref, par, 20), _run(hyb, par, 20)
    assert np.max(np.abs(b["dt"] / a["dt"] - 1)) < 1e-12
    r = a["real"] == 1
    assert max(rel_l1_cols(b["prim"][r], a["prim"][r])) < 1e-12
    assert max(rel_l1_cols(b["cons"][r], a["cons"][r])) < 1e-12
    for k in ("iL", "iR", "LRtype"):
        assert np.array_equal(a["faces_1"][k], b["faces_1"][k]), k
    assert np.max(np.abs(b["Qrz"] - a["Qrz"])) <= 1e-12 * np.max(np.abs(a["Qrz"]))


@pytest.mark.parametrize("cfg,case,n", [("c1_mhd2d_nograv", "c1_ct_rigid", 8),
                                        ("c1_mhd3d_nograv", "c1_ct3d_rigid", 6)])
def test_dropin_constrained_transport_bitexact(cfg, case, n):
    """Constrained transport through the drop-in (2D CT_MODE 1, 3D CT_MODE 2):
    the reference's own set_B_fields on the host, then the device steps; the
    face-flux slots real cells read travel both ways through the shim."""
    ref, hyb = _binaries(cfg)
    par = os.path.join(GOLDEN, case + ".par")
    a, b = _run(ref, par, n), _run(hyb, par, n)
    assert np.array_equal(a["dt"], b["dt"])
    r = a["real"] == 1
    for k in ("prim", "cons"):
        assert np.array_equal(a[k][r], b[k][r]), k
    for k in ("piph", "dphi", "wiph"):
        assert np.array_equal(a[k], b[k]), k
    m = a["meta"]
    Nr, Nz = m["Nr"], m["Nz"]
    jk = np.repeat(np.arange(Nr * Nz), a["Np"])
    j, k = jk % Nr, jk // Nr
    rj = (j >= m["NgRa"]) & (j < Nr - m["NgRb"])
    rk = (k >= m["NgZa"]) & (k < Nz - m["NgZb"])
    assert np.array_equal(a["Phi"][r, 0], b["Phi"][r, 0])
    masks = {1: (j >= m["NgRa"]) & (j <= Nr - m["NgRb"]) & rk,
             2: (j >= m["NgRa"] - 1) & (j <= Nr - m["NgRb"] - 1) & rk}
    if a["Phi"].shape[1] == 5:
        masks[3] = rj & (k >= m["NgZa"]) & (k <= Nz - m["NgZb"])
        masks[4] = rj & (k >= m["NgZa"] - 1) & (k <= Nz - m["NgZb"] - 1)
    for s, mk in masks.items():
        assert np.array_equal(a["Phi"][mk, s], b["Phi"][mk, s]), s


@pytest.mark.parametrize("cfg,par", [("c0_cm2", "c0_cm2.par"), ("c1_mhd2d_nograv", "c1_ct_rigid.par")])
def test_dropin_report(cfg, par):
    """report() through the drop-in: the line computed on the device from the
    resident state against the reference's report.c on its own state (both
    printed with %le, 6 significant digits): binary torque terms (cm2) and
    the magnetic terms (MHD with CT)."""
    ref, hyb = _binaries(cfg)
    p = os.path.join(GOLDEN, par)
    a, b = _run(ref, p, 6, report=True), _run(hyb, p, 6, report=True)
    ra, rb = a["report"], b["report"]
    assert len(ra) == len(rb) == 17
    for n, (x, y) in enumerate(zip(ra, rb)):
        if np.isinf(x) or np.isinf(y):          # bM = PdV / B2 without a field
            assert x == y, (n, x, y)
        else:
            assert abs(x - y) <= 5e-6 * abs(x) + 1e-300, (n, x, y)


def test_dropin_restart_from_checkpoint(tmp_path):
    """A run restarted by the reference's own set-up (setupCells with Restart
    1; the checkpoint read by oracle/ref_checkpoint.c in place of h5in.c) and
    continued through the drop-in: the shim uploads the checkpoint's planets
    (the binary has moved since initializePlanets), so 4 steps match the
    reference restarted from the same file, planets included."""
    ref, hyb = _binaries("c0_cm2")
    g = golden("ck_cm2")
    raw = ck_to_raw(g, str(tmp_path / "ck"))
    par = os.path.join(GOLDEN, "ck_cm2.par")
    b = _run(hyb, par, int(g["msteps"]), env_extra={"DISCO_REF_RESTART": raw},
             par_over={"Restart": 1})
    r = g["real"] == 1
    assert np.max(np.abs(b["dt"] / g["rM_dt"] - 1)) < 1e-11
    assert max(rel_l1_cols(b["prim"][r], g["rM_prim"][r])) < 1e-11
    assert abs(b["meta"]["t"] / g["rM_t"] - 1) < 1e-12
    assert np.abs(b["planets"] - g["rM_planets"]).max() < 1e-11
    # the planets really moved: a restart that re-initialised them would not match
    assert np.abs(g["rM_planets"][:, 4] - np.array([np.pi, 0.0])).min() > 0.1


def test_dropin_ascii_output(tmp_path):
    """The reference's ascii output module through the drop-in, after the
    device state is copied back (disco_gpu_sync_to_host): byte for byte the
    reference's file for the libm-free case."""
    ref, hyb = _binaries("c0_nograv")
    g = golden("ck_rigid")
    out = str(tmp_path / "ascii")
    _run(hyb, os.path.join(GOLDEN, "ck_rigid.par"), int(g["nsteps"]),
         env_extra={"DISCO_REF_ASCII": out})
    with open(out + ".dat", "rb") as f:
        assert f.read() == bytes(g["ascii"])


def test_dropin_polar():
    """A grid down to the axis with the polar boundary module through the
    drop-in (the shim maps BOUNDARY polar), against the reference binary."""
    ref, hyb = _binaries("c0_polar")
    par = os.path.join(GOLDEN, "c0_polar.par")
    a, b = _run(ref, par, 10), _run(hyb, par, 10)
    assert np.max(np.abs(b["dt"] / a["dt"] - 1)) < 1e-12
    r = a["real"] == 1
    assert max(rel_l1_cols(b["prim"][r], a["prim"][r])) < 1e-12
    for k in ("iL", "iR", "LRtype"):
        assert np.array_equal(a["faces_1"][k], b["faces_1"][k]), k


def test_dropin_reference_initial_module():
    """A reference Initial module (Initial/rigid.c) the device does not have:
    the host set-up evaluates it, the shim runs the steps with zero-gradient
    boundaries (which never call initial() again) -- bit for bit with the
    reference binary over 10 steps (no libm call in the steps)."""
    ref, hyb = _binaries("c0_rigid_zg")
    par = os.path.join(GOLDEN, "c0_rigid_zg.par")
    a, b = _run(ref, par, 10), _run(hyb, par, 10)
    assert np.array_equal(a["dt"], b["dt"])
    r = a["real"] == 1
    for k in ("prim", "piph", "dphi"):
        assert np.array_equal(a[k][r], b[k][r]), k
