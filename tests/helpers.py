"""Shared test helpers: golden cases, disks, comparisons."""
import os
import tempfile

import numpy as np

import disco_b200 as db
import pyoracle

TESTS = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(TESTS, "golden")
TEMPLATES = db.TEMPLATES
CASES = ["c0_log16", "c0_lin20", "c0_hll_fe_mm3", "c0_cm2", "c0_rigid"]
# MHD fixtures (Hydro/mhd.c, hlld.c): pinned to the reference binary directly;
# the C restatement oracle/oracle.c covers the Euler module only
MHD_CASES = ["c1_mhd_hlld", "c1_mhd_hllc", "c1_mhd_hll_fe", "c1_mhd_rigid"]
# zero-gradient boundaries and 3D (z faces), also pinned to the reference binary
EXT_CASES = ["c0_zg", "c0_3d", "c1_mhd3d", "c1_mhd3d_rigid", "c0_circular", "c0_cm", "c0_cm_t0",
             "c0_diag_euler", "c0_diag_euler3d", "c0_nobc_rmax", "c1_diag_mhdmri"]


def golden(case):
    return dict(np.load(os.path.join(GOLDEN, case + ".npz")))


def case_disk(case):
    g = golden(case)
    cfg = str(g["cfg"])
    return db.Disk.from_files(os.path.join(GOLDEN, case + ".par"), os.path.join(TEMPLATES, cfg + ".in")), g


def par_with(overrides, base="c0_kepler2d"):
    """Write a copy of a template in.par with some keys replaced; returns its path."""
    out = []
    with open(os.path.join(TEMPLATES, base + ".par")) as f:
        for line in f:
            key = line.split()[0] if line.split() else ""
            if key in overrides:
                line = "%s\t\t%s\n" % (key, overrides[key])
            out.append(line)
    fd, path = tempfile.mkstemp(suffix=".par")
    with os.fdopen(fd, "w") as f:
        f.write("".join(out))
    return path


def observed_slots(disk, nfs):
    """Mask (ncell x nfs) of the face-flux slots Phi real cells read under
    constrained transport: Phi[0] of real cells and the owned-face slots of
    every track next to a real annulus.  The other slots (ghost cells' own
    faces towards further ghosts) follow edge fields the reference leaves
    stale, and nothing reads them."""
    Nr, Nz, Ng = disk.Nr, disk.Nz, disk.Ng
    jk = np.repeat(np.arange(Nr * Nz), disk.Np)
    j, k = jk % Nr, jk // Nr
    rj = (j >= Ng[0]) & (j < Nr - Ng[1])
    rk = (k >= Ng[2]) & (k < Nz - Ng[3])
    m = np.zeros((disk.ncell, nfs), bool)
    m[:, 0] = disk.real == 1
    m[:, 1] = (j >= Ng[0]) & (j <= Nr - Ng[1]) & rk
    m[:, 2] = (j >= Ng[0] - 1) & (j <= Nr - Ng[1] - 1) & rk
    if nfs == 5 and Nz > 1:
        m[:, 3] = rj & (k >= Ng[2]) & (k <= Nz - Ng[3])
        m[:, 4] = rj & (k >= Ng[2] - 1) & (k <= Nz - Ng[3] - 1)
    return m


def oracle_for(disk):
    return pyoracle.Oracle(disk.params, disk.modules, disk.Nr, disk.Nz, disk.Ng, disk.Np,
                           disk.r_jph, disk.z_kph)


def rel_l1(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    den = np.sum(np.abs(b))
    return float(np.sum(np.abs(a - b)) / den) if den > 0 else float(np.sum(np.abs(a - b)))


def rel_l1_cols(a, b):
    return [rel_l1(a[:, q], b[:, q]) for q in range(a.shape[1])]


CKPT_CASES = ["ck_cm2", "ck_rigid", "ck_ct_rigid", "ck_ct3d_rigid", "ck_noise"]
CK_NAMES = {"T": "Grid/T", "r_jph": "Grid/r_jph", "z_kph": "Grid/z_kph", "Index": "Grid/Index",
            "Np": "Grid/Np", "Id_phi0": "Grid/Id_phi0", "Cells": "Data/Cells",
            "Planets": "Data/Planets", "Diagnostics": "Data/Diagnostics"}


def ck_to_npz(g, path):
    """The reference's checkpoint datasets of a ck_* fixture as the .npz
    container (written by numpy, under the HDF5 dataset paths)."""
    np.savez(path, **{CK_NAMES[k]: g["ck_" + k] for k in CK_NAMES})
    return path


def ck_to_raw(g, d):
    """The same datasets as oracle/ref_checkpoint.c's raw directory."""
    os.makedirs(d, exist_ok=True)
    NzT, NrT = g["ck_Np"].shape
    Nc, Nq = g["ck_Cells"].shape
    Npl, NpDat = g["ck_Planets"].shape
    with open(os.path.join(d, "dims.txt"), "w") as f:
        f.write("%d %d %d %d %d %d %d\n" % (NrT, NzT, Nc, Nq, Npl, NpDat, g["ck_Diagnostics"].shape[2]))
    for k in CK_NAMES:
        a = g["ck_" + k]
        a.astype(np.int32 if a.dtype.kind == "i" else np.float64).tofile(
            os.path.join(d, k + (".i32" if a.dtype.kind == "i" else ".f64")))
    return d
