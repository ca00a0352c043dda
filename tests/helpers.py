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
EXT_CASES = ["c0_zg", "c0_3d", "c1_mhd3d", "c1_mhd3d_rigid"]


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


def oracle_for(disk):
    return pyoracle.Oracle(disk.params, disk.modules, disk.Nr, disk.Nz, disk.Ng, disk.Np,
                           disk.r_jph, disk.z_kph)


def rel_l1(a, b):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    den = np.sum(np.abs(b))
    return float(np.sum(np.abs(a - b)) / den) if den > 0 else float(np.sum(np.abs(a - b)))


def rel_l1_cols(a, b):
    return [rel_l1(a[:, q], b[:, q]) for q in range(a.shape[1])]
