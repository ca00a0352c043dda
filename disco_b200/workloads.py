"""Named workloads (seeded, synthetic in.par sets) used by bench.py and tests.

ragged64: 64 independent 2D Keplerian hydro disks (Euler, HLLC, PLM 1.5, RK2,
          CFL 0.5, sun gravity, fixed boundaries), each a copy of the config-0
          disk with Num_R drawn from [32, 256], Mach_Number from [10, 40] and
          its own density-noise seed; log zoning over r in [0.5, 3] gives each
          disk Np = floor(2 pi / (1 - 6^(-1/Num_R))) cells per annulus, so the
          batch is ragged across disks (~5.7M cells in total).
config0:  the single config-0 disk (Num_R = 128, 57,856 cells).
"""
import os
import tempfile

import numpy as np

from . import Disk, read_opt, read_par, template_paths


def write_par(overrides, base="c0_kepler2d", directory=None):
    """Copy a template in.par with some keys replaced; return the new path."""
    par, _ = template_paths(base)
    out = []
    with open(par) as f:
        for line in f:
            tok = line.split()
            if tok and tok[0] in overrides:
                line = "%s\t\t%s\n" % (tok[0], overrides[tok[0]])
            out.append(line)
    fd, path = tempfile.mkstemp(suffix=".par", dir=directory)
    with os.fdopen(fd, "w") as f:
        f.write("".join(out))
    return path


def ragged_specs(ndisk=64, seed=314159, rank=0):
    """(Num_R, Mach_Number, noise seed) per disk; the sizes do not depend on
    rank (fixed work per GPU), the noise seeds do."""
    rng = np.random.default_rng(seed)
    nr = rng.integers(32, 257, size=ndisk)
    mach = rng.uniform(10.0, 40.0, size=ndisk)
    seeds = seed + np.arange(ndisk) + rank * ndisk
    return [(int(a), float(b), int(c)) for a, b, c in zip(nr, mach, seeds)]


def ragged_disks(ndisk=64, seed=314159, rank=0, keep_pars=False):
    _, opt = template_paths("c0_kepler2d")
    mods = read_opt(opt)
    disks, pars = [], []
    for nr, mach, s in ragged_specs(ndisk, seed, rank):
        p = write_par({"Num_R": nr, "Mach_Number": repr(mach), "Init_Par0": s})
        disks.append(Disk(read_par(p), mods))
        if keep_pars:
            pars.append(p)
        else:
            os.unlink(p)
    return (disks, pars) if keep_pars else disks


def config0_disk():
    return Disk.from_files(*template_paths("c0_kepler2d"))


def config4_disk(nz=128):
    """The config-4 disk (3D MHD circumbinary, CT, 384 x 128 annuli); nz < 128
    takes the mid-plane slab of nz layers with the same dz."""
    par, opt = template_paths("c4_binary3d")
    if nz == 128:
        return Disk.from_files(par, opt)
    p = write_par({"Num_Z": nz, "Z_Min": -0.5 * nz / 128, "Z_Max": 0.5 * nz / 128}, base="c4_binary3d")
    try:
        return Disk.from_files(p, opt)
    finally:
        os.unlink(p)
