"""bench.py's reference arm writes its in.par files without importing the
disco_b200 package; they must describe the same disks as the GPU arm's
(disco_b200.workloads), and both arms print the same `config`."""
import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, REPO)

import bench  # noqa: E402
from disco_b200 import workloads  # noqa: E402


def test_ragged_specs_agree():
    for n in (8, 64):
        for rank in (0, 1):
            assert bench.ragged_specs(n, rank=rank) == workloads.ragged_specs(n, rank=rank)


def test_reference_pars_match_workloads(tmp_path):
    pars = bench.reference_pars("ragged8", str(tmp_path))
    for p, (nr, mach, seed) in zip(pars, workloads.ragged_specs(8)):
        ref = workloads.write_par({"Num_R": nr, "Mach_Number": repr(mach), "Init_Par0": seed})
        try:
            assert open(p).read() == open(ref).read()
        finally:
            os.unlink(ref)


def test_config_is_implementation_free():
    c = bench.workload_config("ragged64", 5490132)
    assert c["real_cells_per_gpu"] == 5490132 and c["disks_per_gpu"] == 64
    assert bench.workload_config("ragged64", 5490132) == c


def test_config4_cell_count_without_the_library():
    """The reference arm names the config-4 workload's real cells from a
    per-layer constant (Np depends on r only), without building the disk."""
    d = bench.c4_disk()
    assert d.nreal == bench.C4_REAL_PER_LAYER * bench.C4_NZ
    assert bench.c4_disk(8).nreal == bench.C4_REAL_PER_LAYER * 8
    c = bench.workload_config("config4", d.nreal)
    assert c["workload"] == "config4" and c["real_cells_per_gpu"] == d.nreal


def test_config4_slab_par_text():
    """The reference arm's 4-layer slab of config 4: the template with the
    z extent of 4 of the 128 layers."""
    text = bench.write_par_text("c4_binary3d", {"Num_Z": bench.C4_SLAB_NZ,
                                               "Z_Min": -0.5 * bench.C4_SLAB_NZ / bench.C4_NZ,
                                               "Z_Max": 0.5 * bench.C4_SLAB_NZ / bench.C4_NZ})
    kv = {l.split()[0]: l.split()[1] for l in text.splitlines() if l.split()}
    assert kv["Num_Z"] == "4" and float(kv["Z_Max"]) == 0.015625 and kv["Num_R"] == "384"
