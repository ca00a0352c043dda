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
