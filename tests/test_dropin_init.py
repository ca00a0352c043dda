"""disco_gpu_init, the drop-in's explicit upload: a module selection the
device does not run is refused with a status before any CUDA call, so this
runs without a GPU.  The hybrid binary is the reference's own host code
linked with disco_b200/shim (oracle/Makefile target hybrid) for a config-0
disk whose Analysis module is diag_grmhdmri: its diagnostics are not
computed on the device, so the upload must refuse it (DISCO_ERR_UNSUPPORTED)
rather than run without them."""
import os
import shutil
import subprocess
import tempfile

import pytest

import pyoracle
from helpers import par_with


def test_gpu_init_refuses_unsupported_analysis():
    hyb = os.path.join(os.path.dirname(pyoracle.ref_binary("c0_grdiag")), "disco_hybrid")
    if not os.path.exists(hyb):
        pytest.skip("hybrid binary for c0_grdiag not built")
    work = tempfile.mkdtemp(prefix="gpuinit_")
    try:
        par = par_with({"Num_R": 16})
        shutil.move(par, os.path.join(work, "in.par"))
        r = subprocess.run([hyb, work, "1", "--time"], capture_output=True, text=True, timeout=120)
        assert r.returncode == 4, r.stderr
        assert "disco_gpu_init: status 3" in r.stderr      # DISCO_ERR_UNSUPPORTED
        assert "seconds" not in r.stdout                    # no step ran
    finally:
        shutil.rmtree(work, ignore_errors=True)
