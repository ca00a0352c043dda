"""The persistent one-launch step (disco_step_persist.cuh) against the
multi-kernel step: both run the same block bodies, so after several steps of
a multi-disk batch every field, the face lists, the time and the
diagnostics must be identical bit for bit, in the FP64 path and in the mixed
form.  The ragged batch has annuli of several blocks and disks of different
sizes, so blocks of one annulus, of neighbouring annuli and of different
disks run at different times in the persistent schedule."""
import numpy as np
import pytest

import disco_b200 as db
from disco_b200 import workloads

pytestmark = pytest.mark.gpu


def _pair(disks, prec, nsteps):
    out = []
    for sched in (db.SCHED_KERNELS, db.SCHED_PERSISTENT):
        b = db.Batch(disks, precision=prec)
        b.schedule = sched
        assert b.schedule == sched
        b.run(nsteps)
        b.sync()
        st = b.get_cells()
        st["faces"] = b.faces(0, 1)
        st["faces_last"] = b.faces(len(disks) - 1, 1)
        st["time"] = [b.time(d) for d in range(len(disks))]
        st["dt"] = b.mindt()
        st["diag"] = b.diagnostics(0)[0]
        b.close()
        out.append(st)
    return out


@pytest.mark.parametrize("prec", [db.PREC_FP64, db.PREC_MIXED])
def test_persistent_step_equals_kernels(prec):
    disks = workloads.ragged_disks(6)
    a, p = _pair(disks, prec, 4)
    for k in ("prim", "cons", "piph", "dphi", "wiph"):
        assert np.array_equal(a[k], p[k]), k
    for key in ("faces", "faces_last"):
        for k in ("iL", "iR", "LRtype"):
            assert np.array_equal(a[key][k], p[key][k]), (key, k)
    assert a["time"] == p["time"]
    assert np.array_equal(a["dt"], p["dt"])
    assert np.array_equal(a["diag"], p["diag"])


def test_schedule_selection():
    b = db.Batch([workloads.config0_disk()])
    assert b.schedule == db.SCHED_KERNELS          # the default
    b.schedule = db.SCHED_PERSISTENT
    assert b.schedule == db.SCHED_PERSISTENT
    b.close()
    # 3D (z faces) runs on the multi-kernel path and refuses the persistent one
    disk = db.Disk.from_files(*db.template_paths("c1_mhd3d"))
    b = db.Batch([disk])
    assert b.schedule == db.SCHED_KERNELS
    with pytest.raises(db.DiscoError):
        b.schedule = db.SCHED_PERSISTENT
    b.close()


def test_persistent_single_disk_long_run():
    """config 0 for 50 steps, persistent against multi-kernel."""
    disk = workloads.config0_disk()
    a, p = _pair([disk], db.PREC_FP64, 50)
    for k in ("prim", "cons", "piph", "dphi"):
        assert np.array_equal(a[k], p[k]), k
