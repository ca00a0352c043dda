"""report() on the device (disco_batch_report) against the reference's
report.c formulas (report.c:60-193) evaluated in numpy on the same state: MHD
without planets, after the fixture's steps.  The torque terms (two planets)
are compared with the reference binary itself through the drop-in
(test_gpu_dropin.py::test_dropin_report)."""
import numpy as np
import pytest

import disco_b200 as db
from helpers import case_disk

pytestmark = pytest.mark.gpu


def report_numpy(disk, st, t, gam, mhd):
    """report.c's loop over the real cells, in numpy (host libm)."""
    Nr, Nz, Ng = disk.Nr, disk.Nz, disk.Ng
    rj, zk = disk.r_jph, disk.z_kph          # index 0 is edge -1
    off = np.concatenate([[0], np.cumsum(disk.Np)])
    acc = dict.fromkeys(["PsiR", "PsiI", "L1_isen", "L1_rho", "L1_B", "Br2", "BrBp", "B2", "PdV",
                         "Mdot", "Vol", "Mass", "S_R", "S_0"], 0.0)
    rho_min = np.inf
    rhoavg_min = np.inf
    for j in range(Ng[0], Nr - Ng[1]):
        arho = avol = 0.0
        for k in range(Ng[2], Nz - Ng[3]):
            a = j + Nr * k
            c = np.arange(off[a], off[a + 1])
            p = st["prim"][c]
            piph, dphi = st["piph"][c], st["dphi"][c]
            phi = piph - .5 * dphi
            dph = piph - (piph - dphi)
            rp, rm, zp, zm = rj[j + 1], rj[j], zk[k + 1], zk[k]
            dV = (.5 * (rp + rm)) * (rp - rm) * dph * (zp - zm)
            r = 2.0 * (rp * rp + rp * rm + rm * rm) / (3.0 * (rp + rm))
            rho, Pp, vr = p[:, 0], p[:, 1], p[:, 2]
            acc["PsiR"] += np.sum(rho * dV * np.cos(phi))
            acc["PsiI"] += np.sum(rho * dV * np.sin(phi))
            acc["L1_isen"] += np.sum(np.abs(Pp / rho ** gam - 1.) * dV)
            acc["L1_rho"] += np.sum(np.abs(rho - 1.) * dV)
            if mhd:
                Br, Bp, Bz = p[:, 5], p[:, 6], p[:, 7]
                acc["L1_B"] += np.sum(np.abs(Br) * dV)
                acc["Br2"] += np.sum(.5 * Br * Br * dV)
                acc["BrBp"] += np.sum(Br * Bp * dV)
                acc["B2"] += np.sum(.5 * (Br * Br + Bp * Bp + Bz * Bz) * dV)
            acc["PdV"] += np.sum(Pp * dV)
            acc["Mdot"] += np.sum(2. * np.pi * r * rho * dV * vr)
            acc["Vol"] += np.sum(dV)
            acc["Mass"] += np.sum(rho * dV)
            acc["S_R"] += np.sum(rho ** 4. * r * dV)
            acc["S_0"] += np.sum(rho ** 4. * dV)
            rho_min = min(rho_min, rho.min())
            arho += np.sum(rho * dV)
            avol += np.sum(dV)
        rhoavg_min = min(rhoavg_min, arho / avol)
    V = acc["Vol"]
    return np.array([t, 0.0, 0.0, 0.0, rho_min, rhoavg_min, acc["PsiR"], acc["PsiI"], acc["Mass"],
                     acc["Mdot"] / V, acc["S_R"] / acc["S_0"], acc["L1_rho"] / V, acc["L1_isen"] / V,
                     acc["L1_B"] / V, acc["Br2"], acc["BrBp"] / acc["PdV"],
                     acc["PdV"] / acc["B2"] if acc["B2"] else np.inf])


@pytest.mark.parametrize("case", ["c1_ct_rigid", "c1_mhd_hlld"])
def test_report_matches_formulas(case):
    disk, g = case_disk(case)
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"],
                Phi=g.get("s0_Phi"))
    b.run(int(g["nsteps"]))
    b.sync()
    st = b.get_cells()
    t, _ = b.time()
    got = b.report()
    want = report_numpy(disk, st, t, disk.params.Adiabatic_Index, True)
    for n, name in enumerate(db.Batch.REPORT_FIELDS):
        x, y = got[n], want[n]
        # the cos / sin weighted sums nearly cancel: measured against the mass
        tol = 1e-12 * (abs(want[8]) if name in ("PsiR", "PsiI") else abs(y))
        assert abs(x - y) <= tol + 1e-300, (name, x, y)
