"""The GRMHD timestep (HYDRO = grmhd2, METRIC = schw_ks_rpz, FRAME = normal,
HLL) against the reference binary built with that module selection
(oracle/Makefile, config c3_grtorus; fixtures from tests/golden/make_golden.py).

Every operation of the step with this module set is +, -, *, / or sqrt, all
correctly rounded on both sides, and the device keeps the reference's
operation order (--fmad=false), so the set-up, the dt sequence, every field
after N steps and the face lists are compared bit for bit: the torus with
the by-cell mesh (get_omega of grmhd2 moves the cells) and on a fixed mesh,
and with the horizon boundary (Boundary/horizon.c): no inner ghosts at
r = 0.5, every annulus inside 0.7 r_H re-initialised at its midpoint each
substep and left out of the dt minimum.  The comparison covers every cell the
grid calls real, the excised ones included."""
import numpy as np
import pytest

import disco_b200 as db
from helpers import case_disk

pytestmark = pytest.mark.gpu

GR_CASES = ["c3_grtorus", "c3_grtorus_mm0", "c3_grhorizon"]


def _real(disk, g):
    """The grid's real cells; the reference's flag also drops the excised ones."""
    r = disk.real == 1
    assert (g["real"][~r] == 0).all()
    return r


@pytest.mark.parametrize("case", GR_CASES)
def test_grmhd_setup_matches_reference(case):
    disk, g = case_disk(case)
    assert disk.modules.hydro == db.HYDRO["grmhd2"]
    b = db.Batch([disk])
    st = b.get_cells()
    r = _real(disk, g)
    assert np.array_equal(st["prim"][r], g["s0_prim"][r])
    assert np.array_equal(st["cons"][r], g["s0_cons"][r])
    assert np.array_equal(st["wiph"][r], g["s0_wiph"][r])
    assert np.array_equal(st["piph"], g["s0_piph"])
    if case == "c3_grhorizon":
        ex = r & (g["real"] == 0)
        assert ex.sum() > 0
        assert np.array_equal(st["prim"], g["s0_prim"])
    b.close()


@pytest.mark.parametrize("case", GR_CASES)
def test_grmhd_steps_bitexact(case):
    disk, g = case_disk(case)
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    dts = []
    for _ in range(int(g["nsteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    b.sync()
    assert np.array_equal(np.array(dts), g["dt"]), (np.array(dts) - g["dt"])
    st = b.get_cells()
    r = _real(disk, g)
    for k in ("prim", "cons"):
        assert np.array_equal(st[k][r], g["sN_" + k][r]), k
    assert np.array_equal(st["piph"], g["sN_piph"])
    assert np.array_equal(st["dphi"][r], g["sN_dphi"][r])
    F = b.faces(0, 1)
    for k in ("iL", "iR", "LRtype"):
        assert np.array_equal(F[k], g[k]), k
    Z = b.faces(0, 2)
    for k in ("iL", "iR", "LRtype"):
        assert np.array_equal(Z[k], g["z_" + k]), k
    assert b.mindt()[0] == g["sN_dt_next"]
    b.close()


def test_grmhd_graph_run_equals_steps():
    """disco_batch_run (graph replay, dt kept on the device) against the
    host-driven loop."""
    disk, g = case_disk("c3_grtorus")
    out = []
    for graph in (False, True):
        b = db.Batch([disk], setup=False)
        b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
        b.mindt()
        if graph:
            b.run(3)
        else:
            for _ in range(3):
                b.timestep()
        b.sync()
        out.append(b.get_cells())
        b.close()
    for k in ("prim", "cons", "piph"):
        assert np.array_equal(out[0][k], out[1][k]), k


def test_grmhd_c2p_dump_reproduces_the_step():
    """disco_batch_set_gr_dump: the cons->prim inputs the step's last
    substep solved, handed to the standalone solver (disco_gr_cons2prim with
    the step's metric, gamma, floors, tol 1e-12, tail 10, cap 30), give the
    step's prims of every real cell bit for bit -- so training pairs written
    by the plain solver on these dumps are pairs of the run itself."""
    import torch
    from disco_b200.gr import GR
    disk, g = case_disk("c3_grtorus")
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"])
    buf = torch.zeros((db.GR_DUMP_ROWS, b.ncell), dtype=torch.float64, device="cuda")
    b.set_gr_dump(buf)
    for _ in range(2):
        b.timestep(b.mindt()[0])
    b.sync()
    st = b.get_cells()
    b.set_gr_dump(None)
    b.close()
    r = disk.real == 1
    idx = torch.nonzero(torch.from_numpy(r)).squeeze(1).cuda()
    cons = buf[0:9][:, idx].contiguous()
    prim = buf[9:18][:, idx].contiguous()
    x = buf[18:21][:, idx].contiguous()
    assert torch.isfinite(cons).all() and (x[0] > 0).all()
    gr = GR(gamma_law=1.3333333333333, rho_floor=0.0, p_floor=0.0, M=1.0, a=0.0, metric="schw",
            tol=1e-12, nextra=10, max_iter=30)
    gr.cons2prim(cons, x, prim)
    assert np.array_equal(prim.cpu().numpy().T, st["prim"][r])


def test_grmhd_dump_needs_grmhd():
    import torch
    disk, _ = case_disk("c0_log16")
    b = db.Batch([disk])
    buf = torch.zeros((db.GR_DUMP_ROWS, b.ncell), dtype=torch.float64, device="cuda")
    with pytest.raises(db.DiscoError) as e:
        b.set_gr_dump(buf)
    assert e.value.status == 3
    b.close()
