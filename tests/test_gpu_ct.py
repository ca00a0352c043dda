"""GPU parity of constrained transport (Constrained_Transport 1) against the
reference's own build (bfields.c, riemann.c edge bookkeeping, onestep.c:
140-185), from the fixtures of tests/golden/make_golden.py: CT_MODE 1 in 2D
and CT_MODE 2 in 3D (z faces, E_phi edges, make_edge_adjust).

The CT state is the per-cell face-flux array Phi[NUM_FACES] (Phi[0] the phi
face at piph, Phi[1] / Phi[2] the r face the cell owns in the track inside /
outside it, Phi[3] / Phi[4] the z face below / above it).  The comparison
covers every slot a real cell reads: Phi[0] of real cells and the owned-face
slots of every track next to a real annulus; the remaining slots (ghost
cells' own faces towards further ghosts) follow edge fields the reference
leaves stale and reach nothing.

- c1_ct_rigid, c1_ct3d_rigid (no gravity, so no libm call whose value
  matters): bit-exact, state, slots, dt sequence and face lists.
- c1_ct2d, c1_ct3d (Keplerian, point-mass gravity) and c1_ct_hll_fe (HLL,
  forward Euler, by-cell mesh): relative L1 1e-11 (the libm differences of
  the point-mass force, as for the other MHD fixtures), face lists bit-exact.
- At full size, the property CT exists for: each real cell's discrete
  divergence (net flux through its faces) stays at its initial value to
  round-off (the reference's own runs keep it to 1e-17 of 1e-4), in 2D and
  in 3D.
"""
import os

import numpy as np
import pytest

import disco_b200 as db
from helpers import case_disk, observed_slots as _observed_slots, par_with, rel_l1, rel_l1_cols

pytestmark = pytest.mark.gpu

# c4_binary3d: config 4's module set with the softened binary
# (Planets/binary_soft.c in the reference build)
# c1_ct3d_zpole, c1_polar3d_zpole: 3D CT with z boundaries without ghost
# layers (avg_Efields' z-pole average, k_ct_zpole); the polar one also down
# to the axis (polar sources call sin: 1e-12)
CT_CASES = ["c1_ct2d", "c1_ct_rigid", "c1_ct_hll_fe", "c1_ct3d", "c1_ct3d_rigid", "c4_binary3d",
            "c1_ct3d_zpole", "c1_polar3d_zpole"]
CT_TOL = {"c1_ct2d": 1e-11, "c1_ct_hll_fe": 1e-11, "c1_ct3d": 1e-11, "c4_binary3d": 1e-11,
          "c1_polar3d_zpole": 1e-12}


def _from_golden(disk, g):
    b = db.Batch([disk], setup=False)
    b.set_cells(g["s0_prim"], g["s0_cons"], g["s0_piph"], g["s0_dphi"], g["s0_wiph"], g["real"],
                Phi=g["s0_Phi"])
    return b


def divergence(b, disk):
    """Net magnetic flux out of each cell through its current faces: outer
    r faces - inner r faces (+ upper z faces - lower z faces) + Phi[0](c) -
    Phi[0](c-1)."""
    st = b.get_cells()
    Phi = st["Phi"]
    div = np.zeros(disk.ncell)
    dims = [(1, 2, 1)] + ([(2, 4, 3)] if disk.Nz > 1 and Phi.shape[1] == 5 else [])
    for dim, s0, s1 in dims:
        F = b.faces(0, dim)
        L, R, lr = F["iL"], F["iR"], F["LRtype"]
        v = np.where(lr == 0, Phi[L, s0], Phi[R, s1])
        np.add.at(div, L, v)
        np.add.at(div, R, -v)
    off = np.concatenate([[0], np.cumsum(disk.Np)])
    for a in range(len(disk.Np)):
        c = np.arange(off[a], off[a + 1])
        div[c] += Phi[c, 0] - Phi[np.roll(c, 1), 0]
    return div, Phi


@pytest.mark.parametrize("case", CT_CASES)
def test_ct_setup_matches_reference(case):
    """set_B_fields + B_faces_to_cells + cons2prim on the device reproduce the
    reference's step-0 state bit for bit."""
    disk, g = case_disk(case)
    b = db.Batch([disk])
    st = b.get_cells()
    r = disk.real == 1
    assert np.array_equal(st["prim"][r], g["s0_prim"][r])
    assert np.array_equal(st["cons"][r], g["s0_cons"][r])
    m = _observed_slots(disk, b.num_faces)
    assert np.array_equal(st["Phi"][m], g["s0_Phi"][m])
    assert b.mindt()[0] == g["s0_dt_next"]


@pytest.mark.parametrize("case", CT_CASES)
def test_ct_steps_match_reference(case):
    disk, g = case_disk(case)
    b = _from_golden(disk, g)
    dts = []
    for _ in range(int(g["nsteps"])):
        dt = b.mindt()[0]
        dts.append(dt)
        b.timestep(dt)
    b.sync()
    st = b.get_cells()
    r = disk.real == 1
    m = _observed_slots(disk, b.num_faces)
    F = b.faces(0, 1)
    for k in ("fIndex", "iL", "iR", "LRtype"):
        assert np.array_equal(F[k], g[k]), k
    if disk.Nz > 1:
        Fz = b.faces(0, 2)
        for k in ("fIndex", "iL", "iR", "LRtype"):
            assert np.array_equal(Fz[k], g["z_" + k]), ("z", k)
    if case not in CT_TOL:
        assert np.array_equal(np.array(dts), g["dt"])
        assert np.array_equal(st["prim"][r], g["sN_prim"][r])
        assert np.array_equal(st["cons"][r], g["sN_cons"][r])
        assert np.array_equal(st["Phi"][m], g["sN_Phi"][m])
        return
    tol = CT_TOL[case]
    assert np.max(np.abs(np.array(dts) / g["dt"] - 1.0)) < tol
    for q, e in enumerate(rel_l1_cols(st["prim"][r], g["sN_prim"][r])):
        assert e < tol, ("prim", q, e)
    for q, e in enumerate(rel_l1_cols(st["cons"][r], g["sN_cons"][r])):
        assert e < tol, ("cons", q, e)
    for s in range(m.shape[1]):
        if m[:, s].any():
            e = rel_l1(st["Phi"][m[:, s], s], g["sN_Phi"][m[:, s], s])
            assert e < tol, ("Phi", s, e)


def _ct_disk(nr, ct):
    _, opt = db.template_paths("c1_mhd2d")
    p = par_with({"Num_R": nr, "Constrained_Transport": ct, "Init_Par5": 20.0,
                  "Init_Par6": 0.05, "Init_Par1": 0.05}, base="c1_mhd2d")
    disk = db.Disk.from_files(p, opt)
    os.unlink(p)
    return disk


def test_ct_preserves_divergence():
    """128 annuli (about 70k cells), 40 steps of the Keplerian disk with
    shear, so faces flip in every step: the discrete divergence of each
    real cell is unchanged to round-off under CT."""
    disk = _ct_disk(128, 1)
    b = db.Batch([disk])
    d0, P0 = divergence(b, disk)
    F0 = b.faces(0, 1)
    b.run(40)
    b.sync()
    d1, P1 = divergence(b, disk)
    F1 = b.faces(0, 1)
    # the sliding annuli have re-paired their faces (flips happened)
    assert not np.array_equal(F0["iR"], F1["iR"])
    r = disk.real == 1
    scale = np.abs(P1).max()
    drift = np.abs(d1 - d0)[r].max()
    print("div drift %.3e of max |Phi| %.3e (initial max |div| %.3e)" % (drift, scale, np.abs(d0[r]).max()))
    assert drift <= 1e-12 * scale
    assert np.abs(P1[r, 1:]).max() > 1.5 * np.abs(P0[r, 1:]).max()   # the field did evolve


def test_ct3d_preserves_divergence():
    """3D: 24 annuli x 16 layers of the Keplerian disk, 20 steps; r, z and
    phi faces and the E_phi edges all take part."""
    _, opt = db.template_paths("c1_mhd3d")
    p = par_with({"Num_R": 24, "Num_Z": 16, "Constrained_Transport": 1, "Init_Par5": 20.0,
                  "Init_Par6": 0.05, "Init_Par1": 0.05}, base="c1_mhd3d")
    disk = db.Disk.from_files(p, opt)
    os.unlink(p)
    b = db.Batch([disk])
    d0, P0 = divergence(b, disk)
    b.run(20)
    b.sync()
    d1, P1 = divergence(b, disk)
    r = disk.real == 1
    scale = np.abs(P1).max()
    drift = np.abs(d1 - d0)[r].max()
    print("3D div drift %.3e of max |Phi| %.3e (initial max |div| %.3e)" % (drift, scale, np.abs(d0[r]).max()))
    assert drift <= 1e-12 * scale


def test_ct_refuses_unsupported():
    """CT_MODE 1 stores no z-face fluxes: refused in 3D."""
    _, opt = db.template_paths("c1_mhd3d")
    p = par_with({"Num_R": 8, "Num_Z": 6, "Constrained_Transport": 1}, base="c1_mhd3d")
    disk = db.Disk.from_files(p, opt)
    os.unlink(p)
    disk.modules.ct_mode = 1
    with pytest.raises(db.DiscoError) as e:
        db.Batch([disk])
    assert e.value.status == 3


TOL_MIXED_CT = 1e-5


@pytest.mark.parametrize("base,nr,nz,steps", [("c1_mhd2d", 64, 1, 40), ("c1_mhd3d", 24, 16, 20)])
def test_ct_mixed_form(base, nr, nz, steps):
    """The mixed form with CT: FP32 edge arithmetic, FP64 face fluxes.  Against
    FP64 CT from the same set-up, density and pressure within the mixed form's
    stated 1e-5 relative L1; its own discrete div B kept to FP64 round-off (the
    face-flux updates are FP64 and CT's structure conserves it whatever the
    edge values' precision)."""
    _, opt = db.template_paths(base)
    over = {"Num_R": nr, "Constrained_Transport": 1, "Init_Par5": 20.0, "Init_Par6": 0.05}
    if nz > 1:
        over["Num_Z"] = nz
    p = par_with(over, base=base)
    disk = db.Disk.from_files(p, opt)
    os.unlink(p)
    a = db.Batch([disk], precision=db.PREC_FP64)
    m = db.Batch([disk], precision=db.PREC_MIXED)
    dm0, _ = divergence(m, disk)
    a.run(steps)
    m.run(steps)
    a.sync()
    m.sync()
    sa, sm = a.get_cells(), m.get_cells()
    r = disk.real == 1
    err = {q: rel_l1(sm["prim"][r, q], sa["prim"][r, q]) for q in (0, 1, 3)}
    dm1, Pm = divergence(m, disk)
    drift = np.abs(dm1 - dm0)[r].max() / np.abs(Pm).max()
    print("%s mixed CT vs FP64 CT: rel L1 rho %.2e P %.2e Omega %.2e; div drift %.2e of max |Phi|"
          % (base, err[0], err[1], err[3], drift))
    assert max(err.values()) < TOL_MIXED_CT, err
    assert drift <= 1e-12
