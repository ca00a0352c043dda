"""GRMHD cons -> prim oracle, on the CPU.

The restatement (oracle/c2p_oracle.c) is pinned bit for bit against the
reference's own Hydro/grmhd2.c prim2cons and Noble-2D cons2prim built from its
sources (Schwarzschild-KS metric, normal frame, the reference's tol 1e-12,
tail 10 and cap 30).  The Kerr-KS module is checked against Schwarzschild at
a = 0 and through its own identities; the network's backward formulas are
checked against finite differences of its forward pass.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle import pyc2p

HAVE_REF = os.path.isdir(pyc2p.REF_SRC) or os.path.exists(pyc2p.REF_LIB)


def torus_par(a=0.0, amp=4e-2, seed=314159):
    tp = pyc2p.TorusPar()
    tp.M, tp.a, tp.gam = 1.0, a, 5.0 / 3.0
    tp.rc, tp.wr, tp.hr, tp.K = 12.0, 4.0, 0.3, 5e-3
    tp.rho_atm, tp.p_atm, tp.s_cut, tp.amp = 1e-4, 1e-6, 0.2, amp
    tp.B0 = tp.wr * np.sqrt(2.0 * tp.K / 100.0)
    tp.seed = seed
    return tp


def sample_states(n, a=0.0, seed=7, eps=1e-3):
    """Torus prims at random cell centres (r log in [1.5, 50], z in
    [-20, 20]), and the same prims perturbed by eps (the next step's)."""
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 3))
    x[:, 0] = np.exp(rng.uniform(np.log(1.5), np.log(50.0), n))
    x[:, 1] = rng.uniform(0, 2 * np.pi, n)
    x[:, 2] = rng.uniform(-20.0, 20.0, n)
    cells = np.arange(n, dtype=np.uint64)
    p0 = pyc2p.torus_prims(torus_par(a), x, cells)
    u = rng.uniform(-1, 1, (n, 9))
    p1 = p0 * (1.0 + eps * u)
    return x, p0, p1


@pytest.mark.skipif(not HAVE_REF, reason="reference grmhd2.c not available")
def test_prim2cons_bitexact_vs_reference():
    x, p0, p1 = sample_states(4000)
    ref = pyc2p.C2PReference()
    orc = pyc2p.C2POracle(metric=0)
    np.testing.assert_array_equal(orc.prim2cons(p1, x), ref.prim2cons(p1, x))


@pytest.mark.skipif(not HAVE_REF, reason="reference grmhd2.c not available")
@pytest.mark.parametrize("eps", [1e-3, 0.3])
def test_cons2prim_bitexact_vs_reference(eps):
    """Warm start from the previous prims, as calc_prim does (F10)."""
    x, p0, p1 = sample_states(4000, eps=eps)
    ref = pyc2p.C2PReference()
    orc = pyc2p.C2POracle(metric=0, tol=1e-12, nextra=10, max_iter=30)
    cons = ref.prim2cons(p1, x)
    pr = ref.cons2prim(cons, x, p0)
    po, it, ok, _ = orc.cons2prim(cons, x, p0)
    np.testing.assert_array_equal(po, pr)
    assert it.min() >= 11 and it.max() <= 30
    # converged cells reproduce the perturbed prims
    good = ok.astype(bool)
    assert good.mean() > 0.99
    rel = np.abs(po[good] - p1[good]).sum() / np.abs(p1[good]).sum()
    assert rel < 1e-10


def test_kerr_at_zero_spin_is_schwarzschild():
    x, p0, p1 = sample_states(2000)
    s = pyc2p.C2POracle(metric=0)
    k = pyc2p.C2POracle(metric=1, a=0.0)
    cs, ck = s.prim2cons(p1, x), k.prim2cons(p1, x)
    assert np.abs(cs - ck).max() <= 1e-13 * np.abs(cs).max()
    ps = s.cons2prim(cs, x, p0)[0]
    pk = k.cons2prim(cs, x, p0)[0]
    assert np.abs(ps - pk).sum() <= 1e-12 * np.abs(ps).sum()


@pytest.mark.parametrize("metric,a", [(0, 0.0), (1, 0.9)])
def test_round_trip(metric, a):
    """prim -> cons -> prim recovers the prims at tol 1e-10 (both metrics)."""
    x, p0, p1 = sample_states(3000, a=a, eps=1e-2)
    o = pyc2p.C2POracle(metric=metric, a=a, tol=1e-10)
    cons = o.prim2cons(p1, x)
    prim, it, ok, _ = o.cons2prim(cons, x, p0)
    assert ok.all()
    err = np.abs(prim - p1).sum(axis=0) / np.maximum(np.abs(p1).sum(axis=0), 1e-300)
    assert err.max() < 1e-9, err


def test_kerr_identities():
    """gamma_ij gamma^jk = delta, alpha^2 = 1/(1+f) and the KS lapse/shift
    reproduce g^tt = -1/alpha^2 = -(1+f) at a = 0.9 through the p2c of a
    static fluid: D = rho sqrt(gamma) alpha u^t = rho * jac, jac = 1."""
    x, p0, _ = sample_states(500, a=0.9)
    st = p0.copy()
    st[:, 2:5] = 0.0
    st[:, 5:8] = 0.0
    o = pyc2p.C2POracle(metric=1, a=0.9)
    cons = o.prim2cons(st, x)
    # static (u_i = 0): u^t = 1/alpha, D = jac * rho * u0 -> D/rho = 1/alpha
    al = cons[:, 0] / st[:, 0]
    r, z = x[:, 0], x[:, 2]
    a = 0.9
    b = r * r + z * z - a * a
    R2 = 0.5 * (b + np.sqrt(b * b + 4 * a * a * z * z))
    f = 2 * np.sqrt(R2) * R2 / (R2 * R2 + a * a * z * z)
    np.testing.assert_allclose(al, np.sqrt(1 + f), rtol=1e-13)


def test_mlp_backward_matches_finite_differences():
    orc = pyc2p.C2POracle()
    orc.lib.orc_mlp_exact(1)
    try:
        rng = np.random.default_rng(3)
        param = (rng.standard_normal(pyc2p.NPARAM) * 0.3).astype(np.float32)
        norm = np.concatenate([np.zeros(8), np.ones(8), np.zeros(2), np.ones(2)]).astype(np.float32)
        feat = rng.standard_normal((64, 8)).astype(np.float32)
        tgt = rng.standard_normal((64, 2)).astype(np.float32)
        loss, grad, _ = orc.mlp_loss_grad(param, norm, feat, tgt)
        idx = rng.choice(pyc2p.NPARAM, 60, replace=False)
        for i in idx:
            h = 1e-2
            pp = param.copy(); pp[i] += h
            pm = param.copy(); pm[i] -= h
            hp = float(pp[i]) - float(param[i])
            hm = float(param[i]) - float(pm[i])
            lp = orc.mlp_loss_grad(pp, norm, feat, tgt)[0]
            lm = orc.mlp_loss_grad(pm, norm, feat, tgt)[0]
            fd = (lp - lm) / (hp + hm)
            assert abs(fd - grad[i]) <= 1e-4 * max(1.0, abs(grad[i])) + 1e-6, (i, fd, grad[i])
    finally:
        orc.lib.orc_mlp_exact(0)
