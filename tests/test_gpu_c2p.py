"""GRMHD cons -> prim on the GPU against the oracle (oracle/c2p_oracle.c,
itself pinned to the reference's grmhd2.c), and the learned guess.

- prim2cons and the warm-start Noble-2D solve: bit-exact with the oracle
  (Schwarzschild-KS and Kerr-KS a = 0.9), iteration counts identical; and
  bit-exact with the reference's own grmhd2.c where its build is present.
- Network gradients from the training kernels against the oracle's double
  forward/backward with the same BF16 weights (relative L2 <= 1e-3: the GPU
  accumulates in FP32 and its FP32 activations can round to a neighbouring
  BF16 value).
- Learned vs plain: both run Newton to the same tol and tail; the solutions
  agree to 1e-12 and the trained network cuts the iteration count where the
  previous prims are a poor start.
"""
import numpy as np
import pytest

from oracle import pyc2p

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _gr(**kw):
    from disco_b200.gr import GR
    return GR(**kw)


def _states(n, a, eps, seed=11):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 3))
    x[:, 0] = np.exp(rng.uniform(np.log(1.5), np.log(50.0), n))
    x[:, 1] = rng.uniform(0, 2 * np.pi, n)
    x[:, 2] = rng.uniform(-20.0, 20.0, n)
    tp = pyc2p.TorusPar()
    from disco_b200.gr import torus_defaults
    t = torus_defaults(a=a)
    for k, _ in pyc2p.TorusPar._fields_:
        setattr(tp, k, getattr(t, k))
    p0 = pyc2p.torus_prims(tp, x, np.arange(n, dtype=np.uint64))
    p1 = p0 * (1.0 + eps * rng.uniform(-1, 1, (n, 9)))
    return x, p0, p1


def _soa(a):
    return torch.from_numpy(np.ascontiguousarray(a.T)).cuda()


def _aos(t):
    return t.cpu().numpy().T.copy()


@pytest.mark.parametrize("metric,a", [("schw", 0.0), ("kerr", 0.9)])
@pytest.mark.parametrize("eps", [1e-3, 0.3])
def test_c2p_bitexact_vs_oracle(metric, a, eps):
    n = 20000
    x, p0, p1 = _states(n, a, eps)
    orc = pyc2p.C2POracle(metric=0 if metric == "schw" else 1, a=a, tol=1e-12, nextra=10, max_iter=30)
    cons = orc.prim2cons(p1, x)
    gr = _gr(metric=metric, a=a, tol=1e-12, nextra=10, max_iter=30)
    cg = gr.prim2cons(_soa(p1), _soa(x))
    np.testing.assert_array_equal(_aos(cg), cons)
    prim_o, it_o, ok_o, _ = orc.cons2prim(cons, x, p0)
    pg = _soa(p0)
    rep = gr.cons2prim(_soa(cons), _soa(x), pg, iters=True)
    np.testing.assert_array_equal(_aos(pg), prim_o)
    np.testing.assert_array_equal(rep["iters"].cpu().numpy().astype(np.int32), it_o)
    assert rep["n_fail"] == int(np.sum(ok_o == 0))
    assert rep["iters_max"] == it_o.max()
    assert abs(rep["iters_mean"] - it_o.mean()) < 1e-9
    assert rep["hist"].sum() == n


def test_c2p_bitexact_vs_reference():
    try:
        ref = pyc2p.C2PReference()
    except (FileNotFoundError, OSError) as e:
        pytest.skip("reference grmhd2.c build absent: %s" % e)
    x, p0, p1 = _states(20000, 0.0, 1e-2)
    cons = ref.prim2cons(p1, x)
    gr = _gr(metric="schw", tol=1e-12, nextra=10, max_iter=30)
    np.testing.assert_array_equal(_aos(gr.prim2cons(_soa(p1), _soa(x))), cons)
    pg = _soa(p0)
    gr.cons2prim(_soa(cons), _soa(x), pg)
    np.testing.assert_array_equal(_aos(pg), ref.cons2prim(cons, x, p0))


def test_torus_module_matches_cpu():
    gr = _gr(metric="kerr", a=0.9)
    x = gr.grid(8, 6, 32, 1.5, 50.0, -20.0, 20.0)
    pg = _aos(gr.torus(x))
    from disco_b200.gr import torus_defaults
    t = torus_defaults(a=0.9)
    tp = pyc2p.TorusPar()
    for k, _ in pyc2p.TorusPar._fields_:
        setattr(tp, k, getattr(t, k))
    pc = pyc2p.torus_prims(tp, _aos(x), np.arange(x.shape[1], dtype=np.uint64))
    assert np.all(np.abs(pg - pc) <= 1e-13 * np.abs(pc) + 1e-300)


def _pairs_from_runs(gr, x, p0, seeds_eps):
    out = []
    for seed, eps in seeds_eps:
        p1 = gr.perturb(p0, seed, eps)
        cons = gr.prim2cons(p1, x)
        pr = p0.clone()
        out.append(gr.cons2prim(cons, x, pr, pairs=True)["pairs"])
    return torch.cat(out)


# gradient tolerances against the oracle's double forward / backward: the
# CUDA-core backward keeps dA2 / dA1 in FP32; the tensor-core one
# (tcgen05.mma) takes them as BF16 operands, as the forward's activations
GRAD_TOL = {"cuda": (1e-3, 2e-3), "tensor": (1e-3, 5e-3)}


@pytest.mark.parametrize("backend", ["tensor", "cuda"])
def test_mlp_gradient_vs_oracle(backend):
    gr = _gr(metric="kerr", a=0.9, tol=1e-10)
    gr.mlp_backend(backend)
    x = gr.grid(16, 8, 64, 1.5, 50.0, -20.0, 20.0)
    p0 = gr.torus(x)
    pairs = _pairs_from_runs(gr, x, p0, [(5, 1e-2), (6, 0.3)])
    gr.mlp_init(7)
    gr.mlp_fit_norm(pairs)
    sel = pairs[torch.isfinite(pairs).all(dim=1)][:4096].contiguous()
    loss_g, grad_g = gr.mlp_grad(sel)
    param, norm = gr.mlp_get()
    s = sel.cpu().numpy()
    t = ((s[:, 8:10] - norm[16:18]) / norm[18:20]).astype(np.float32)
    orc = pyc2p.C2POracle()
    loss_o, grad_o, _ = orc.mlp_loss_grad(param, norm, s[:, :8], t)
    assert abs(loss_g / loss_o - 1) < 1e-5, (loss_g, loss_o)
    tol, tol_block = GRAD_TOL[backend]
    rel = np.linalg.norm(grad_g - grad_o) / np.linalg.norm(grad_o)
    print(backend, "gradient rel L2 %.2e" % rel)
    assert rel < tol, rel
    # each layer's block on its own
    for lo, hi in [(0, 512), (512, 576), (576, 4672), (4672, 4736), (4736, 4864), (4864, 4866)]:
        r = np.linalg.norm(grad_g[lo:hi] - grad_o[lo:hi]) / max(np.linalg.norm(grad_o[lo:hi]), 1e-30)
        assert r < tol_block, (lo, hi, r)


def test_mlp_tensor_core_gradient_repeatable():
    """The tcgen05 backward called again and again on the same pairs gives the
    same gradient up to the order of the blocks' float atomics: a race in the
    kernel's tile set-up or MMA hand-offs shows as an occasional call far
    from the others (one such race once put the output layer's bias
    gradient 36x off in a single call)."""
    gr = _gr(metric="kerr", a=0.9, tol=1e-10)
    gr.mlp_backend("tensor")
    x = gr.grid(16, 8, 64, 1.5, 50.0, -20.0, 20.0)
    p0 = gr.torus(x)
    pairs = _pairs_from_runs(gr, x, p0, [(5, 1e-2), (6, 0.3)])
    gr.mlp_init(7)
    gr.mlp_fit_norm(pairs)
    sel = pairs[torch.isfinite(pairs).all(dim=1)].contiguous()
    l0, g0 = gr.mlp_grad(sel)
    worst = 0.0
    for _ in range(24):
        l1, g1 = gr.mlp_grad(sel)
        assert abs(l1 / l0 - 1) < 1e-9, (l1, l0)
        worst = max(worst, float(np.linalg.norm(g1 - g0) / np.linalg.norm(g0)))
    print("tensor gradient, 25 calls: largest rel L2 difference %.2e" % worst)
    assert worst < 1e-5, worst


def test_mlp_tensor_core_gradient_matches_cuda_cores():
    """The tcgen05 backward against the CUDA-core one on the same pairs and
    network, over many 128-sample groups per block (the tensor-memory
    accumulators carry across groups), and both trainings converge."""
    gr = _gr(metric="kerr", a=0.9, tol=1e-10)
    x = gr.grid(32, 16, 96, 1.5, 50.0, -20.0, 20.0)
    p0 = gr.torus(x)
    pairs = _pairs_from_runs(gr, x, p0, [(11, 1e-2), (12, 0.3)])
    gr.mlp_init(5)
    gr.mlp_fit_norm(pairs)
    sel = pairs[torch.isfinite(pairs).all(dim=1)].contiguous()
    assert sel.shape[0] > 128 * 2 * 148 * 2          # several groups per block
    out = {}
    for backend in ("cuda", "tensor"):
        gr.mlp_backend(backend)
        out[backend] = gr.mlp_grad(sel)
    (lc, gc), (lt, gt) = out["cuda"], out["tensor"]
    assert abs(lt / lc - 1) < 1e-5, (lt, lc)
    rel = np.linalg.norm(gt - gc) / np.linalg.norm(gc)
    print("tensor vs CUDA cores: rel L2 %.2e" % rel)
    assert rel < 1e-2, rel
    for backend in ("tensor", "cuda"):
        gr.mlp_init(5)
        gr.mlp_fit_norm(pairs)
        gr.mlp_backend(backend)
        hist = gr.mlp_train(sel, steps=300, batch=4096, lr=2e-3, seed=3)
        assert hist[-20:].mean() < 0.2 * hist[:5].mean(), (backend, hist[:5], hist[-20:])


def test_learned_without_network_is_refused():
    from disco_b200 import DiscoError
    gr = _gr(metric="kerr", a=0.9)
    x = gr.grid(2, 2, 8, 1.5, 50.0, -20.0, 20.0)
    p = gr.torus(x)
    c = gr.prim2cons(p, x)
    with pytest.raises(DiscoError) as e:
        gr.cons2prim(c, x, p.clone(), guess="learned")
    assert e.value.status == 7


def test_learned_guess_gain():
    """Train on pairs from plain solves, then solve fresh states both ways
    at tol 1e-10 with the reference's tail (10) and cap (30)."""
    gr = _gr(metric="kerr", a=0.9, tol=1e-10, nextra=10, max_iter=30)
    x = gr.grid(48, 24, 128, 1.5, 50.0, -20.0, 20.0)
    p0 = gr.torus(x)
    pairs = _pairs_from_runs(gr, x, p0, [(101, 1e-3), (102, 3e-2), (103, 0.3), (104, 0.1)])
    gr.mlp_init(3)
    gr.mlp_fit_norm(pairs)
    hist = gr.mlp_train(pairs, steps=1500, batch=4096, lr=2e-3, seed=9)
    assert hist[-50:].mean() < 0.2 * hist[:20].mean(), (hist[:5], hist[-5:])
    rows = []
    for eps in (1e-3, 0.3):
        p1 = gr.perturb(p0, 777, eps)
        cons = gr.prim2cons(p1, x)
        a, b = p0.clone(), p0.clone()
        ra = gr.cons2prim(cons, x, a, guess="previous", iters=True)
        rb = gr.cons2prim(cons, x, b, guess="learned")
        good = ra["iters"] < 30          # cells the plain solve converged on
        d = (a - b)[:, good].abs().sum(dim=1) / a[:, good].abs().sum(dim=1).clamp_min(1e-300)
        rows.append((eps, ra["iters_mean"], rb["iters_mean"], ra["iters_max"], rb["iters_max"],
                     rb["n_fallback"], ra["n_fail"], rb["n_fail"], float(d.max())))
        assert rb["n_fail"] <= ra["n_fail"]
        assert float(d.max()) < 1e-12, d
    for r in rows:
        print("eps %.0e: iters plain %.3f learned %.3f (max %d/%d), fallbacks %d, fails %d/%d, rel L1 %.1e" % r)
    # the jump case: the previous prims are far from the solution; in the
    # warm case the network must not cost iterations
    assert rows[1][2] < rows[1][1] - 0.7, rows
    assert rows[0][2] <= rows[0][1] + 0.05, rows


def test_pairs_match_oracle():
    """The training pairs a plain solve writes: features against the
    oracle's (float logs on both sides, __logf on the device), targets
    against the oracle's converged (v2, eta) scaled by sigma."""
    n = 20000
    x, p0, p1 = _states(n, 0.9, 0.1)
    orc = pyc2p.C2POracle(metric=1, a=0.9, tol=1e-10, nextra=10, max_iter=30)
    cons = orc.prim2cons(p1, x)
    f_o, sg, wm = orc.features(cons, x, p0)
    _, _, ok, fin = orc.cons2prim(cons, x, p0)
    gr = _gr(metric="kerr", a=0.9, tol=1e-10, nextra=10, max_iter=30)
    pr = gr.cons2prim(_soa(cons), _soa(x), _soa(p0), pairs=True)["pairs"].cpu().numpy()
    np.testing.assert_allclose(pr[:, :8], f_o, rtol=2e-5, atol=2e-5)
    good = ok.astype(bool)
    t0 = np.log1p((fin[:, 1] - wm[:, 1]) / wm[:, 1]) / sg
    t1 = (fin[:, 0] - wm[:, 0]) / sg
    np.testing.assert_allclose(pr[good, 8], t0[good], rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(pr[good, 9], t1[good], rtol=1e-6, atol=1e-6)
    assert np.all(np.isnan(pr[~good, 8]))
