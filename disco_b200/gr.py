"""GRMHD cons -> prim on the GPU: Python host mirror of include/disco_c2p.h.

In the reference, calc_prim (misc.c:290-325) loops over the real cells and
calls the Hydro module's cons2prim(cons, prim, x, dV) (Hydro/grmhd2.c:253),
whose Noble-2D Newton solve starts from the cell's previous prims.  Here the
loop is one launch over device arrays (torch tensors, structure of arrays):

    gr = GR(metric="kerr", a=0.9, tol=1e-10)
    x = gr.grid(192, 96, 462, 1.5, 50.0, -20.0, 20.0)     # (3, n) cell centres
    prim = gr.torus(x)                                    # (9, n)
    cons = gr.prim2cons(gr.perturb(prim, seed=1, eps=1e-3), x)
    rep = gr.cons2prim(cons, x, prim)                     # prim := solution

    pairs = gr.cons2prim(cons, x, prim0, pairs=True)["pairs"]   # training data
    gr.mlp_init(1); gr.mlp_fit_norm(pairs); gr.mlp_train(pairs, 2000, 4096)
    rep = gr.cons2prim(cons, x, prim, guess="learned")

There is no CPU fallback: without the built library or a CUDA device every
call raises DiscoError.
"""
import ctypes as C

import numpy as np

from . import DiscoError, library

NPARAM = 4866
NNORM = 20
GUESS = {"previous": 0, "learned": 1}
METRIC = {"schw": 0, "kerr": 1}


class GRParams(C.Structure):
    """Mirror of disco_gr_params."""
    _fields_ = [("gamma_law", C.c_double), ("rho_floor", C.c_double), ("p_floor", C.c_double),
                ("M", C.c_double), ("a", C.c_double), ("tol", C.c_double),
                ("metric", C.c_int), ("nextra", C.c_int), ("max_iter", C.c_int), ("pad", C.c_int)]


class GRStats(C.Structure):
    """Mirror of disco_gr_stats."""
    _fields_ = [("ncell", C.c_int64), ("iters_sum", C.c_int64), ("iters_max", C.c_int),
                ("n_fallback", C.c_int), ("n_fail", C.c_int), ("pad", C.c_int),
                ("hist", C.c_int64 * 64)]


class Torus(C.Structure):
    """Mirror of disco_gr_torus (disco_b200/csrc/gr_torus.h)."""
    _fields_ = [(k, C.c_double) for k in ("M", "a", "gam", "rc", "wr", "hr", "K",
                                          "rho_atm", "p_atm", "B0", "s_cut", "amp")] + \
               [("seed", C.c_uint64)]


def torus_defaults(a=0.9, amp=4e-2, seed=314159, beta=100.0):
    """The torus of the GRMHD workload: centre r = 12 M, width 4 M, h/r 0.3,
    K = 5e-3 (P/rho ~ 5e-3 at the centre), atmosphere rho 1e-4 R^-3/2,
    P 1e-6 R^-5/2, loop field with beta ~ `beta` at the centre, pressure
    noise `amp`."""
    t = Torus()
    t.M, t.a, t.gam = 1.0, a, 5.0 / 3.0
    t.rc, t.wr, t.hr, t.K = 12.0, 4.0, 0.3, 5e-3
    t.rho_atm, t.p_atm, t.s_cut, t.amp = 1e-4, 1e-6, 0.2, amp
    t.B0 = t.wr * np.sqrt(2.0 * t.K / beta)
    t.seed = seed
    return t


_sig_done = False


def _lib():
    global _sig_done
    lib = library()
    if _sig_done:
        return lib
    P, I, L, D = C.c_void_p, C.c_int, C.c_long, C.c_double
    sig = {
        "disco_gr_create": (I, [I, C.POINTER(GRParams), C.POINTER(P)]),
        "disco_gr_destroy": (None, [P]),
        "disco_gr_set_stream": (I, [P, P]),
        "disco_gr_last_error": (C.c_char_p, [P]),
        "disco_gr_grid": (I, [P, I, I, I, D, D, D, D, I, P]),
        "disco_gr_torus_prims": (I, [P, C.POINTER(Torus), L, P, P]),
        "disco_gr_perturb": (I, [P, L, P, P, C.c_uint64, D]),
        "disco_gr_prim2cons": (I, [P, L, P, P, P]),
        "disco_gr_cons2prim": (I, [P, L, P, P, P, I, P, P, C.POINTER(GRStats)]),
        "disco_gr_mlp_init": (I, [P, C.c_uint64]),
        "disco_gr_mlp_set": (I, [P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "disco_gr_mlp_get": (I, [P, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "disco_gr_mlp_fit_norm": (I, [P, L, P]),
        "disco_gr_mlp_grad": (I, [P, L, P, C.POINTER(C.c_float), C.POINTER(C.c_double)]),
        "disco_gr_mlp_train": (I, [P, L, P, I, I, C.c_float, C.c_uint64, C.POINTER(C.c_double)]),
        "disco_gr_mlp_set_backend": (I, [P, I]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _sig_done = True
    return lib


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class GR:
    """One GRMHD cons -> prim context (parameters, network, scratch) on a GPU."""

    def __init__(self, device=0, gamma_law=5.0 / 3.0, rho_floor=1e-10, p_floor=1e-10, M=1.0,
                 a=0.0, metric="schw", tol=1e-12, nextra=10, max_iter=30):
        import torch
        self.torch = torch
        self.lib = _lib()
        self.device = device
        self.h = None
        p = GRParams(gamma_law, rho_floor, p_floor, M, a, tol, METRIC[metric], nextra, max_iter, 0)
        h = C.c_void_p()
        self._check(self.lib.disco_gr_create(device, C.byref(p), C.byref(h)), "disco_gr_create")
        self.h = h
        self.params = p

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.disco_gr_destroy(self.h)
            self.h = None

    def _check(self, st, where):
        if st != 0:
            msg = self.lib.disco_gr_last_error(self.h).decode() if getattr(self, "h", None) else ""
            raise DiscoError(st, where + (": " + msg if msg else ""))

    def _dev(self, a, dtype):
        t = self.torch
        if not isinstance(a, t.Tensor):
            a = t.from_numpy(np.ascontiguousarray(a))
        return a.to(device="cuda:%d" % self.device, dtype=dtype).contiguous()

    def set_stream(self, stream):
        """Launch on a torch.cuda.Stream (or a raw cudaStream_t int)."""
        s = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
        self._check(self.lib.disco_gr_set_stream(self.h, C.c_void_p(s)), "set_stream")

    # ---- states ------------------------------------------------------
    def grid(self, Nr, Nz, Np, rmin, rmax, zmin, zmax, log_r=True):
        n = Nr * Nz * Np
        x = self.torch.empty((3, n), dtype=self.torch.float64, device="cuda:%d" % self.device)
        self._check(self.lib.disco_gr_grid(self.h, Nr, Nz, Np, rmin, rmax, zmin, zmax, int(log_r),
                                           _ptr(x)), "grid")
        return x

    def torus(self, x, tp=None):
        tp = tp or torus_defaults(a=self.params.a)
        x = self._dev(x, self.torch.float64)
        n = x.shape[1]
        prim = self.torch.empty((9, n), dtype=self.torch.float64, device=x.device)
        self._check(self.lib.disco_gr_torus_prims(self.h, C.byref(tp), n, _ptr(x), _ptr(prim)), "torus")
        return prim

    def perturb(self, prim, seed, eps):
        prim = self._dev(prim, self.torch.float64)
        out = self.torch.empty_like(prim)
        self._check(self.lib.disco_gr_perturb(self.h, prim.shape[1], _ptr(prim), _ptr(out), seed, eps),
                    "perturb")
        return out

    # ---- the conversions --------------------------------------------
    def prim2cons(self, prim, x):
        prim = self._dev(prim, self.torch.float64)
        x = self._dev(x, self.torch.float64)
        cons = self.torch.empty_like(prim)
        self._check(self.lib.disco_gr_prim2cons(self.h, prim.shape[1], _ptr(prim), _ptr(x), _ptr(cons)),
                    "prim2cons")
        return cons

    def cons2prim(self, cons, x, prim, guess="previous", iters=False, pairs=False, stats=True):
        """Solve in place: `prim` (a (9, n) float64 CUDA tensor) holds the
        previous prims on entry and the solution on return.  Returns a dict
        with the iteration report and, if asked, the per-cell iteration
        counts and training pairs (n, 10)."""
        t = self.torch
        n = cons.shape[1]
        it = t.empty(n, dtype=t.uint8, device=cons.device) if iters else None
        pr = t.empty((n, 10), dtype=t.float32, device=cons.device) if pairs else None
        st = GRStats()
        self._check(self.lib.disco_gr_cons2prim(self.h, n, _ptr(cons), _ptr(x), _ptr(prim), GUESS[guess],
                                                _ptr(it), _ptr(pr), C.byref(st) if stats else None),
                    "cons2prim")
        out = {}
        if stats:
            out.update(ncell=st.ncell, iters_mean=st.iters_sum / max(st.ncell, 1),
                       iters_max=st.iters_max, n_fallback=st.n_fallback, n_fail=st.n_fail,
                       hist=np.array(st.hist[:], dtype=np.int64))
        if iters:
            out["iters"] = it
        if pairs:
            out["pairs"] = pr
        return out

    # ---- the network -------------------------------------------------
    def mlp_init(self, seed=1):
        self._check(self.lib.disco_gr_mlp_init(self.h, seed), "mlp_init")

    def mlp_set(self, param, norm):
        p = np.ascontiguousarray(param, np.float32)
        q = np.ascontiguousarray(norm, np.float32)
        assert p.size == NPARAM and q.size == NNORM
        self._check(self.lib.disco_gr_mlp_set(self.h, p.ctypes.data_as(C.POINTER(C.c_float)),
                                              q.ctypes.data_as(C.POINTER(C.c_float))), "mlp_set")

    def mlp_get(self):
        p = np.zeros(NPARAM, np.float32)
        q = np.zeros(NNORM, np.float32)
        self._check(self.lib.disco_gr_mlp_get(self.h, p.ctypes.data_as(C.POINTER(C.c_float)),
                                              q.ctypes.data_as(C.POINTER(C.c_float))), "mlp_get")
        return p, q

    def mlp_fit_norm(self, pairs):
        self._check(self.lib.disco_gr_mlp_fit_norm(self.h, pairs.shape[0], _ptr(pairs)), "mlp_fit_norm")

    def mlp_grad(self, pairs):
        pairs = self._dev(pairs, self.torch.float32)
        g = np.zeros(NPARAM, np.float32)
        loss = C.c_double()
        self._check(self.lib.disco_gr_mlp_grad(self.h, pairs.shape[0], _ptr(pairs),
                                               g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)),
                    "mlp_grad")
        return loss.value, g

    def mlp_backend(self, backend):
        """"tensor" (tcgen05 MMAs, the default) or "cuda" (the FP32 CUDA-core
        backward) for mlp_grad / mlp_train."""
        self._check(self.lib.disco_gr_mlp_set_backend(self.h, {"cuda": 0, "tensor": 1}[backend]),
                    "mlp_set_backend")

    def mlp_train(self, pairs, steps, batch=4096, lr=2e-3, seed=1):
        hist = np.zeros(steps)
        self._check(self.lib.disco_gr_mlp_train(self.h, pairs.shape[0], _ptr(pairs), steps, batch, lr, seed,
                                                hist.ctypes.data_as(C.POINTER(C.c_double))), "mlp_train")
        return hist


def _main(argv=None):
    """Demo and profiling case: torus on an Nr x Nz x Np grid, pairs from one
    plain solve, a short training run, then plain and learned solves of a
    fresh perturbation; prints the iteration report of both."""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m disco_b200.gr")
    ap.add_argument("--nr", type=int, default=64)
    ap.add_argument("--nz", type=int, default=32)
    ap.add_argument("--np", type=int, default=462)
    ap.add_argument("--eps", type=float, default=0.3)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--nextra", type=int, default=10)
    a = ap.parse_args(argv)
    gr = GR(metric="kerr", a=0.9, tol=1e-10, nextra=a.nextra, max_iter=30)
    x = gr.grid(a.nr, a.nz, a.np, 1.5, 50.0, -20.0, 20.0)
    p0 = gr.torus(x)
    cons = gr.prim2cons(gr.perturb(p0, 103, a.eps), x)
    pairs = gr.cons2prim(cons, x, p0.clone(), pairs=True, stats=False)["pairs"]
    gr.mlp_init(3)
    gr.mlp_fit_norm(pairs)
    gr.mlp_train(pairs, steps=a.steps, batch=8192, lr=2e-3, seed=9)
    cons = gr.prim2cons(gr.perturb(p0, 777, a.eps), x)
    out = {"ncell": int(x.shape[1])}
    for guess in ("previous", "learned"):
        rep = gr.cons2prim(cons, x, p0.clone(), guess=guess)
        out[guess] = {k: rep[k] for k in ("iters_mean", "iters_max", "n_fallback", "n_fail")}
    print(json.dumps(out))


if __name__ == "__main__":
    _main()
