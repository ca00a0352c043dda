"""ORACLE TEST INFRASTRUCTURE -- not part of the product.

Python bindings for the GRMHD cons -> prim oracle: the CPU restatement
oracle/c2p_oracle.c (liboracle_c2p.so) and the reference's own grmhd2.c
state conversions built by `make -C oracle c2p` (oracle/_ref/c2p/libc2p_ref.so,
behind oracle/c2p_ref.c).  Used by tests/ and bench.py as the checker only.

States are AoS here (n x 9 prims/cons, n x 3 positions), as the reference
passes them one cell at a time.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liboracle_c2p.so")
REF_LIB = os.path.join(HERE, "_ref", "c2p", "libc2p_ref.so")
# the reference source tree the oracle builds compile; DISCO_REF overrides it
REF_SRC = os.environ.get("DISCO_REF", "/root/reference")

NPARAM = 64 * 8 + 64 + 64 * 64 + 64 + 2 * 64 + 2
NNORM = 2 * 8 + 2 * 2

_D = C.POINTER(C.c_double)
_F = C.POINTER(C.c_float)
_I = C.POINTER(C.c_int)


def build_c2p_oracle(force=False):
    """Compile c2p_oracle.c into oracle/liboracle_c2p.so (-O3, no FMA)."""
    src = os.path.join(HERE, "c2p_oracle.c")
    deps = [src, os.path.join(REPO, "disco_b200", "csrc", "gr_torus.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    subprocess.run(["gcc", "-O3", "-fPIC", "-shared", "-std=gnu11", "-ffp-contract=off",
                    src, "-o", LIB + ".tmp", "-lm"], check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_c2p_ref():
    """Build the reference's grmhd2.c conversions (needs the reference tree)."""
    if not os.path.isdir(REF_SRC):
        if os.path.exists(REF_LIB):
            return REF_LIB
        raise FileNotFoundError("reference tree absent and oracle/_ref/c2p not built")
    subprocess.run(["make", "-s", "-C", HERE, "c2p", "REF=" + REF_SRC], check=True, stdout=subprocess.DEVNULL)
    return REF_LIB


def _p(a, t):
    return a.ctypes.data_as(t)


class C2POracle:
    """The restatement, metric 0 (Schwarzschild-KS) or 1 (Kerr-KS, spin a)."""

    def __init__(self, gam=5.0 / 3.0, rho_floor=1e-10, p_floor=1e-10, M=1.0, a=0.0,
                 metric=0, tol=1e-12, nextra=10, max_iter=30):
        self.lib = C.CDLL(build_c2p_oracle())
        self.lib.orc_gr_setup.argtypes = [C.c_double] * 5 + [C.c_int, C.c_double, C.c_int, C.c_int]
        self.lib.orc_mlp_loss_grad.restype = C.c_double
        self.args = (gam, rho_floor, p_floor, M, a, metric, tol, nextra, max_iter)

    def _setup(self):
        self.lib.orc_gr_setup(*self.args)

    def prim2cons(self, prim, x):
        self._setup()
        prim = np.ascontiguousarray(prim, np.float64); x = np.ascontiguousarray(x, np.float64)
        cons = np.empty_like(prim)
        self.lib.orc_gr_prim2cons(C.c_long(len(prim)), _p(prim, _D), _p(x, _D), _p(cons, _D))
        return cons

    def cons2prim(self, cons, x, guess):
        """Warm-start solve from the prims `guess`: (prim, iters, ok, (v2, eta))."""
        self._setup()
        n = len(cons)
        cons = np.ascontiguousarray(cons, np.float64); x = np.ascontiguousarray(x, np.float64)
        prim = np.array(guess, np.float64, copy=True, order="C")
        it = np.zeros(n, np.int32); ok = np.zeros(n, np.int32); fin = np.zeros((n, 2))
        self.lib.orc_gr_cons2prim(C.c_long(n), _p(cons, _D), _p(x, _D), _p(prim, _D),
                                  _p(it, _I), _p(ok, _I), _p(fin, _D))
        return prim, it, ok, fin

    def newton_from(self, cons, x, v2eta):
        self._setup()
        n = len(cons)
        cons = np.ascontiguousarray(cons, np.float64); x = np.ascontiguousarray(x, np.float64)
        g = np.ascontiguousarray(v2eta, np.float64)
        prim = np.zeros((n, 9)); it = np.zeros(n, np.int32); ok = np.zeros(n, np.int32)
        self.lib.orc_gr_newton_from(C.c_long(n), _p(cons, _D), _p(x, _D), _p(g, _D),
                                    _p(prim, _D), _p(it, _I), _p(ok, _I))
        return prim, it, ok

    def features(self, cons, x, guess):
        """(features[n, 8], sigma[n], warm start (v2_0, eta_0)[n, 2]) of the learned guess."""
        self._setup()
        n = len(cons)
        cons = np.ascontiguousarray(cons, np.float64); x = np.ascontiguousarray(x, np.float64)
        guess = np.ascontiguousarray(guess, np.float64)
        f = np.zeros((n, 8), np.float32)
        sg = np.zeros(n)
        wm = np.zeros((n, 2))
        self.lib.orc_gr_features(C.c_long(n), _p(cons, _D), _p(x, _D), _p(guess, _D), _p(f, _F),
                                 _p(sg, _D), _p(wm, _D))
        return f, sg, wm

    def mlp_loss_grad(self, param, norm, feat, target=None):
        """(loss, grad[NPARAM] float64, out[n,2]) in double precision."""
        param = np.ascontiguousarray(param, np.float32); norm = np.ascontiguousarray(norm, np.float32)
        feat = np.ascontiguousarray(feat, np.float32)
        n = len(feat)
        out = np.zeros((n, 2))
        grad = np.zeros(NPARAM) if target is not None else None
        t = np.ascontiguousarray(target, np.float32) if target is not None else None
        loss = self.lib.orc_mlp_loss_grad(C.c_long(n), _p(param, _F), _p(norm, _F), _p(feat, _F),
                                          _p(t, _F) if t is not None else None,
                                          _p(grad, _D) if grad is not None else None, _p(out, _D))
        return loss, grad, out


class TorusPar(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("M", "a", "gam", "rc", "wr", "hr", "K",
                                          "rho_atm", "p_atm", "B0", "s_cut", "amp")] + \
               [("seed", C.c_uint64)]


def torus_prims(tp, x, cells):
    """The torus module on the CPU (same header the device uses)."""
    lib = C.CDLL(build_c2p_oracle())
    x = np.ascontiguousarray(x, np.float64)
    cells = np.ascontiguousarray(cells, np.uint64)
    prim = np.zeros((len(x), 9))
    lib.orc_gr_torus(C.byref(tp), C.c_long(len(x)), _p(x, _D),
                     cells.ctypes.data_as(C.POINTER(C.c_uint64)), _p(prim, _D))
    return prim


class C2PReference:
    """The reference's grmhd2.c (Schwarzschild-KS, normal frame), one cell per
    call exactly as calc_prim makes them; its tolerance, tail and cap are the
    reference's constants (1e-12, 10, 30)."""

    def __init__(self, gam=5.0 / 3.0, rho_floor=1e-10, p_floor=1e-10, M=1.0):
        self.lib = C.CDLL(build_c2p_ref())
        self.lib.ref_c2p_setup.argtypes = [C.c_double] * 4
        self.args = (gam, rho_floor, p_floor, M)

    def prim2cons(self, prim, x):
        self.lib.ref_c2p_setup(*self.args)
        prim = np.ascontiguousarray(prim, np.float64); x = np.ascontiguousarray(x, np.float64)
        cons = np.empty_like(prim)
        self.lib.ref_prim2cons(C.c_int(len(prim)), _p(prim, _D), _p(x, _D), _p(cons, _D))
        return cons

    def cons2prim(self, cons, x, guess):
        self.lib.ref_c2p_setup(*self.args)
        cons = np.ascontiguousarray(cons, np.float64); x = np.ascontiguousarray(x, np.float64)
        prim = np.array(guess, np.float64, copy=True, order="C")
        self.lib.ref_cons2prim(C.c_int(len(cons)), _p(cons, _D), _p(x, _D), _p(prim, _D))
        return prim
