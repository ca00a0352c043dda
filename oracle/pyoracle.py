"""ORACLE TEST INFRASTRUCTURE -- not part of the product.

Python bindings for the oracle: the CPU restatement liboracle.so (oracle.c)
and the reference binaries oracle/_ref/<cfg>/disco_ref built from the
reference's own sources by oracle/Makefile.  Used only by tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg, as the checker.
"""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liboracle.so")
# the reference source tree the oracle builds compile; DISCO_REF overrides it
REF_SRC = os.environ.get("DISCO_REF", "/root/reference")


def build_oracle(force=False):
    """Compile oracle.c into oracle/liboracle.so (plain C, -O3, no FMA)."""
    src = os.path.join(HERE, "oracle.c")
    deps = [src, os.path.join(HERE, "oracle.h"),
            os.path.join(REPO, "disco_b200", "csrc", "ic_kepler_noise.h"),
            os.path.join(REPO, "include", "disco_b200.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    cmd = ["gcc", "-O3", "-fPIC", "-shared", "-std=gnu11", "-ffp-contract=off",
           "-I" + os.path.join(REPO, "include"), "-I" + os.path.join(REPO, "disco_b200", "csrc"),
           src, "-o", LIB + ".tmp", "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def ref_binary(cfg):
    return os.path.join(HERE, "_ref", cfg, "disco_ref")


def build_ref(cfg):
    """Build oracle/_ref/<cfg>/disco_ref from the reference sources (needs the tree)."""
    if not os.path.isdir(REF_SRC):
        if os.path.exists(ref_binary(cfg)):
            return ref_binary(cfg)
        raise FileNotFoundError("reference tree absent and oracle/_ref/%s not built" % cfg)
    subprocess.run(["make", "-s", "-C", HERE, "CFG=" + cfg, "REF=" + REF_SRC, "-j8"], check=True,
                   stdout=subprocess.DEVNULL)
    return ref_binary(cfg)


def load_dump(d):
    meta = {}
    with open(os.path.join(d, "meta.txt")) as f:
        for line in f:
            k, v = line.split()
            meta[k] = float(v) if "." in v or "e" in v else int(v)
    Q, N = meta["Q"], meta["Ncell"]
    rd = lambda n, t: np.fromfile(os.path.join(d, n), dtype=t)
    out = dict(meta=meta, Np=rd("Np.i32", np.int32), r_jph=rd("r_jph.f64", np.float64),
               z_kph=rd("z_kph.f64", np.float64),
               prim=rd("prim.f64", np.float64).reshape(N, Q), cons=rd("cons.f64", np.float64).reshape(N, Q),
               piph=rd("piph.f64", np.float64), dphi=rd("dphi.f64", np.float64),
               wiph=rd("wiph.f64", np.float64), real=rd("real.i32", np.int32),
               dt=rd("dt.f64", np.float64), Qrz=rd("Qrz.f64", np.float64),
               dt_next=rd("dt_next.f64", np.float64)[0])
    if os.path.exists(os.path.join(d, "planets.f64")):
        out["planets"] = rd("planets.f64", np.float64).reshape(-1, 7)
    if os.path.exists(os.path.join(d, "gpu_faces_1.i32")):      # the drop-in's own face lists
        out["gpu_faces_1"] = dict(iL=rd("gpu_faces_1.i32", np.int32), iR=rd("gpu_facesR_1.i32", np.int32))
    if meta.get("num_faces", 0) > 0 and os.path.exists(os.path.join(d, "Phi.f64")):
        out["Phi"] = rd("Phi.f64", np.float64).reshape(N, meta["num_faces"])
    for dim in (1, 2):
        fn = os.path.join(d, "faces_%d.i32" % dim)
        if os.path.exists(fn):
            idx = rd("faces_%d.i32" % dim, np.int32).reshape(-1, 3)
            out["faces_%d" % dim] = dict(fIndex=rd("fIndex_%d.i32" % dim, np.int32), iL=idx[:, 0],
                                         iR=idx[:, 1], LRtype=idx[:, 2],
                                         geom=rd("faces_%d.f64" % dim, np.float64).reshape(-1, 8))
    return out


def run_ref(cfg, par_text_or_path, nsteps, keep=None):
    """Run the reference for nsteps from its own set-up; return the dump dict."""
    binary = build_ref(cfg)
    work = tempfile.mkdtemp(prefix="disco_ref_")
    try:
        par = os.path.join(work, "in.par")
        if os.path.exists(par_text_or_path):
            shutil.copy(par_text_or_path, par)
        else:
            with open(par, "w") as f:
                f.write(par_text_or_path)
        dump = os.path.join(work, "dump")
        subprocess.run([binary, work, str(nsteps), dump], check=True, stdout=subprocess.DEVNULL)
        return load_dump(dump)
    finally:
        if keep is None:
            shutil.rmtree(work, ignore_errors=True)


def time_ref(cfg, par_path, nsteps):
    """Wall time of nsteps of the reference (fixed-step driver, setup excluded)."""
    binary = build_ref(cfg)
    work = tempfile.mkdtemp(prefix="disco_reft_")
    try:
        shutil.copy(par_path, os.path.join(work, "in.par"))
        r = subprocess.run([binary, work, str(nsteps), "--time"], check=True, capture_output=True, text=True)
        import json
        return json.loads(r.stdout.strip().splitlines()[-1])
    finally:
        shutil.rmtree(work, ignore_errors=True)


class Oracle:
    """The CPU restatement of one disk's step (oracle.c)."""

    def __init__(self, params, modules, Nr, Nz, Ng, Np, r_jph, z_kph):
        lib = C.CDLL(build_oracle())
        D = C.POINTER(C.c_double); I = C.POINTER(C.c_int)
        lib.orc_create.restype = C.c_void_p
        lib.orc_create.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, I, I, D, D]
        lib.orc_destroy.argtypes = [C.c_void_p]
        lib.orc_ncell.argtypes = [C.c_void_p]
        lib.orc_set_cells.argtypes = [C.c_void_p, D, D, D, D, D, I]
        lib.orc_get_cells.argtypes = [C.c_void_p, D, D, D, D, D]
        lib.orc_mindt.restype = C.c_double
        lib.orc_mindt.argtypes = [C.c_void_p]
        lib.orc_timestep.argtypes = [C.c_void_p, C.c_double]
        lib.orc_time.restype = C.c_double
        lib.orc_time.argtypes = [C.c_void_p]
        lib.orc_get_faces.argtypes = [C.c_void_p, C.c_int, I, I, I, I, D]
        lib.orc_get_diagnostics.argtypes = [C.c_void_p, D, D]
        lib.orc_stage.argtypes = [C.c_void_p, C.c_char_p, C.c_double, C.c_double]
        lib.orc_get_grad.argtypes = [C.c_void_p, C.c_int, D]
        self.lib = lib
        self._keep = [np.ascontiguousarray(Ng, np.int32), np.ascontiguousarray(Np, np.int32),
                      np.ascontiguousarray(r_jph, np.float64), np.ascontiguousarray(z_kph, np.float64)]
        Ng_, Np_, rj_, zk_ = self._keep
        self.params, self.modules = params, modules
        self.h = lib.orc_create(C.byref(params), C.byref(modules), Nr, Nz, Ng_.ctypes.data_as(I),
                                Np_.ctypes.data_as(I), rj_.ctypes.data_as(D), zk_.ctypes.data_as(D))
        self.ncell = lib.orc_ncell(self.h)
        self.q = modules.num_c + modules.num_n
        self.Nr, self.Nz, self.Np = Nr, Nz, Np_

    def __del__(self):
        try:
            self.lib.orc_destroy(self.h)
        except Exception:
            pass

    def set_cells(self, prim, cons, piph, dphi, wiph, real):
        D = C.POINTER(C.c_double); I = C.POINTER(C.c_int)
        a = [np.ascontiguousarray(x, np.float64) for x in (prim, cons, piph, dphi, wiph)]
        r = np.ascontiguousarray(real, np.int32)
        self.lib.orc_set_cells(self.h, *[x.ctypes.data_as(D) for x in a], r.ctypes.data_as(I))

    def get_cells(self):
        D = C.POINTER(C.c_double)
        n, q = self.ncell, self.q
        prim = np.zeros((n, q)); cons = np.zeros((n, q))
        piph = np.zeros(n); dphi = np.zeros(n); wiph = np.zeros(n)
        self.lib.orc_get_cells(self.h, *[x.ctypes.data_as(D) for x in (prim, cons, piph, dphi, wiph)])
        return dict(prim=prim, cons=cons, piph=piph, dphi=dphi, wiph=wiph)

    def mindt(self):
        return self.lib.orc_mindt(self.h)

    def timestep(self, dt):
        self.lib.orc_timestep(self.h, dt)

    def time(self):
        return self.lib.orc_time(self.h)

    def faces(self, dim=1):
        D = C.POINTER(C.c_double); I = C.POINTER(C.c_int)
        ntr = (self.Nr - 1) * self.Nz if dim == 1 else (self.Nz - 1) * self.Nr
        nmax = int(self.Np.sum()) * 2 + 16
        fI = np.zeros(ntr + 1, np.int32)
        iL = np.zeros(nmax, np.int32); iR = np.zeros(nmax, np.int32); LR = np.zeros(nmax, np.int32)
        g = np.zeros((nmax, 8))
        n = self.lib.orc_get_faces(self.h, dim, fI.ctypes.data_as(I), iL.ctypes.data_as(I),
                                   iR.ctypes.data_as(I), LR.ctypes.data_as(I), g.ctypes.data_as(D))
        return dict(fIndex=fI, iL=iL[:n], iR=iR[:n], LRtype=LR[:n], geom=g[:n])

    def diagnostics(self):
        D = C.POINTER(C.c_double)
        Q = np.zeros(self.Nr * self.Nz * 5); t = C.c_double()
        self.lib.orc_get_diagnostics(self.h, Q.ctypes.data_as(D), C.byref(t))
        return Q, t.value

    def stage(self, name, RK=0.0, dt=0.0):
        if self.lib.orc_stage(self.h, name.encode(), RK, dt) != 0:
            raise ValueError(name)

    def grad(self, which):
        out = np.zeros((self.ncell, self.q))
        self.lib.orc_get_grad(self.h, which, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out
