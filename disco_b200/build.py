"""Native build of the disco_b200 library.

Compiles the sm_100a CUDA kernels + C ABI (disco_b200/csrc) and the host C
start-up code (disco_b200/host) into one in-tree shared library,
disco_b200/libdisco_b200.so, with nvcc.  The FP64 parity path is compiled with
--fmad=false so that a*b+c rounds as two operations, as the reference's gcc
x86-64 build does.
"""
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdisco_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]))
    return r


def sources():
    cu = [os.path.join(HERE, "csrc", f) for f in sorted(os.listdir(os.path.join(HERE, "csrc")))
          if f.endswith(".cu")]
    c = [os.path.join(HERE, "host", f) for f in sorted(os.listdir(os.path.join(HERE, "host")))
         if f.endswith(".c")]
    return cu, c


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = []
    for d in ("csrc", "host"):
        for f in os.listdir(os.path.join(HERE, d)):
            deps.append(os.path.join(HERE, d, f))
    for f in os.listdir(os.path.join(REPO, "include")):
        deps.append(os.path.join(REPO, "include", f))
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False):
    """Build disco_b200/libdisco_b200.so (sm_100a).  Returns its path."""
    if not force and not needs_build():
        return LIB
    nvcc = nvcc_path()
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    inc = ["-I" + os.path.join(REPO, "include"), "-I" + os.path.join(HERE, "csrc")]
    cu, c = sources()
    objs = []
    for src in cu:
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        # the FP64 parity path must not contract a*b+c into FMA (the reference's
        # x86-64 build does not); the FP32 mixed form (*_mixed.cu) may
        fmad = "--fmad=true" if src.endswith("_mixed.cu") else "--fmad=false"
        _run([nvcc] + ARCH + ["-O3", "-lineinfo", fmad, "-std=c++17",
                              "-Xcompiler", "-fPIC", "-Xptxas", "-v"] + inc +
             ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    for src in c:
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        _run(["gcc", "-O2", "-fPIC", "-std=gnu11"] + inc + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    tmp = LIB + ".tmp"
    _run([nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs + ["-lm", "-lz"], verbose)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
