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
import time
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libdisco_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def precision_flags(src):
    """nvcc's floating-point flags for a translation unit.  The FP64 parity
    path must not contract a*b+c into an FMA (the reference's x86-64 build
    does not).  The FP32 mixed form (*_mixed.cu) is held to a stated
    tolerance, not to the reference's bits: it contracts, and its FP32
    divisions and square roots use the approximate forms (about 2 ulp);
    its FP64 parts (mesh, dt, compensated update) are not affected."""
    if src.endswith("_mixed.cu"):
        return ["--fmad=true", "--prec-div=false", "--prec-sqrt=false"]
    return ["--fmad=false"]


def nvcc_path():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose:
        # the command, then ptxas's register / spill report of each kernel
        print(" ".join(cmd) + "\n" + r.stdout + r.stderr, flush=True)
    if r.returncode != 0:
        if not verbose:
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
    t0 = time.time()
    nvcc = nvcc_path()
    bdir = os.path.join(HERE, "_build")
    os.makedirs(bdir, exist_ok=True)
    inc = ["-I" + os.path.join(REPO, "include"), "-I" + os.path.join(HERE, "csrc")]
    cu, c = sources()
    jobs, objs = [], []
    for src in cu:
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        jobs.append([nvcc] + ARCH + ["-O3", "-lineinfo"] + precision_flags(src) + ["-std=c++17",
                                     "-Xcompiler", "-fPIC", "-Xptxas", "-v"] + inc + ["-c", src, "-o", obj])
        objs.append(obj)
    for src in c:
        obj = os.path.join(bdir, os.path.basename(src) + ".o")
        jobs.append(["gcc", "-O2", "-fPIC", "-std=gnu11"] + inc + ["-c", src, "-o", obj])
        objs.append(obj)
    # the translation units compile independently: all at once
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        for f in [ex.submit(_run, j, verbose) for j in jobs]:
            f.result()
    tmp = LIB + ".tmp"
    _run([nvcc] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs + ["-lm", "-lz"], verbose)
    os.replace(tmp, LIB)
    # dated to the build's start, so a source edited during it is newer
    os.utime(LIB, (t0, t0))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
