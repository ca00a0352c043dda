"""Autotuner for the step kernels' launch shapes.

The step kernels are bound by memory latency: the block size and how many
blocks an SM keeps resident (which __launch_bounds__ turns into each
kernel's register budget) decide how many loads are in flight, and the best
values differ per kernel, per precision and per GPU.  This tool

  1. builds the library once per candidate shape -- a block size CB (cell
     and face kernels alike) and an occupancy target MB for every kernel,
     both precisions -- into a cache directory,
  2. times each kernel of one step of a workload with CUDA events
     (disco_batch_kernel_times, median of several instrumented steps), one
     child process per candidate and precision,
  3. keeps the block size whose per-kernel best times add up to the fastest
     FP64 step (the host's block tables serve both precisions, so there is
     one), then per kernel and precision the fastest MB at that block size,
     and writes them to csrc/tuned.h with the measured table.

    python -m disco_b200.autotune build   [--cache DIR] [--mb 4,6,...] [--cb 128]   (no GPU)
    python -m disco_b200.autotune measure [--cache DIR] [--workload ragged64] [--write]

The MB list is given for 128-thread blocks and scaled for other block sizes
so that every block size sees the same register budgets.  Kernels are
independent of each other's launch shape, so one sweep picks every kernel's
value at once.
"""
import argparse
import json
import os
import subprocess
import sys

from . import build as native

HERE = native.HERE
CSRC = os.path.join(HERE, "csrc")
TUNED = os.path.join(CSRC, "tuned.h")
DEFAULT_CACHE = os.path.join(HERE, "_tune")
DEFAULT_MB = (4, 6, 8, 10, 12, 16)

# kernel name (as disco_batch_kernel_times reports it) -> macro
MACROS = {"k_begin": "MB_BEGIN", "k_faces": "MB_FACES", "k_gradr": "MB_GRAD",
          "k_flux_r": "MB_FLUX", "k_update": "MB_UPDATE", "k_c2p": "MB_C2P"}
PRECISIONS = {"fp64": 0, "mixed": 1}


def _variant_dir(cache, cb, mb):
    return os.path.join(cache, "cb%d_mb%d" % (cb, mb))


def _parse_variant(name):
    cb, mb = name[2:].split("_mb")
    return int(cb), int(mb)


def build_variants(cache=DEFAULT_CACHE, mbs=DEFAULT_MB, cbs=(128,), verbose=False):
    """Compile one library per candidate shape; returns {(cb, mb): path}."""
    nvcc = native.nvcc_path()
    native.build()                                 # objects of the untuned TUs
    bdir = os.path.join(HERE, "_build")
    inc = ["-I" + os.path.join(native.REPO, "include"), "-I" + CSRC]
    cu, c = native.sources()
    tuned = ("disco_batch.cu", "disco_batch_mixed.cu")
    shared = [os.path.join(bdir, os.path.basename(s) + ".o") for s in cu
              if os.path.basename(s) not in tuned]
    shared += [os.path.join(bdir, os.path.basename(s) + ".o") for s in c]
    out = {}
    shapes = sorted({(cb, max(1, min(2048 // cb, mb * 128 // cb))) for cb in cbs for mb in mbs})
    for cb, mb in shapes:
        vdir = _variant_dir(cache, cb, mb)
        os.makedirs(vdir, exist_ok=True)
        lib = os.path.join(vdir, "libdisco_b200.so")
        defs = ["-D%s=%d" % (m, mb) for m in MACROS.values()] + ["-DCB=%d" % cb, "-DFB=%d" % cb]
        objs = []
        for name in tuned:
            src = os.path.join(CSRC, name)
            obj = os.path.join(vdir, name + ".o")
            fmad = "--fmad=true" if name.endswith("_mixed.cu") else "--fmad=false"
            native._run([nvcc] + native.ARCH + ["-O3", "-lineinfo", fmad, "-std=c++17",
                                                "-Xcompiler", "-fPIC"] + defs + inc +
                        ["-c", src, "-o", obj], verbose)
            objs.append(obj)
        native._run([nvcc] + native.ARCH + ["-shared", "-cudart", "static", "-o", lib] +
                    objs + shared + ["-lm"], verbose)
        for o in objs:
            os.unlink(o)
        out[(cb, mb)] = lib
    return out


def _child(lib, workload, precision, reps):
    """Runs in a fresh process: load `lib`, time `reps` instrumented steps."""
    import numpy as np
    import disco_b200 as db
    db.LIBPATH = lib
    from disco_b200 import workloads
    disks = workloads.ragged_disks() if workload == "ragged64" else \
        workloads.ragged_disks(ndisk=8) if workload == "ragged8" else [workloads.config0_disk()]
    b = db.Batch(disks, precision=precision)
    b.run(3)
    b.sync()
    per = {}
    for _ in range(reps):
        tot = {}
        for name, ms in b.kernel_times():
            tot[name] = tot.get(name, 0.0) + ms
        for k, v in tot.items():
            per.setdefault(k, []).append(v)
    b.sync()
    return {k: float(np.median(v)) for k, v in per.items()}


def measure(cache=DEFAULT_CACHE, workload="ragged64", reps=7):
    """{precision: {(cb, mb): {kernel: ms per step}}} for every built candidate."""
    res = {}
    shapes = sorted(_parse_variant(d) for d in os.listdir(cache) if d.startswith("cb") and
                    os.path.exists(os.path.join(cache, d, "libdisco_b200.so")))
    for pname, prec in PRECISIONS.items():
        res[pname] = {}
        for cb, mb in shapes:
            lib = os.path.join(_variant_dir(cache, cb, mb), "libdisco_b200.so")
            r = subprocess.run([sys.executable, "-m", "disco_b200.autotune", "_child", lib, workload,
                                str(prec), str(reps)], capture_output=True, text=True,
                               cwd=native.REPO, timeout=900)
            if r.returncode != 0:
                sys.stderr.write(r.stderr[-2000:])
                raise RuntimeError("autotune child failed for cb %d mb %d (%s)" % (cb, mb, pname))
            res[pname][(cb, mb)] = json.loads(r.stdout.strip().splitlines()[-1])
    return res


def choose(res):
    """The block size, then the fastest MB per (precision, kernel) at it:
    {"cb": CB, "fp64": {kernel: MB}, "mixed": {...}}."""
    def best_total(table, cb):
        tot = 0.0
        for k in MACROS:
            cand = [t[k] for (c, _), t in table.items() if c == cb and k in t]
            tot += min(cand) if cand else 0.0
        return tot
    ref = res.get("fp64") or next(iter(res.values()))
    cbs = sorted({c for c, _ in ref})
    cb = min(cbs, key=lambda c: best_total(ref, c))
    best = {"cb": cb}
    for pname, table in res.items():
        best[pname] = {}
        for k in MACROS:
            cand = [(t[k], mb) for (c, mb), t in table.items() if c == cb and k in t]
            if cand:
                best[pname][k] = min(cand)[1]
    return best


def write_header(res, best, workload, path=TUNED):
    cb = best["cb"]
    lines = ["/*",
             " * Launch shapes of the step kernels: CB threads per block and, per kernel,",
             " * the resident blocks per SM MB (register budget 65536 / (CB * MB)), written",
             " * by disco_b200/autotune.py from CUDA-event kernel times of one step of the",
             " * %s workload (median of the instrumented steps, ms per step;" % workload,
             " * columns CB/MB):", " *"]
    for pname, table in res.items():
        shapes = sorted(table)
        lines.append(" *   %-6s %-10s %s" % (pname, "kernel", " ".join("%8s" % ("%d/%d" % s) for s in shapes)))
        for k in MACROS:
            row = " ".join("%8.4f" % table[s].get(k, float("nan")) for s in shapes)
            lines.append(" *   %-6s %-10s %s   -> %d" % ("", k, row, best[pname].get(k, 0)))
    lines += [" *", " * Values given with -D on the command line win.", " */", "#pragma once",
              "#ifndef CB", "#define CB %d" % cb, "#endif", "#ifndef FB", "#define FB %d" % cb, "#endif"]
    for pname, cond in (("mixed", "#ifdef DISCO_MIXED_TU"), ("fp64", "#else")):
        lines.append(cond)
        for k, m in MACROS.items():
            if k in best[pname]:
                lines += ["#ifndef %s" % m, "#define %s %d" % (m, best[pname][k]), "#endif"]
    lines.append("#endif")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m disco_b200.autotune")
    sub = ap.add_subparsers(dest="cmd", required=True)
    b = sub.add_parser("build")
    b.add_argument("--cache", default=DEFAULT_CACHE)
    b.add_argument("--mb", default=",".join(str(m) for m in DEFAULT_MB),
                   help="occupancy targets for 128-thread blocks (scaled for other sizes)")
    b.add_argument("--cb", default="128", help="block sizes, e.g. 64,128,256")
    m = sub.add_parser("measure")
    m.add_argument("--cache", default=DEFAULT_CACHE)
    m.add_argument("--workload", default="ragged64", choices=["ragged64", "ragged8", "config0"])
    m.add_argument("--reps", type=int, default=7)
    m.add_argument("--write", action="store_true", help="write csrc/tuned.h")
    m.add_argument("--json", default=None, help="also save the measured table here")
    c = sub.add_parser("_child")
    c.add_argument("lib"); c.add_argument("workload"); c.add_argument("precision", type=int)
    c.add_argument("reps", type=int)
    a = ap.parse_args(argv)
    if a.cmd == "build":
        for shape, lib in build_variants(a.cache, [int(x) for x in a.mb.split(",")],
                                         [int(x) for x in a.cb.split(",")]).items():
            print(shape, lib)
    elif a.cmd == "measure":
        res = measure(a.cache, a.workload, a.reps)
        best = choose(res)
        if a.json:
            with open(a.json, "w") as f:
                json.dump({"workload": a.workload, "best": best,
                           "res": {p: {"%d/%d" % s: t for s, t in tab.items()} for p, tab in res.items()}},
                          f, indent=1)
        print(json.dumps(best))
        if a.write:
            write_header(res, best, a.workload)
    else:
        print(json.dumps(_child(a.lib, a.workload, a.precision, a.reps)))


if __name__ == "__main__":
    main()
