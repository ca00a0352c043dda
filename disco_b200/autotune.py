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

    python -m disco_b200.autotune build   [--family hydro|mhd] [--cache DIR] [--mb 4,6,...] [--cb 128]
    python -m disco_b200.autotune measure [--family hydro|mhd] [--cache DIR] [--workload W] [--write]

The MB list is given for 128-thread blocks and scaled for other block sizes
so that every block size sees the same register budgets.  Kernels are
independent of each other's launch shape, so one sweep picks every kernel's
value at once.  Two families of instantiations are tuned apart: `hydro`
(Q = 6, the macros MB_BEGIN ... MB_C2P, block size included, csrc/tuned.h,
on the ragged 2D workloads) and `mhd` (Q = 9, MB_MHD_BEGIN ... MB_MHD_C2P at
the hydro family's block size, csrc/tuned_mhd.h, on the 16-layer mid-plane
slab of config 4, where the r and z passes of k_grad and k_flux_t share one
value each and are timed together).  `build` needs no GPU.
"""
import argparse
import json
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

from . import build as native

HERE = native.HERE
CSRC = os.path.join(HERE, "csrc")
TUNED = os.path.join(CSRC, "tuned.h")
DEFAULT_CACHE = os.path.join(HERE, "_tune")
DEFAULT_MB = (4, 6, 8, 10, 12, 16)

# kernel name (as disco_batch_kernel_times reports it) -> macro
MACROS = {"k_begin": "MB_BEGIN", "k_faces": "MB_FACES", "k_gradr": "MB_GRAD",
          "k_flux_r": "MB_FLUX", "k_update": "MB_UPDATE", "k_c2p": "MB_C2P"}
# the MHD family: k_grad = k_gradr + k_gradz, k_flux = k_flux_r + k_flux_z
MACROS_MHD = {"k_begin": "MB_MHD_BEGIN", "k_grad": "MB_MHD_GRAD", "k_flux": "MB_MHD_FLUX",
              "k_update": "MB_MHD_UPDATE", "k_c2p": "MB_MHD_C2P"}
FAMILIES = {"hydro": {"macros": MACROS, "header": TUNED, "workload": "ragged64"},
            "mhd": {"macros": MACROS_MHD, "header": os.path.join(CSRC, "tuned_mhd.h"),
                    "workload": "config4_nz16"}}
PRECISIONS = {"fp64": 0, "mixed": 1}


def _variant_dir(cache, cb, mb, family="hydro"):
    return os.path.join(cache, ("" if family == "hydro" else family + "_") + "cb%d_mb%d" % (cb, mb))


def _parse_variant(name, family="hydro"):
    pre = "" if family == "hydro" else family + "_"
    cb, mb = name[len(pre) + 2:].split("_mb")
    return int(cb), int(mb)


def _is_variant(name, family):
    return name.startswith("cb") if family == "hydro" else name.startswith(family + "_cb")


def build_variants(cache=DEFAULT_CACHE, mbs=DEFAULT_MB, cbs=(128,), verbose=False, family="hydro"):
    """Compile one library per candidate shape; returns {(cb, mb): path}.
    The variants' translation units compile concurrently."""
    nvcc = native.nvcc_path()
    native.build()                                 # objects of the untuned TUs
    bdir = os.path.join(HERE, "_build")
    inc = ["-I" + os.path.join(native.REPO, "include"), "-I" + CSRC]
    cu, c = native.sources()
    tuned = ("disco_batch.cu", "disco_batch_mixed.cu")
    shared = [os.path.join(bdir, os.path.basename(s) + ".o") for s in cu
              if os.path.basename(s) not in tuned]
    shared += [os.path.join(bdir, os.path.basename(s) + ".o") for s in c]
    macros = FAMILIES[family]["macros"]
    if family != "hydro":
        cbs = (128,)                               # the hydro family's block size
    shapes = sorted({(cb, max(1, min(2048 // cb, mb * 128 // cb))) for cb in cbs for mb in mbs})
    jobs, libs = [], {}
    for cb, mb in shapes:
        vdir = _variant_dir(cache, cb, mb, family)
        os.makedirs(vdir, exist_ok=True)
        defs = ["-D%s=%d" % (m, mb) for m in macros.values()]
        if family == "hydro":
            defs += ["-DCB=%d" % cb, "-DFB=%d" % cb]
        objs = []
        for name in tuned:
            obj = os.path.join(vdir, name + ".o")
            jobs.append([nvcc] + native.ARCH + ["-O3", "-lineinfo"] + native.precision_flags(name) + ["-std=c++17",
                                                "-Xcompiler", "-fPIC"] + defs + inc +
                        ["-c", os.path.join(CSRC, name), "-o", obj])
            objs.append(obj)
        libs[(cb, mb)] = (os.path.join(vdir, "libdisco_b200.so"), objs)
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for f in [ex.submit(native._run, j, verbose) for j in jobs]:
            f.result()
    out = {}
    for shape, (lib, objs) in libs.items():
        native._run([nvcc] + native.ARCH + ["-shared", "-cudart", "static", "-o", lib] +
                    objs + shared + ["-lm", "-lz"], verbose)
        for o in objs:
            os.unlink(o)
        out[shape] = lib
    return out


def _disks(workload):
    from disco_b200 import workloads
    if workload == "ragged64":
        return workloads.ragged_disks()
    if workload == "ragged8":
        return workloads.ragged_disks(ndisk=8)
    if workload.startswith("config4_nz"):
        return [workloads.config4_disk(int(workload[len("config4_nz"):]))]
    return [workloads.config0_disk()]


def _child(lib, workload, precision, reps):
    """Runs in a fresh process: load `lib`, time `reps` instrumented steps."""
    import numpy as np
    import disco_b200 as db
    db.LIBPATH = lib
    b = db.Batch(_disks(workload), precision=precision)
    b.run(3)
    b.sync()
    per = {}
    for _ in range(reps):
        tot = {}
        for name, ms in b.kernel_times(cap=128):
            tot[name] = tot.get(name, 0.0) + ms
        tot["k_grad"] = tot.get("k_grad", 0.0) + tot.get("k_gradr", 0.0) + tot.get("k_gradz", 0.0)
        tot["k_flux"] = tot.get("k_flux_r", 0.0) + tot.get("k_flux_z", 0.0)
        for k, v in tot.items():
            per.setdefault(k, []).append(v)
    b.sync()
    return {k: float(np.median(v)) for k, v in per.items()}


def measure(cache=DEFAULT_CACHE, workload="ragged64", reps=7, family="hydro"):
    """{precision: {(cb, mb): {kernel: ms per step}}} for every built candidate."""
    res = {}
    shapes = sorted(_parse_variant(d, family) for d in os.listdir(cache) if _is_variant(d, family) and
                    os.path.exists(os.path.join(cache, d, "libdisco_b200.so")))
    for pname, prec in PRECISIONS.items():
        res[pname] = {}
        for cb, mb in shapes:
            lib = os.path.join(_variant_dir(cache, cb, mb, family), "libdisco_b200.so")
            r = subprocess.run([sys.executable, "-m", "disco_b200.autotune", "_child", lib, workload,
                                str(prec), str(reps)], capture_output=True, text=True,
                               cwd=native.REPO, timeout=900)
            if r.returncode != 0:
                sys.stderr.write(r.stderr[-2000:])
                raise RuntimeError("autotune child failed for cb %d mb %d (%s)" % (cb, mb, pname))
            res[pname][(cb, mb)] = json.loads(r.stdout.strip().splitlines()[-1])
    return res


def choose(res, macros=MACROS):
    """The block size, then the fastest MB per (precision, kernel) at it:
    {"cb": CB, "fp64": {kernel: MB}, "mixed": {...}}."""
    def best_total(table, cb):
        tot = 0.0
        for k in macros:
            cand = [t[k] for (c, _), t in table.items() if c == cb and k in t]
            tot += min(cand) if cand else 0.0
        return tot
    ref = res.get("fp64") or next(iter(res.values()))
    cbs = sorted({c for c, _ in ref})
    cb = min(cbs, key=lambda c: best_total(ref, c))
    best = {"cb": cb}
    for pname, table in res.items():
        best[pname] = {}
        for k in macros:
            cand = [(t[k], mb) for (c, mb), t in table.items() if c == cb and k in t]
            if cand:
                best[pname][k] = min(cand)[1]
    return best


def write_header(res, best, workload, path=TUNED, family="hydro"):
    cb = best["cb"]
    macros = FAMILIES[family]["macros"]
    what = ("the step kernels: CB threads per block and, per kernel," if family == "hydro" else
            "the MHD (Q = 9) instantiations of the step kernels: per kernel,")
    lines = ["/*",
             " * Launch shapes of %s" % what,
             " * the resident blocks per SM MB (register budget 65536 / (CB * MB)), written",
             " * by disco_b200/autotune.py from CUDA-event kernel times of one step of the",
             " * %s workload (median of the instrumented steps, ms per step;" % workload,
             " * columns CB/MB):", " *"]
    for pname, table in res.items():
        shapes = sorted(table)
        lines.append(" *   %-6s %-10s %s" % (pname, "kernel", " ".join("%8s" % ("%d/%d" % s) for s in shapes)))
        for k in macros:
            row = " ".join("%8.4f" % table[s].get(k, float("nan")) for s in shapes)
            lines.append(" *   %-6s %-10s %s   -> %d" % ("", k, row, best[pname].get(k, 0)))
    lines += [" *", " * Values given with -D on the command line win.", " */", "#pragma once"]
    if family == "hydro":
        lines += ["#ifndef CB", "#define CB %d" % cb, "#endif", "#ifndef FB", "#define FB %d" % cb, "#endif"]
    for pname, cond in (("mixed", "#ifdef DISCO_MIXED_TU"), ("fp64", "#else")):
        lines.append(cond)
        for k, m in macros.items():
            if k in best[pname]:
                lines += ["#ifndef %s" % m, "#define %s %d" % (m, best[pname][k]), "#endif"]
    lines.append("#endif")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m disco_b200.autotune")
    sub = ap.add_subparsers(dest="cmd", required=True)
    b = sub.add_parser("build")
    b.add_argument("--family", default="hydro", choices=sorted(FAMILIES))
    b.add_argument("--cache", default=DEFAULT_CACHE)
    b.add_argument("--mb", default=",".join(str(m) for m in DEFAULT_MB),
                   help="occupancy targets for 128-thread blocks (scaled for other sizes)")
    b.add_argument("--cb", default="128", help="block sizes, e.g. 64,128,256")
    m = sub.add_parser("measure")
    m.add_argument("--family", default="hydro", choices=sorted(FAMILIES))
    m.add_argument("--cache", default=DEFAULT_CACHE)
    m.add_argument("--workload", default=None,
                   help="ragged64 | ragged8 | config0 | config4_nzN (default: the family's)")
    m.add_argument("--header", default=None, help="where --write puts the header (default: csrc)")
    m.add_argument("--reps", type=int, default=7)
    m.add_argument("--write", action="store_true", help="write csrc/tuned.h")
    m.add_argument("--json", default=None, help="also save the measured table here")
    c = sub.add_parser("_child")
    c.add_argument("lib"); c.add_argument("workload"); c.add_argument("precision", type=int)
    c.add_argument("reps", type=int)
    a = ap.parse_args(argv)
    if a.cmd == "build":
        for shape, lib in build_variants(a.cache, [int(x) for x in a.mb.split(",")],
                                         [int(x) for x in a.cb.split(",")], family=a.family).items():
            print(shape, lib)
    elif a.cmd == "measure":
        fam = FAMILIES[a.family]
        a.workload = a.workload or fam["workload"]
        res = measure(a.cache, a.workload, a.reps, a.family)
        best = choose(res, fam["macros"])
        if a.json:
            with open(a.json, "w") as f:
                json.dump({"workload": a.workload, "best": best,
                           "res": {p: {"%d/%d" % s: t for s, t in tab.items()} for p, tab in res.items()}},
                          f, indent=1)
        print(json.dumps(best))
        if a.write:
            write_header(res, best, a.workload, a.header or fam["header"], a.family)
    else:
        print(json.dumps(_child(a.lib, a.workload, a.precision, a.reps)))


if __name__ == "__main__":
    main()
