"""Run a Disco configuration on the GPU for a number of steps.

    python -m disco_b200.run --template c1_mhd3d --set Constrained_Transport=1 --steps 20
    python -m disco_b200.run --par in.par --opt Makefile_opt.in --steps 100 --mixed
    python -m disco_b200.run --template c0_kepler2d --steps 50 --checkpoint checkpoint_0001
    python -m disco_b200.run --template c0_kepler2d --restart checkpoint_0001.npz --steps 50

The in.par / Makefile_opt.in pair (or a bundled template, with --set
overrides) is read with the reference's semantics, set up on the device as
setupCells does, and advanced by `steps` full timesteps (getmindt + timestep,
as main.c's loop) captured in a CUDA graph.  Prints one JSON line: real
cells, device time per step, zone-updates/s and, with --kernels, the device
time of each kernel of one instrumented step.  --restart starts from a
checkpoint (the Restart path of setupCells), --checkpoint / --ascii write the
output modules' files after the run.
"""
import argparse
import json
import os

from . import Batch, DiscoError, Disk, PREC_FP64, PREC_MIXED, template_paths


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m disco_b200.run")
    ap.add_argument("--template", help="bundled configuration (disco_b200/templates/<name>.par/.in)")
    ap.add_argument("--par", help="in.par")
    ap.add_argument("--opt", help="Makefile_opt.in")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                    help="override an in.par entry (repeatable)")
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--mixed", action="store_true", help="the mixed-precision form")
    ap.add_argument("--kernels", action="store_true", help="per-kernel times of one step")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--restart", metavar="PATH", help="start from this checkpoint (.npz) instead of "
                    "the Initial module (in.par Restart 1)")
    ap.add_argument("--checkpoint", metavar="FILESTART",
                    help="write FILESTART.npz after the run (the checkpoint datasets)")
    ap.add_argument("--ascii", metavar="FILESTART", help="write FILESTART.dat after the run (ascii output)")
    a = ap.parse_args(argv)
    if a.template:
        par, opt = template_paths(a.template)
    elif a.par and a.opt:
        par, opt = a.par, a.opt
    else:
        ap.error("give --template or both --par and --opt")
    tmp = None
    if a.set:
        from .workloads import write_par
        over = dict(s.split("=", 1) for s in a.set)
        base = os.path.splitext(os.path.basename(par))[0] if a.template else None
        if base is None:
            ap.error("--set needs --template")
        tmp = par = write_par(over, base=base)
    try:
        disk = Disk.from_files(par, opt)
    finally:
        if tmp:
            os.unlink(tmp)
    import torch
    b = Batch([disk], device=a.device, precision=PREC_MIXED if a.mixed else PREC_FP64,
              setup=a.restart is None)
    if a.restart:
        b.restart(a.restart)
    stream = torch.cuda.Stream(device=a.device)
    b.set_stream(stream.cuda_stream)          # the events below time the batch's own launches
    b.run(a.warmup)
    b.sync()
    kt = None
    if a.kernels:
        kt = {}
        for name, ms in b.kernel_times():
            kt[name] = round(kt.get(name, 0.0) + ms, 4)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run(a.steps)
    e1.record(stream)
    e1.synchronize()
    err = b.last_error()
    if err:
        raise DiscoError(err, "device step")
    ms = e0.elapsed_time(e1) / max(a.steps, 1)
    out = {"config": a.template or par, "precision": "mixed" if a.mixed else "fp64",
           "real_cells": disk.nreal, "cells": disk.ncell, "steps": a.steps,
           "ms_per_step": ms, "zone_updates_per_s": disk.nreal / (ms / 1e3)}
    if kt is not None:
        out["kernels_ms_per_step"] = dict(sorted(kt.items(), key=lambda x: -x[1]))
    out["t"], out["count_steps"] = b.time()
    if a.checkpoint:
        out["checkpoint"] = b.write_checkpoint(a.checkpoint)
    if a.ascii:
        out["ascii"] = b.write_ascii(a.ascii)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
