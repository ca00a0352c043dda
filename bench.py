#!/usr/bin/env python
"""Benchmark of the B200 Disco RK timestep (zone-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ragged64|config0]

A step is one full RK2 timestep (two substeps, fused getmindt) of every disk
of the workload, inputs resident in HBM.  Default workload `ragged64`: 64
ragged 2D hydro disks (~5.7M cells, the config-2 batch, FP64 plain path).
Multi-GPU: one process per GPU (torchrun), each GPU advances its own 64
disks (same sizes, own noise seeds): the disks are independent, so there is
no data-path collective ("scaling": "weak"); only a barrier and a max of the
timings over ranks.

--impl reference times the reference Disco serial CPU code itself
(oracle/_ref, built from the reference's own sources) on the same disks, one
process per disk spread over all host cores.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "oracle"))

METRIC = "zone-updates/s"
Q = 6                                   # NUM_C 5 + NUM_N 1 (hydro)
B_ALG_STEP = 576                        # HBM bytes per zone-update, FP64 hydro (10Q+12 words)


def peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# dram__bytes_read.sum + dram__bytes_write.sum of one first-substep launch on
# the ragged8 workload (1,049,795 cells, 2,089,252 r-faces), from an ncu
# capture of k_update and k_flux_t on that workload: (bytes, units the
# launch processed)
DRAM_UPDATE_RAGGED8 = (289.8e6 + 53.7e6, 1049795)
DRAM_FLUX_RAGGED8 = (216.2e6 + 72.5e6, 2089252)


def kernel_bytes(name, first, N, Nf, Na, nreal=0):
    """Algorithmic (compulsory, each element once) HBM bytes of one launch.
    N cells, Nf r-faces, Na annuli; Q doubles per cell.  k_step, the whole
    RK2 step as one launch, moves the step's 576 bytes per real zone-update."""
    w = 8
    if name == "k_step":
        return B_ALG_STEP * nreal
    if name == "k_begin":
        return N * w * ((5 * Q + 4) if first else (5 * Q + 1))
    if name == "k_c2p":
        # reads cons, piph, dphi (+wiph on the last substep); writes prim
        return N * w * (2 * Q + 2) + (N * w if not first else 0)
    if name == "k_I0":
        # RK2 keeps the faces in the first substep (k_I0 returns at once)
        return 0 if first else N * w + Na * 4
    if name == "k_faces":
        # reads piph, dphi, prim, gradp; writes the face lists, geometry,
        # PLM face slopes and consL/consR -- or, in the first substep, reads
        # the kept face cells and centres and writes the slopes only
        if first:
            return N * w * (2 * Q + 2) + Nf * (4 + 4 + w + Q * w)
        return N * w * (2 * Q + 2) + N * 8 + Nf * (4 + 4 + 1 + 3 * w + Q * w)
    if name == "k_gradr":
        # reads the face slopes and areas, the cell's geometry; writes gradr
        return Nf * w * (Q + 1) + N * (w * Q + 3 * w + 8)
    if name == "k_flux_r":
        return Nf * (4 + 4 + 2 * w + Q * w) + N * w * (3 * Q + 2)
    if name == "k_update":
        # reads cons, prim, gradp (phi faces), piph, dphi, wiph, the consume
        # indices and the r-face fluxes; writes cons (+ piph_new -> piph,
        # dphi in the first substep)
        return N * w * (4 * Q + (6 if first else 3)) + N * 8 + Nf * w * Q
    return 0


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1])); smax.append(float(p[2]))
                except ValueError:
                    continue
                for n, v in zip(names, p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def make_disks(workload, rank):
    from disco_b200 import workloads
    if workload == "config0":
        return [workloads.config0_disk()]
    if workload == "ragged8":
        return workloads.ragged_disks(8, rank=rank)
    return workloads.ragged_disks(64, rank=rank)


# The reference arm builds its in.par files here, in plain Python, so that it
# imports nothing of the disco_b200 package: the same seeded draws as
# disco_b200.workloads.ragged_specs (tests/test_bench_config.py checks that
# they agree) written into the same template.
TEMPLATE_PAR = os.path.join(REPO, "disco_b200", "templates", "c0_kepler2d.par")
NDISK = {"ragged64": 64, "ragged8": 8, "config0": 1}


def ragged_specs(ndisk, seed=314159, rank=0):
    """(Num_R, Mach_Number, noise seed) per disk of a ragged workload."""
    import numpy as np
    rng = np.random.default_rng(seed)
    nr = rng.integers(32, 257, size=ndisk)
    mach = rng.uniform(10.0, 40.0, size=ndisk)
    seeds = seed + np.arange(ndisk) + rank * ndisk
    return [(int(a), float(b), int(c)) for a, b, c in zip(nr, mach, seeds)]


def template_par(overrides, directory):
    """The config-0 template in.par with some keys replaced, written to a
    new file in `directory`; returns its path."""
    out = []
    with open(TEMPLATE_PAR) as f:
        for line in f:
            tok = line.split()
            if tok and tok[0] in overrides:
                line = "%s\t\t%s\n" % (tok[0], overrides[tok[0]])
            out.append(line)
    fd, path = tempfile.mkstemp(suffix=".par", dir=directory)
    with os.fdopen(fd, "w") as f:
        f.write("".join(out))
    return path


def reference_pars(workload, directory, rank=0):
    if workload == "config0":
        return [template_par({}, directory)]
    return [template_par({"Num_R": nr, "Mach_Number": repr(mach), "Init_Par0": s}, directory)
            for nr, mach, s in ragged_specs(NDISK[workload], rank=rank)]


def workload_config(workload, nreal):
    """The `config` object of both arms' lines: the workload, nothing of
    either implementation."""
    base = ("64 2D Keplerian hydro disks" if workload == "ragged64" else
            "8 2D Keplerian hydro disks" if workload == "ragged8" else "the config-0 2D Keplerian hydro disk")
    grid = ("Num_R drawn from [32, 256] per disk (seeded), log r in [0.5, 3], Np constant per disk"
            if workload.startswith("ragged") else "Num_R 128, log r in [0.5, 3], Np 452")
    return {"workload": workload, "description": base, "disks_per_gpu": NDISK[workload],
            "real_cells_per_gpu": int(nreal), "grid": grid,
            "physics": "Euler, HLLC, PLM 1.5, RK2, CFL 0.5, sun gravity, fixed boundaries, Mesh_Motion 1",
            "precision": "fp64",
            "l2_policy": "inputs larger than L2 (%.2f GB of prim+cons state per GPU)" % (nreal * 8 * 2 * Q / 1e9)}


def time_reference(workload, nsteps, max_workers=None):
    """The reference's serial CPU code on every disk of the workload, one
    process per disk, statically spread over the host cores.  Returns
    (zone-updates/s, cores, sample description, real cells)."""
    import pyoracle
    binary = pyoracle.ref_binary("c0_kepler2d")
    if not os.path.exists(binary):
        pyoracle.build_ref("c0_kepler2d")
    pdir = tempfile.mkdtemp(prefix="dpar_")
    pars = reference_pars(workload, pdir)
    cores = max_workers or min(os.cpu_count() or 1, len(pars))
    work = []
    for p in pars:
        d = tempfile.mkdtemp(prefix="dref_")
        with open(p) as f, open(os.path.join(d, "in.par"), "w") as g:
            g.write(f.read())
        work.append(d)
    # static round-robin assignment: worker w runs disks w, w+cores, ...
    procs = []
    for w in range(cores):
        jobs = work[w::cores]
        cmd = " ; ".join("%s %s %d --time" % (binary, d, nsteps) for d in jobs)
        procs.append(subprocess.Popen(["bash", "-c", cmd], stdout=subprocess.PIPE, text=True))
    per_worker, zones, nreal = [], 0, 0
    for pr in procs:
        out, _ = pr.communicate()
        s = 0.0
        for line in out.strip().splitlines():
            if line.startswith("{"):
                r = json.loads(line)
                s += r["seconds"]
                zones += r["real_cells"] * r["steps"]
                nreal += r["real_cells"]
        per_worker.append(s)
    for d in work + [pdir]:
        subprocess.run(["rm", "-rf", d])
    wall = max(per_worker)
    sample = "%s: all %d disks x %d step(s), %d processes on %d cores, step-loop time only" % (
        workload, len(pars), nsteps, len(pars), cores)
    return zones / wall, cores, sample, nreal


def run_reference(args, world, rank):
    if rank != 0:
        return
    v, cores, sample, nreal = time_reference(args.workload, max(1, args.steps // 4))
    line = {"metric": METRIC, "value": v, "unit": "zone-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": workload_config(args.workload, nreal),
            "parallelism": "one host process per disk",
            "cpu_baseline": {"value": v, "unit": "zone-updates/s", "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": v, "unit": "zone-updates/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def div_b(disk, batch, st):
    """Discrete div B of every real cell from the face fluxes of the
    cell-centred field: sum over the cell's phi, r and z faces of the
    face-averaged normal B times the face area, over the cell volume.
    Returns (sum |div B| dV, sum |B| dV) over the real cells."""
    import numpy as np
    p = st["prim"]
    Br, Bp, Bz = p[:, 5], p[:, 6], p[:, 7]
    nc = len(p)
    flux = np.zeros(nc)
    off = np.concatenate([[0], np.cumsum(disk.Np)])
    rj, zk = disk.r_jph, disk.z_kph          # index 0 is edge -1
    vol = np.zeros(nc)
    for a in range(disk.Nr * disk.Nz):
        j, k = a % disk.Nr, a // disk.Nr
        c = np.arange(off[a], off[a + 1])
        cn = np.roll(c, -1)
        dr, dz = rj[j + 1] - rj[j], zk[k + 1] - zk[k]
        f = 0.5 * (Bp[c] + Bp[cn]) * dr * dz
        flux[c] += f
        flux[cn] -= f
        vol[c] = 0.5 * (rj[j + 1] + rj[j]) * dr * st["dphi"][c] * dz
    for dim, comp in ((1, Br), (2, Bz)):
        fa = batch.faces(0, dim, geom=True)
        if len(fa["iL"]) == 0:
            continue
        f = 0.5 * (comp[fa["iL"]] + comp[fa["iR"]]) * fa["geom"][:, 7]
        np.add.at(flux, fa["iL"], f)
        np.add.at(flux, fa["iR"], -f)
    r = disk.real == 1
    bmag = np.sqrt(Br ** 2 + Bp ** 2 + Bz ** 2)
    return float(np.abs(flux[r]).sum()), float((bmag[r] * vol[r]).sum())


def config1_leg(args, local, stream):
    """3D Newtonian MHD shearing disk (HLLD, zerograd): FP64 and the mixed
    form for 200 steps from the same state without constrained transport (B
    through the fluxes), their throughput, the mixed form's error and drifts
    against FP64; then FP64 with constrained transport (the configuration's
    stated form) and its face-flux divergence drift."""
    import numpy as np
    import torch
    import disco_b200 as db
    par, opt = db.template_paths("c1_mhd3d")
    disk = db.Disk.from_files(par, opt)
    nsteps = 200
    out = {"workload": "3D MHD shearing disk, HLLD, zerograd, Nr=%d Nz=%d, Np max %d, %d real cells"
                       % (disk.Nr, disk.Nz, int(np.max(disk.Np)), disk.nreal),
           "steps": nsteps, "warmup": 3,
           "note": "errors and drifts after warm-up + timed steps, both forms from the same set-up"}
    states = {}
    for prec, key in ((db.PREC_FP64, "fp64"), (db.PREC_MIXED, "mixed")):
        b = db.Batch([disk], device=local, precision=prec)
        b.set_stream(stream.cuda_stream)
        if key == "fp64":
            states["s0"] = b.get_cells()
            states["div0"] = div_b(disk, b, states["s0"])
        b.run(3)                    # warm-up (and the step graph's capture)
        b.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run(nsteps)
        e1.record(stream)
        e1.synchronize()
        if b.last_error() != 0:
            raise RuntimeError("device error in the config-1 leg")
        ms = e0.elapsed_time(e1)
        st = b.get_cells()
        states[key] = st
        out[key] = {"zone_updates_per_s": disk.nreal * nsteps / (ms / 1e3), "ms_per_step": ms / nsteps,
                    "div_b": div_b(disk, b, st)}
        if key == "fp64":
            # per-kernel times of one more step, after the state both forms
            # are compared on was taken (each form has run 3 + nsteps steps)
            kt = {}
            for name, t in b.kernel_times():
                kt[name] = kt.get(name, 0.0) + t
            out["fp64_kernels_ms_per_step"] = {k: round(v, 4) for k, v in
                                               sorted(kt.items(), key=lambda x: -x[1])}
        b.close()
    r = disk.real == 1
    a, m, s0 = states["fp64"], states["mixed"], states["s0"]
    names = ["rho", "P", "v_r", "omega", "v_z", "B_r", "B_phi", "B_z", "X"]
    err = {}
    for q, nm in enumerate(names):
        den = np.abs(a["prim"][r, q]).sum()
        err[nm] = float(np.abs(m["prim"][r, q] - a["prim"][r, q]).sum() / den) if den > 0 else None
    out["mixed_rel_l1_vs_fp64"] = err
    tot = lambda st, q: float(st["cons"][r, q].sum())
    out["drift"] = {
        "mass_fp64": tot(a, 0) / tot(s0, 0) - 1.0, "mass_mixed": tot(m, 0) / tot(s0, 0) - 1.0,
        "ang_mom_fp64": tot(a, 3) / tot(s0, 3) - 1.0, "ang_mom_mixed": tot(m, 3) / tot(s0, 3) - 1.0,
        "mixed_vs_fp64_mass": tot(m, 0) / tot(a, 0) - 1.0,
        "div_b_rel_step0": states["div0"][0] / states["div0"][1],
        "div_b_rel_fp64": out["fp64"]["div_b"][0] / out["fp64"]["div_b"][1],
        "div_b_rel_mixed": out["mixed"]["div_b"][0] / out["mixed"]["div_b"][1]}
    out["mixed_speedup_vs_fp64"] = out["mixed"]["zone_updates_per_s"] / out["fp64"]["zone_updates_per_s"]

    # The configuration's stated form: constrained transport (CT_MODE 2,
    # Constrained_Transport 1), FP64.  Its invariant is each cell's net face
    # flux (the discrete div B of the face fluxes), which CT keeps.
    from disco_b200.workloads import write_par
    p = write_par({"Constrained_Transport": 1}, base="c1_mhd3d")
    diskc = db.Disk.from_files(p, opt)
    os.unlink(p)
    b = db.Batch([diskc], device=local)
    b.set_stream(stream.cuda_stream)
    d0, _ = face_flux_div(diskc, b)
    b.run(3)
    b.sync()
    kt = {}
    for name, t in b.kernel_times():
        kt[name] = kt.get(name, 0.0) + t
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run(nsteps)
    e1.record(stream)
    e1.synchronize()
    if b.last_error() != 0:
        raise RuntimeError("device error in the config-1 CT leg")
    ms = e0.elapsed_time(e1)
    d1, phimax = face_flux_div(diskc, b)
    rc = diskc.real == 1
    out["fp64_ct"] = {"zone_updates_per_s": diskc.nreal * nsteps / (ms / 1e3), "ms_per_step": ms / nsteps,
                      "kernels_ms_per_step": {k: round(v, 4) for k, v in
                                              sorted(kt.items(), key=lambda x: -x[1])},
                      "face_div_b_drift_rel": float(np.abs(d1 - d0)[rc].max() / phimax),
                      "note": "max over real cells of |net face flux(t) - net face flux(0)| / max |Phi|"}
    b.close()
    return out


B_ALG_MHD_CT = {"fp64": 1056, "mixed": 1200}   # HBM bytes per zone-update, MHD Q=9 with CT (5 faces)


def config4_leg(args, local, stream):
    """3D MHD circumbinary disk with constrained transport (softened
    equal-mass binary, HLLD, CT_MODE 2, zerograd; Nr 384 x Nz 128, Np up to
    1536, 39.5M real cells): 50 steps of the mixed form (FP32 bulk, FP64
    phi/mesh/Kahan update, FP64 face fluxes) against the FP64 plain path,
    from the same set-up; throughput, step-level fraction of the HBM
    roofline, and the mixed form's density / pressure error."""
    import numpy as np
    import torch
    import disco_b200 as db
    par, opt = db.template_paths("c4_binary3d")
    disk = db.Disk.from_files(par, opt)
    nsteps = 50
    hbm, kind = peaks()
    out = {"workload": "3D MHD circumbinary disk, softened equal-mass binary, HLLD + CT, zerograd, "
                       "Nr=%d Nz=%d (incl. ghosts), Np max %d, %d real cells (the configuration's "
                       "'about 50M' is not reachable with Np <= 1536 on 384 x 128 annuli)"
                       % (disk.Nr, disk.Nz, int(np.max(disk.Np)), disk.nreal),
           "steps": nsteps, "warmup": 3}
    ref = None
    r = disk.real == 1
    for prec, key in ((db.PREC_FP64, "fp64"), (db.PREC_MIXED, "mixed")):
        b = db.Batch([disk], device=local, precision=prec)
        b.set_stream(stream.cuda_stream)
        b.run(3)
        b.sync()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run(nsteps)
        e1.record(stream)
        e1.synchronize()
        if b.last_error() != 0:
            raise RuntimeError("device error in the config-4 leg")
        ms = e0.elapsed_time(e1)
        zu = disk.nreal * nsteps / (ms / 1e3)
        out[key] = {"zone_updates_per_s": zu, "ms_per_step": ms / nsteps,
                    "step_roofline": {"bytes_per_zone_update": B_ALG_MHD_CT[key],
                                      "achieved": B_ALG_MHD_CT[key] * zu / 1e9, "peak": hbm,
                                      "unit": "GB/s", "frac": B_ALG_MHD_CT[key] * zu / 1e9 / hbm,
                                      "peak_kind": kind}}
        st = b.get_cells()
        if key == "fp64":
            ref = st["prim"][r][:, :2].copy()
        else:
            pm = st["prim"][r][:, :2]
            out["mixed_rel_l1_vs_fp64"] = {
                nm: float(np.abs(pm[:, q] - ref[:, q]).sum() / np.abs(ref[:, q]).sum())
                for q, nm in ((0, "rho"), (1, "P"))}
        del st
        b.close()
    out["mixed_speedup_vs_fp64"] = out["mixed"]["zone_updates_per_s"] / out["fp64"]["zone_updates_per_s"]
    if rank0_cpu(args):
        out["cpu_baseline"] = reference_slice_rate("c4_binary3d", {"Num_Z": 4, "Z_Min": -0.5 * 4 / 128,
                                                                  "Z_Max": 0.5 * 4 / 128}, 1,
                                                   "reference mhd + hlld + 3D CT + binary_soft, the full "
                                                   "384-annulus r grid and Np on 4 z layers, 1 step, one "
                                                   "process")
    return out


def reference_slice_rate(cfg, overrides, nsteps, sample):
    """The reference binary of a module configuration on a reduced slice of
    a workload (its template in.par with overrides), one process: the
    cpu_baseline object."""
    try:
        import pyoracle
        binary = pyoracle.ref_binary(cfg)
        if not os.path.exists(binary):
            pyoracle.build_ref(cfg)
        d = tempfile.mkdtemp(prefix="dref_")
        with open(os.path.join(d, "in.par"), "w") as f:
            f.write(write_par_text(cfg, overrides))
        res = subprocess.run([binary, d, str(nsteps), "--time"], capture_output=True, text=True, timeout=900)
        subprocess.run(["rm", "-rf", d])
        rr = json.loads([l for l in res.stdout.splitlines() if l.startswith("{")][0])
        return {"value": rr["zone_updates_per_s"], "unit": "zone-updates/s", "cores": 1, "kind": "reference",
                "sample": sample + " (%d real cells)" % rr["real_cells"]}
    except Exception as ex:
        return {"value": None, "sample": "unavailable: %s" % ex}


def face_flux_div(disk, batch):
    """Net magnetic flux out of each cell through its faces under CT (the
    face-flux slots Phi), and max |Phi|."""
    import numpy as np
    st = batch.get_cells()
    Phi = st["Phi"]
    div = np.zeros(disk.ncell)
    dims = [(1, 2, 1)] + ([(2, 4, 3)] if disk.Nz > 1 and Phi.shape[1] == 5 else [])
    for dim, s0, s1 in dims:
        F = batch.faces(0, dim)
        L, R, lr = F["iL"], F["iR"], F["LRtype"]
        v = np.where(lr == 0, Phi[L, s0], Phi[R, s1])
        np.add.at(div, L, v)
        np.add.at(div, R, -v)
    off = np.concatenate([[0], np.cumsum(disk.Np)])
    for a in range(len(disk.Np)):
        c = np.arange(off[a], off[a + 1])
        div[c] += Phi[c, 0] - Phi[np.roll(c, 1), 0]
    return div, float(np.abs(Phi).max())


B_ALG_GR = 8 * (10 * 9 + 12)            # HBM bytes per zone-update, Q = 9 without face fluxes (816)
C3_GRID = {"Num_R": 192, "Num_Z": 96, "aspect": 0.75}          # Np 463 per annulus


def config3_leg(args, local, stream):
    """Config 3: the GRMHD torus timestep (grmhd2, Kerr-Schild a = 0.9, HLL,
    noble2d cons->prim, fixed3d), 192 x 96 annuli of 463 cells (8.53M real
    cells), FP64; throughput, step roofline against the 816 B/zone-update of
    the Q = 9 state without face fluxes, and the reference's serial CPU code
    on a reduced-Nz slice of the same grid (Schwarzschild, a = 0: the
    reference has no Kerr metric)."""
    import numpy as np
    import torch
    import disco_b200 as db
    from disco_b200.workloads import write_par
    hbm, kind = peaks()
    over = dict(C3_GRID, Metric_Par3=0.9)
    if args.c3_nz != C3_GRID["Num_Z"]:           # a slice of the torus (profiling runs)
        over.update(Num_Z=args.c3_nz, Z_Min=-20.0 * args.c3_nz / 96, Z_Max=20.0 * args.c3_nz / 96)
    p = write_par(over, base="c3_grtorus")
    disk = db.Disk.from_files(p, os.path.join(db.TEMPLATES, "c3_grtorus_kerr.in"))
    os.unlink(p)
    nsteps = 10
    out = {"workload": "GRMHD torus, Kerr-Schild a=0.9, HLL, Nr=%d Nz=%d (real), Np %d, %d real cells"
                       % (C3_GRID["Num_R"], over["Num_Z"], int(np.max(disk.Np)), disk.nreal),
           "steps": nsteps, "warmup": 3}
    b = db.Batch([disk], device=local)
    b.set_stream(stream.cuda_stream)
    b.run(3)
    b.sync()
    kt = {}
    for name, t in b.kernel_times():
        kt[name] = kt.get(name, 0.0) + t
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    b.run(nsteps)
    e1.record(stream)
    e1.synchronize()
    if b.last_error() != 0:
        raise RuntimeError("device error in the config-3 leg")
    ms = e0.elapsed_time(e1)
    zu = disk.nreal * nsteps / (ms / 1e3)
    st = b.get_cells()
    r = disk.real == 1
    out["fp64"] = {"zone_updates_per_s": zu, "ms_per_step": ms / nsteps,
                   "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(kt.items(), key=lambda x: -x[1])},
                   "step_roofline": {"bytes_per_zone_update": B_ALG_GR, "achieved": B_ALG_GR * zu / 1e9,
                                     "peak": hbm, "unit": "GB/s", "frac": B_ALG_GR * zu / 1e9 / hbm,
                                     "peak_kind": kind},
                   "finite": bool(np.isfinite(st["prim"][r]).all())}
    del st
    b.close()
    if rank0_cpu(args):
        out["cpu_baseline"] = reference_slice_rate(
            "c3_grtorus", dict(C3_GRID, Num_Z=8, Z_Min=-20.0 * 8 / 96, Z_Max=20.0 * 8 / 96), 2,
            "reference grmhd2 + schw_ks_rpz (a = 0; the reference has no Kerr metric), the full r grid "
            "and Np on 8 z layers, 2 steps, one process")
    return out


def rank0_cpu(args):
    return not args.no_cpu_baseline and int(os.environ.get("RANK", "0")) == 0


def write_par_text(base, overrides):
    """A bundled template in.par with keys replaced, as text."""
    out = []
    with open(os.path.join(REPO, "disco_b200", "templates", base + ".par")) as f:
        for line in f:
            tok = line.split()
            if tok and tok[0] in overrides:
                line = "%s\t\t%s\n" % (tok[0], overrides[tok[0]])
            out.append(line)
    return "".join(out)


C2P_GRID = {"Nr": 192, "Nz": 96, "Np": 462, "rmin": 1.5, "rmax": 50.0, "zmin": -20.0, "zmax": 20.0}
C2P_TOL, C2P_NEXTRA, C2P_MAXIT = 1e-10, 10, 30
C2P_BYTES = 8 * (9 + 3 + 5 + 9)         # read cons, x, the 5 prims of the warm start; write prims


def c2p_leg(args, local, stream):
    """GRMHD cons -> prim on the torus workload (Kerr-KS a = 0.9): the
    network is trained on pairs written by plain solves of four perturbation
    sizes, then plain (previous prims) and learned guesses are timed on fresh
    states, both finished by Newton to |d eta/eta| < 1e-10 with the
    reference's tail of 10 and cap of 30."""
    import numpy as np
    import torch
    from disco_b200.gr import GR

    g = C2P_GRID
    gr = GR(device=local, metric="kerr", a=0.9, tol=C2P_TOL, nextra=C2P_NEXTRA, max_iter=C2P_MAXIT)
    gr.set_stream(stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    out = {"workload": "GRMHD torus, Kerr-KS a=0.9, %dx%dx%d cells (r %.1f-%.0f log, z +-%.0f)" %
                       (g["Nr"], g["Nz"], g["Np"], g["rmin"], g["rmax"], g["zmax"]),
           "tol": C2P_TOL, "nextra": C2P_NEXTRA, "max_iter": C2P_MAXIT}
    with torch.cuda.stream(stream):
        x = gr.grid(g["Nr"], g["Nz"], g["Np"], g["rmin"], g["rmax"], g["zmin"], g["zmax"])
        p0 = gr.torus(x)
        n = x.shape[1]
        out["ncell"] = n
        pairs = []
        for seed, eps in ((101, 1e-3), (102, 3e-2), (103, 0.1), (104, 0.3)):
            cons = gr.prim2cons(gr.perturb(p0, seed, eps), x)
            pr = p0.clone()
            pairs.append(gr.cons2prim(cons, x, pr, pairs=True, stats=False)["pairs"])
            del cons, pr
        pairs = torch.cat(pairs)
        gr.mlp_init(3)
        gr.mlp_fit_norm(pairs)
        steps, batch = 3000, 8192
        ev[0].record(stream)
        hist = gr.mlp_train(pairs, steps=steps, batch=batch, lr=2e-3, seed=9)
        ev[1].record(stream)
        ev[1].synchronize()
        out["train"] = {"pairs": int(pairs.shape[0]), "steps": steps, "batch": batch,
                        "ms": ev[0].elapsed_time(ev[1]), "loss_first": float(hist[:10].mean()),
                        "loss_last": float(hist[-50:].mean())}
        del pairs
        # the same network in a solver without the tail (tol only)
        gr0 = GR(device=local, metric="kerr", a=0.9, tol=C2P_TOL, nextra=0, max_iter=C2P_MAXIT)
        gr0.set_stream(stream)
        gr0.mlp_set(*gr.mlp_get())
        work = torch.empty_like(p0)
        hbm, _ = peaks()
        for name, eps in (("warm", 1e-3), ("jump", 0.3)):
            cons = gr.prim2cons(gr.perturb(p0, 777, eps), x)
            for solver, tail in ((gr, ""), (gr0, "_tail0")):
                row = {"eps": eps, "nextra": C2P_NEXTRA if solver is gr else 0}
                for guess, key in (("previous", "plain"), ("learned", "learned")):
                    ts = []
                    for r in range(4):
                        work.copy_(p0)
                        ev[0].record(stream)
                        solver.cons2prim(cons, x, work, guess=guess, stats=False)
                        ev[1].record(stream)
                        ev[1].synchronize()
                        if r:
                            ts.append(ev[0].elapsed_time(ev[1]))
                    work.copy_(p0)
                    rep = solver.cons2prim(cons, x, work, guess=guess)
                    ms = statistics.median(ts)
                    gbs = C2P_BYTES * n / (ms / 1e3) / 1e9
                    row[key] = {"ms": ms, "cells_per_s": n / (ms / 1e3), "iters_mean": rep["iters_mean"],
                                "iters_max": rep["iters_max"], "n_fallback": rep["n_fallback"],
                                "n_fail": rep["n_fail"], "hbm_gbs": gbs, "hbm_frac": gbs / hbm}
                row["learned_speedup"] = row["plain"]["ms"] / row["learned"]["ms"]
                row["learned_iteration_ratio"] = row["learned"]["iters_mean"] / row["plain"]["iters_mean"]
                out[name + tail] = row
            del cons
        del gr0
        out["bytes_per_cell"] = C2P_BYTES
        # CPU baseline: the oracle restatement (same tol/tail/cap), one core,
        # on the first 50k cells of the warm case
        if not args.no_cpu_baseline:
            try:
                from oracle import pyc2p
                m = 50000
                xs = x[:, :m].T.cpu().numpy().copy()
                pp = p0[:, :m].T.cpu().numpy().copy()
                cs = gr.prim2cons(gr.perturb(p0, 777, 1e-3), x)[:, :m].T.cpu().numpy().copy()
                orc = pyc2p.C2POracle(metric=1, a=0.9, tol=C2P_TOL, nextra=C2P_NEXTRA, max_iter=C2P_MAXIT)
                t0 = time.perf_counter()
                orc.cons2prim(cs, xs, pp)
                dt = time.perf_counter() - t0
                out["cpu_baseline"] = {"value": m / dt, "unit": "cells/s", "cores": 1, "kind": "port",
                                       "sample": "%d cells of the warm case, oracle restatement" % m}
            except Exception as ex:
                out["cpu_baseline"] = {"value": None, "sample": "unavailable: %s" % ex}
    del gr
    return out


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    import disco_b200 as db

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
        pg = dist

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    from disco_b200.replicas import job_rate, max_over_ranks

    def allmax(x):
        return max_over_ranks(x, pg, device="cuda")

    disks = make_disks(args.workload, rank)
    b = db.Batch(disks, device=local)
    nreal = sum(d.nreal for d in disks)
    ncell = b.ncell
    nf = sum(int(sum(d.Np[j] + d.Np[j + 1] for j in range(d.Nr - 1))) for d in disks)
    na = sum(d.Nr * d.Nz for d in disks)

    stream = torch.cuda.Stream(device=local)
    b.set_stream(stream.cuda_stream)
    b.run(args.warmup)
    b.sync()

    # per-kernel device times of one step (events between launches, same stream)
    kt = b.kernel_times()
    launches_per_step = len(kt)

    barrier()
    clocks = Clocks(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        b.run(args.steps)
        e1.record(stream)
    e1.synchronize()
    ck = clocks.stop()
    barrier()
    if b.last_error() != 0:
        raise RuntimeError("device error during the timed region: %s" % db.STATUS.get(b.last_error()))
    ms = allmax(e0.elapsed_time(e1))
    value = job_rate(world, nreal, args.steps, ms)

    # roofline of the dominant kernel (sum over its launches in the step)
    hbm, peak_kind = peaks()
    tot, byt, seen = {}, {}, {}
    for name, t in kt:
        first = seen.get(name, 0) == 0
        seen[name] = seen.get(name, 0) + 1
        tot[name] = tot.get(name, 0.0) + t
        byt[name] = byt.get(name, 0) + kernel_bytes(name, first, ncell, nf, na, nreal)
    dom = max(tot, key=tot.get)
    achieved = byt[dom] / (tot[dom] / 1e3) / 1e9
    # DRAM bytes of one launch of the dominant kernel: the ncu capture of the
    # same kernel on the smaller ragged8 workload, scaled by the cells (r-faces
    # for k_flux_r) one launch here processes -- the ragged workloads' traffic
    # grows with the cells, each cell's state crossing HBM once
    per_unit = {"k_update": (DRAM_UPDATE_RAGGED8, "cells"), "k_flux_r": (DRAM_FLUX_RAGGED8, "faces")}
    traffic = None
    if dom in per_unit and args.workload.startswith("ragged"):
        (b8, units8), kind = per_unit[dom]
        traffic = b8 / units8 * (ncell if kind == "cells" else nf)
    step_gbs = B_ALG_STEP * (value / world) / 1e9

    # the same step as one persistent launch (disco_batch_set_schedule), for
    # comparison with the default multi-kernel step timed above
    sched_cmp = None
    try:
        b.schedule = db.SCHED_PERSISTENT
    except db.DiscoError:
        pass
    if b.schedule == db.SCHED_PERSISTENT:
        b.run(args.warmup)
        b.sync()
        kt_k = b.kernel_times()
        barrier()
        h0 = torch.cuda.Event(enable_timing=True)
        h1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            h0.record(stream)
            b.run(args.steps)
            h1.record(stream)
        h1.synchronize()
        barrier()
        kms = allmax(h0.elapsed_time(h1))
        ktot = {}
        for name, t in kt_k:
            ktot[name] = ktot.get(name, 0.0) + t
        sched_cmp = {"schedule": "persistent one-launch step", "ms_per_step": kms / args.steps,
                     "value": job_rate(world, nreal, args.steps, kms),
                     "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(ktot.items(), key=lambda x: -x[1])},
                     "launches_per_step": len(kt_k)}
        b.schedule = db.SCHED_KERNELS

    # end to end through the C ABI with host buffers: upload the state from
    # host memory, K x {dt = getmindt() -> host; timestep(dt) from host},
    # download the state.
    # Host buffers are pinned (the state a host code keeps between outputs).
    keep = []

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.from_numpy(np.ascontiguousarray(a)).dtype, pin_memory=True)
        keep.append(t)
        n = t.numpy()
        n[...] = a
        return n
    st = {k: pinned(v) for k, v in b.get_cells().items()}
    out_bufs = {k: pinned(np.zeros_like(v)) for k, v in st.items()}
    h2d = (st["prim"].nbytes + st["cons"].nbytes + st["piph"].nbytes + st["dphi"].nbytes
           + st["wiph"].nbytes + 4 * ncell)
    d2h = h2d - 4 * ncell
    real = pinned(np.concatenate([d.real for d in disks]).astype(np.int32))
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    t_wall = time.perf_counter()
    b.set_cells(st["prim"], st["cons"], st["piph"], st["dphi"], st["wiph"], real)
    for _ in range(args.steps):
        dt = b.mindt()
        b.timestep(dt)
    out = b.get_cells(out=out_bufs)
    f1.record(stream)
    f1.synchronize()
    t_wall = time.perf_counter() - t_wall
    e2e_ms = allmax(max(f0.elapsed_time(f1), t_wall * 1e3))
    e2e = world * nreal * args.steps / (e2e_ms / 1e3)
    del out

    # the mixed-precision form on the same disks, timed the same way
    mixed = None
    if not args.no_mixed:
        bm = db.Batch(disks, device=local, precision=db.PREC_MIXED)
        bm.set_stream(stream.cuda_stream)
        bm.run(args.warmup)
        bm.sync()
        barrier()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            g0.record(stream)
            bm.run(args.steps)
            g1.record(stream)
        g1.synchronize()
        barrier()
        if bm.last_error() != 0:
            raise RuntimeError("device error in the mixed-form timed region")
        mms = allmax(g0.elapsed_time(g1))
        mv = world * nreal * args.steps / (mms / 1e3)
        mixed = {"value": mv, "unit": "zone-updates/s", "ms_per_step": mms / args.steps,
                 "speedup_vs_fp64": mv / value,
                 "precision": "FP32 prim/slopes/fluxes, FP64 mesh/dt/Kahan cons"}
        bm.close()

    config1 = None
    if not args.no_config1:
        config1 = config1_leg(args, local, stream)
        barrier()

    config4 = None
    if not args.no_config4:
        config4 = config4_leg(args, local, stream)
        barrier()

    config3 = None
    if not args.no_config3:
        config3 = config3_leg(args, local, stream)
        barrier()

    c2p = None
    if not args.no_c2p:
        c2p = c2p_leg(args, local, stream)
        barrier()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            v, cores, sample, _ = time_reference(args.workload, 1)
            cpu = {"value": v, "unit": "zone-updates/s", "cores": cores, "kind": "reference",
                   "sample": sample}
        except Exception as ex:  # reference binary missing on this machine
            cpu = {"value": None, "unit": "zone-updates/s", "cores": 0, "kind": "reference",
                   "sample": "unavailable: %s" % ex}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "zone-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": workload_config(args.workload, nreal),
            "layout": {"cells_per_gpu_incl_ghosts": ncell, "r_faces_per_gpu": nf,
                       "precision": "fp64 plain path"},
            "parallelism": "independent disks per GPU" if world > 1 else "single GPU",
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm,
                         "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                         "traffic_source": ("ncu capture on ragged8 (dram bytes of one %s launch), "
                                            "scaled by the units processed" % dom)
                         if traffic is not None else None,
                         "peak_kind": peak_kind},
            "step_roofline": {"bytes_per_zone_update": B_ALG_STEP, "achieved": step_gbs, "peak": hbm,
                              "unit": "GB/s", "frac": step_gbs / hbm},
            "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(tot.items(), key=lambda x: -x[1])},
            "schedule": "persistent one-launch step" if dom == "k_step" else "one kernel per pass",
            "persistent_schedule": sched_cmp,
            "e2e": {"value": e2e, "unit": "zone-updates/s",
                    "h2d_bytes_per_step": (h2d + 8 * len(disks) * args.steps) / args.steps,
                    "d2h_bytes_per_step": (d2h + 8 * len(disks) * args.steps) / args.steps},
            "gpu_launches": launches_per_step * args.steps,
            "mixed_form": mixed,
            "config1_mhd3d": config1,
            "config3_grtorus": config3,
            "config4_binary3d": config4,
            "c2p": c2p,
            "clocks": ck,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    b.close()
    if pg:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ragged64", choices=["ragged64", "ragged8", "config0"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-c2p", action="store_true", help="skip the GRMHD cons->prim leg")
    ap.add_argument("--no-config1", action="store_true", help="skip the 3D MHD (config 1) leg")
    ap.add_argument("--no-config3", action="store_true", help="skip the GRMHD torus (config 3) leg")
    ap.add_argument("--c3-nz", type=int, default=96, help="z layers of the config-3 torus (96)")
    ap.add_argument("--only-config3", action="store_true",
                    help="run the config-3 leg alone (no headline line), e.g. for profiling")
    ap.add_argument("--no-config4", action="store_true",
                    help="skip the 40M-cell 3D MHD circumbinary (config 4) leg")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world, rank, local = dist_setup()
    if args.only_config3:
        import torch
        torch.cuda.set_device(local)
        args.no_cpu_baseline = True
        print(json.dumps({"config3_grtorus": config3_leg(args, local, torch.cuda.Stream(device=local))}),
              flush=True)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
