#!/usr/bin/env python
"""Benchmark of the B200 Disco RK timestep (zone-updates/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload config4|ragged64|ragged8|config0]

A step is one full RK2 timestep (two substeps, fused getmindt) of every disk
of the workload, inputs resident in HBM.  Default workload `config4`, the
largest single-GPU configuration: the 3D MHD circumbinary disk (HLLD,
constrained transport, softened equal-mass binary, zerograd; 384 x 128
annuli, Np up to 1536, 39.5M real cells) in its stated form -- FP32 bulk
(prims, slopes, fluxes, edge fields) with FP64 cell positions, mesh motion,
dt and a Kahan-compensated FP64 conserved update -- with the FP64 plain path
on the same set-up beside it (throughput, roofline, L1 error and drifts of
the FP32 form against it).  The other configurations run as side legs:
config 1 (3D MHD shearing disk), config 2 (`ragged64`, 64 ragged 2D hydro
disks in one batch), config 3 (GRMHD torus) and the cons->prim leg.
Multi-GPU: one process per GPU (torchrun), each GPU advances its own copy of
the workload (independent disks, no data-path collective, "scaling":
"weak"); only a barrier and a max of the timings over ranks.

--impl reference times the reference Disco serial CPU code itself
(oracle/_ref, built from the reference's own sources) on the same module
set, spread over all host cores: for config4 one process per core, each on
the full r grid and Np of the workload on a 4-layer z slab; for the ragged
workloads one process per disk.
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
B_ALG_MHD_CT = {"fp64": 1056, "mixed": 1200}   # HBM bytes per zone-update, MHD Q=9 with CT (5 faces)
C4_NZ = 128
C4_REAL_PER_LAYER = 308974              # real cells of one z layer of config 4 (Np depends on r only)


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


def kernel_bytes_mhd(name, first, N, Nfr, Nfz, mixed):
    """Algorithmic HBM bytes of one launch of a step kernel on a 3D MHD grid
    with constrained transport (Q = 9, 5 face-flux slots per cell): every
    array element the kernel must read or write, once.  N cells (ghosts
    included), Nfr / Nfz r- and z-faces.  In the mixed form the prims, slopes
    and fluxes are FP32 and the conserved update carries an FP32 Kahan term;
    cons, RKcons, piph, dphi, wiph and the face fluxes Phi stay FP64."""
    q, w = 9, 8
    wr = 4 if mixed else 8
    ck = 4 if mixed else 0               # Kahan carry per conserved variable
    phi = 5 * w
    if name == "k_update":
        # cons (+carry) read and written, prim and gradp, piph / dphi / wiph,
        # the four consume indices, the phi-face EMFs written (4); the r- and
        # z-face fluxes read
        return N * (2 * q * (w + ck) + 2 * q * wr + 3 * w + 16 + 4 * wr) + (Nfr + Nfz) * q * wr
    if name in ("k_flux_r", "k_flux_z"):
        nf = Nfr if name == "k_flux_r" else Nfz
        # per face: its two cells, its geometry, the flux and the two edge
        # terms written; per cell once: prim, the slope in this direction, gradp
        return nf * (8 + 3 * w + q * wr + 2 * wr) + N * (3 * q * wr + 2 * w)
    if name == "k_c2p":
        # cons (+carry), piph / dphi (moved in the first substep), the face
        # fluxes rebuilt into the cell field, the prims written (+wiph last)
        return N * (q * (w + ck) + 2 * w + phi + 3 * w + q * wr) + (0 if first else N * w)
    if name == "k_begin":
        rk = q * w if first else q * (w + 2 * ck)
        return N * (2 * q * wr + 2 * q * w + rk + 2 * w + (2 * w if first else 0) + 3 * phi)
    if name in ("k_gradr", "k_gradz"):
        nf = Nfr if name == "k_gradr" else Nfz
        return nf * (q * wr + w) + N * (q * wr + 2 * w + 8)
    if name == "k_grad":
        # r and z in one launch: both face sets, both gradients written
        return (Nfr + Nfz) * (q * wr + w) + N * (2 * q * wr + 2 * w + 16)
    if name == "k_faces":
        nf = Nfr + Nfz
        if first:
            return N * (2 * w + 2 * q * wr) + nf * (8 + w + q * wr)
        return N * (2 * w + 2 * q * wr + 16) + nf * (9 + 3 * w + q * wr)
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


def c4_disk(nz=C4_NZ):
    """The config-4 disk; nz < 128 takes the mid-plane slab of nz layers
    (the same dz) for reduced profiling runs."""
    from disco_b200.workloads import config4_disk
    return config4_disk(nz)


def make_disks(workload, rank, c4_nz=C4_NZ):
    from disco_b200 import workloads
    if workload == "config4":
        return [c4_disk(c4_nz)]
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
NDISK = {"ragged64": 64, "ragged8": 8, "config0": 1, "config4": 1}


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


def workload_config(workload, nreal, c4_nz=C4_NZ):
    """The `config` object of both arms' lines: the workload, nothing of
    either implementation."""
    if workload == "config4":
        return {"workload": "config4" + ("" if c4_nz == C4_NZ else "_nz%d" % c4_nz),
                "description": "3D MHD circumbinary disk, softened equal-mass binary (eps 0.05, "
                               "separation 1), HLLD + constrained transport",
                "disks_per_gpu": 1, "real_cells_per_gpu": int(nreal),
                "grid": "Nr 384 (r in [0.5, 10], linear) x Nz %d (z in [-0.5, 0.5] at 128), aspect 1.66, "
                        "Np up to 1536: %d real cells (changed from the configuration's 'about 50M', "
                        "which Np <= 1536 on 384 x 128 annuli cannot reach)" % (c4_nz, nreal),
                "physics": "MHD, HLLD, PLM 1.5, RK2, CFL 0.2, CT_MODE 2, binary_soft planets, "
                           "zerograd boundaries, Mesh_Motion 3, diag_disk2d",
                "precision": "FP32 bulk (prims, slopes, fluxes, edge fields), FP64 piph / mesh / dt / "
                             "Kahan-compensated conserved update and face fluxes",
                "l2_policy": "inputs larger than L2 (%.1f GB of prim+cons state per GPU)"
                             % (nreal * (4 + 8) * 9 / 1e9)}
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


C4_SLAB_NZ = 4


def time_reference_c4(nsteps, max_workers=None):
    """The reference's serial CPU code on the config-4 module set (mhd,
    hlld, CT_MODE 2, binary_soft, zerograd): one process per host core,
    each the full 384-annulus r grid and Np on a 4-layer mid-plane z slab
    (the slabs a z decomposition of the workload would give each core).
    Returns (zone-updates/s summed over the processes over the slowest
    process's step-loop time, cores, sample description, real cells of one
    slab)."""
    import pyoracle
    binary = pyoracle.ref_binary("c4_binary3d")
    if not os.path.exists(binary):
        pyoracle.build_ref("c4_binary3d")
    cores = max_workers or min(os.cpu_count() or 1, 32)
    text = write_par_text("c4_binary3d", {"Num_Z": C4_SLAB_NZ, "Z_Min": -0.5 * C4_SLAB_NZ / C4_NZ,
                                          "Z_Max": 0.5 * C4_SLAB_NZ / C4_NZ})
    work, procs = [], []
    for w in range(cores):
        d = tempfile.mkdtemp(prefix="dref4_")
        with open(os.path.join(d, "in.par"), "w") as f:
            f.write(text)
        work.append(d)
        procs.append(subprocess.Popen([binary, d, str(nsteps), "--time"], stdout=subprocess.PIPE, text=True))
    secs, zones, cells = [], 0, 0
    for pr in procs:
        out, _ = pr.communicate(timeout=1800)
        r = json.loads([l for l in out.splitlines() if l.startswith("{")][0])
        secs.append(r["seconds"])
        zones += r["real_cells"] * r["steps"]
        cells = r["real_cells"]
    for d in work:
        subprocess.run(["rm", "-rf", d])
    sample = ("config4 module set, %d processes on %d cores, each the full r grid and Np on a %d-layer "
              "z slab (%d real cells) for %d step(s), step-loop time only"
              % (cores, cores, C4_SLAB_NZ, cells, nsteps))
    return zones / max(secs), cores, sample, cells


def run_reference(args, world, rank):
    if rank != 0:
        return
    if args.workload == "config4":
        v, cores, sample, _ = time_reference_c4(max(1, args.steps // 10))
        nreal = C4_REAL_PER_LAYER * args.c4_nz
    else:
        v, cores, sample, nreal = time_reference(args.workload, max(1, args.steps // 4))
    line = {"metric": METRIC, "value": v, "unit": "zone-updates/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": workload_config(args.workload, nreal, args.c4_nz),
            "parallelism": ("one host process per core (z slabs)" if args.workload == "config4"
                            else "one host process per disk"),
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


def c3_disk(nz=96):
    """The config-3 torus disk (Kerr-Schild a = 0.9); nz < 96 takes the
    mid-plane slice of nz layers (profiling runs).  Returns (disk, overrides)."""
    import disco_b200 as db
    from disco_b200.workloads import write_par
    over = dict(C3_GRID, Metric_Par3=0.9)
    if nz != C3_GRID["Num_Z"]:
        over.update(Num_Z=nz, Z_Min=-20.0 * nz / 96, Z_Max=20.0 * nz / 96)
    p = write_par(over, base="c3_grtorus")
    try:
        return db.Disk.from_files(p, os.path.join(db.TEMPLATES, "c3_grtorus_kerr.in")), over
    finally:
        os.unlink(p)


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
    hbm, kind = peaks()
    disk, over = c3_disk(args.c3_nz)
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


C2P_TOL, C2P_NEXTRA, C2P_MAXIT = 1e-10, 10, 30
C2P_BYTES = 8 * (9 + 3 + 5 + 9)         # read cons, x, the 5 prims of the warm start; write prims
C2P_DUMPS = 4                           # steps dumped: 3 for training pairs, the last for timing


def c2p_leg(args, local, stream):
    """GRMHD cons -> prim on the states of the config-3 run (the Kerr-Schild
    a = 0.9 torus, 192 x 96 annuli of 463 cells): after 3 warm-up steps the
    step's own cons->prim inputs of 4 consecutive steps are dumped
    (disco_batch_set_gr_dump: cons / dV, the warm-start prims, x of every
    real cell).  The plain solver writes the training pairs on the first
    three; the network is trained on them; on the fourth, plain (the cell's
    previous prims, as the step starts) and learned guesses are timed, both
    finished by Newton to |d eta/eta| < 1e-10 with the reference's tail of
    10 (and without it) and cap of 30; "jump" starts both from prims
    perturbed by 30% instead, where the previous state is far."""
    import numpy as np
    import torch
    import disco_b200 as db
    from disco_b200.gr import GR

    disk, over = c3_disk(args.c3_nz)
    r = torch.from_numpy(disk.real == 1).to("cuda:%d" % local)
    idx = torch.nonzero(r).squeeze(1)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    out = {"workload": "cons->prim inputs of the config-3 GRMHD torus step (Kerr-Schild a=0.9, Nr=%d "
                       "Nz=%d, Np %d), dumped from %d consecutive steps after 3 warm-up steps"
                       % (C3_GRID["Num_R"], over["Num_Z"], int(np.max(disk.Np)), C2P_DUMPS),
           "tol": C2P_TOL, "nextra": C2P_NEXTRA, "max_iter": C2P_MAXIT}
    with torch.cuda.stream(stream):
        b = db.Batch([disk], device=local)
        b.set_stream(stream.cuda_stream)
        b.run(3)
        b.sync()
        buf = torch.zeros((db.GR_DUMP_ROWS, b.ncell), dtype=torch.float64, device=idx.device)
        b.set_gr_dump(buf)
        dumps = []
        for _ in range(C2P_DUMPS):
            b.timestep(b.mindt()[0])
            torch.cuda.current_stream().wait_stream(stream)
            b.sync()
            dumps.append(buf[:, idx].contiguous())
        b.set_gr_dump(None)
        b.close()
        del buf
        n = int(idx.numel())
        out["ncell"] = n
        gr = GR(device=local, gamma_law=1.3333333333333, rho_floor=0.0, p_floor=0.0, M=1.0, a=0.9,
                metric="kerr", tol=C2P_TOL, nextra=C2P_NEXTRA, max_iter=C2P_MAXIT)
        gr.set_stream(stream)
        pairs = []
        for dmp in dumps[:-1]:
            pr = dmp[9:18].clone()
            pairs.append(gr.cons2prim(dmp[0:9], dmp[18:21], pr, pairs=True, stats=False)["pairs"])
            del pr
        pairs = torch.cat(pairs)
        gr.mlp_init(3)
        gr.mlp_fit_norm(pairs)
        steps, batch = 3000, 8192
        # the CUDA-core backward first (timing only), then the tensor-core
        # (tcgen05) one whose network is used below
        gr.mlp_backend("cuda")
        ev[0].record(stream)
        hist_c = gr.mlp_train(pairs, steps=steps, batch=batch, lr=2e-3, seed=9)
        ev[1].record(stream)
        ev[1].synchronize()
        ms_cuda = ev[0].elapsed_time(ev[1])
        gr.mlp_init(3)
        gr.mlp_fit_norm(pairs)
        gr.mlp_backend("tensor")
        ev[0].record(stream)
        hist = gr.mlp_train(pairs, steps=steps, batch=batch, lr=2e-3, seed=9)
        ev[1].record(stream)
        ev[1].synchronize()
        out["train"] = {"pairs": int(pairs.shape[0]), "source": "the plain solver on the step's own inputs "
                        "of the first %d dumped steps" % (C2P_DUMPS - 1), "steps": steps, "batch": batch,
                        "backend": "tcgen05 tensor cores", "ms": ev[0].elapsed_time(ev[1]),
                        "loss_first": float(hist[:10].mean()), "loss_last": float(hist[-50:].mean()),
                        "cuda_cores_ms": ms_cuda, "cuda_cores_loss_last": float(hist_c[-50:].mean())}
        del pairs
        # the same network in a solver without the tail (tol only)
        gr0 = GR(device=local, gamma_law=1.3333333333333, rho_floor=0.0, p_floor=0.0, M=1.0, a=0.9,
                 metric="kerr", tol=C2P_TOL, nextra=0, max_iter=C2P_MAXIT)
        gr0.set_stream(stream)
        gr0.mlp_set(*gr.mlp_get())
        test = dumps[-1]
        cons, x, warm = test[0:9], test[18:21], test[9:18].contiguous()
        jump = gr.perturb(warm, 777, 0.3)
        work = torch.empty_like(warm)
        hbm, _ = peaks()
        for name, start in (("step", warm), ("jump", jump)):
            for solver, tail in ((gr, ""), (gr0, "_tail0")):
                row = {"start": "the previous prims" if name == "step" else "the previous prims x (1 + 0.3 u)",
                       "nextra": C2P_NEXTRA if solver is gr else 0}
                for guess, key in (("previous", "plain"), ("learned", "learned")):
                    ts = []
                    for rep in range(4):
                        work.copy_(start)
                        ev[0].record(stream)
                        solver.cons2prim(cons, x, work, guess=guess, stats=False)
                        ev[1].record(stream)
                        ev[1].synchronize()
                        if rep:
                            ts.append(ev[0].elapsed_time(ev[1]))
                    work.copy_(start)
                    rep_ = solver.cons2prim(cons, x, work, guess=guess)
                    ms = statistics.median(ts)
                    gbs = C2P_BYTES * n / (ms / 1e3) / 1e9
                    row[key] = {"ms": ms, "cells_per_s": n / (ms / 1e3), "iters_mean": rep_["iters_mean"],
                                "iters_max": rep_["iters_max"], "n_fallback": rep_["n_fallback"],
                                "n_fail": rep_["n_fail"], "hbm_gbs": gbs, "hbm_frac": gbs / hbm}
                row["learned_speedup"] = row["plain"]["ms"] / row["learned"]["ms"]
                row["learned_iteration_ratio"] = row["learned"]["iters_mean"] / row["plain"]["iters_mean"]
                out[name + tail] = row
        del gr0, jump, work
        out["bytes_per_cell"] = C2P_BYTES
        # CPU baseline: the oracle restatement (same tol/tail/cap), one core,
        # on 50k cells of the timed dump
        if not args.no_cpu_baseline:
            try:
                from oracle import pyc2p
                m = 50000
                xs = x[:, :m].T.cpu().numpy().copy()
                pp = warm[:, :m].T.cpu().numpy().copy()
                cs = cons[:, :m].T.cpu().numpy().copy()
                orc = pyc2p.C2POracle(metric=1, a=0.9, gam=1.3333333333333, rho_floor=0.0, p_floor=0.0,
                                      tol=C2P_TOL, nextra=C2P_NEXTRA, max_iter=C2P_MAXIT)
                t0 = time.perf_counter()
                orc.cons2prim(cs, xs, pp)
                dt = time.perf_counter() - t0
                out["cpu_baseline"] = {"value": m / dt, "unit": "cells/s", "cores": 1, "kind": "port",
                                       "sample": "%d cells of the timed dump, oracle restatement" % m}
            except Exception as ex:
                out["cpu_baseline"] = {"value": None, "sample": "unavailable: %s" % ex}
        del dumps, test
    del gr
    return out


def face_counts(disks):
    """(r-faces, z-faces) of the disks' face lists: each track's face count
    is the sum of its two annuli's Np (fIndex, faces_alt.c:97-100)."""
    nfr = nfz = 0
    for d in disks:
        Np = d.Np.reshape(d.Nz, d.Nr)
        nfr += int((Np[:, :-1] + Np[:, 1:]).sum())
        if d.Nz > 1:
            nfz += int((Np[:-1, :] + Np[1:, :]).sum())
    return nfr, nfz


def timed_run(b, stream, steps, barrier, allmax, clocks=None):
    """b.run(steps) between CUDA events on the batch's stream, barriers on
    both sides; returns (max over ranks of the ms, clock record)."""
    import torch
    barrier()
    if clocks:
        clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        b.run(steps)
        e1.record(stream)
    e1.synchronize()
    ck = clocks.stop() if clocks else None
    barrier()
    if b.last_error() != 0:
        import disco_b200 as db
        raise RuntimeError("device error during the timed region: %s" % db.STATUS.get(b.last_error()))
    return allmax(e0.elapsed_time(e1)), ck


def kernel_table(kt):
    tot, cnt = {}, {}
    for name, t in kt:
        tot[name] = tot.get(name, 0.0) + t
        cnt[name] = cnt.get(name, 0) + 1
    return tot, cnt


def dominant_roofline(kt, bytes_of, traffic_of):
    """Roofline object of the kernel with the largest device time in one
    instrumented step: algorithmic bytes of its launches over their time."""
    hbm, peak_kind = peaks()
    tot, byt, seen = {}, {}, {}
    for name, t in kt:
        first = seen.get(name, 0) == 0
        seen[name] = seen.get(name, 0) + 1
        tot[name] = tot.get(name, 0.0) + t
        byt[name] = byt.get(name, 0) + bytes_of(name, first)
    dom = max(tot, key=tot.get)
    achieved = byt[dom] / (tot[dom] / 1e3) / 1e9 if byt[dom] else None
    traffic, src = traffic_of(dom, seen[dom])
    return {"bound": "hbm", "kernel": dom, "launches_per_step": seen[dom],
            "bytes_per_launch": byt[dom] / seen[dom] if byt[dom] else None,
            "ms_per_launch": tot[dom] / seen[dom],
            "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm if achieved else None, "traffic": traffic, "traffic_source": src,
            "peak_kind": peak_kind}, tot


def ragged_leg(args, local, stream, barrier, allmax, rank, world):
    """Config 2: 64 ragged 2D hydro disks in one batch, FP64 plain path (the
    graph-replayed kernel-per-pass step and the persistent one-launch
    schedule), the mixed form, per-kernel times, the dominant kernel's
    roofline and the step roofline; the reference on the same 64 disks."""
    import disco_b200 as db
    disks = make_disks("ragged64", rank)
    b = db.Batch(disks, device=local)
    nreal, ncell = sum(d.nreal for d in disks), b.ncell
    nf, _ = face_counts(disks)
    na = sum(d.Nr * d.Nz for d in disks)
    b.set_stream(stream.cuda_stream)
    b.run(args.warmup)
    b.sync()
    kt = b.kernel_times()
    ms, _ = timed_run(b, stream, args.steps, barrier, allmax)
    value = world * nreal * args.steps / (ms / 1e3)

    def traffic_of(dom, n):
        per_unit = {"k_update": (DRAM_UPDATE_RAGGED8, ncell), "k_flux_r": (DRAM_FLUX_RAGGED8, nf)}
        if dom not in per_unit:
            return None, None
        (b8, u8), units = per_unit[dom]
        return b8 / u8 * units, ("ncu capture on ragged8 (dram bytes of one %s launch), scaled by the "
                                 "units processed" % dom)
    roof, tot = dominant_roofline(kt, lambda nm, first: kernel_bytes(nm, first, ncell, nf, na, nreal),
                                  traffic_of)
    hbm, _ = peaks()
    step_gbs = B_ALG_STEP * (value / world) / 1e9
    out = {"workload": workload_config("ragged64", nreal), "value": value, "unit": "zone-updates/s",
           "ms_per_step": ms / args.steps, "steps": args.steps, "warmup": args.warmup, "dtype": "f64",
           "layout": {"cells_per_gpu_incl_ghosts": ncell, "r_faces_per_gpu": nf},
           "roofline": roof,
           "step_roofline": {"bytes_per_zone_update": B_ALG_STEP, "achieved": step_gbs, "peak": hbm,
                             "unit": "GB/s", "frac": step_gbs / hbm},
           "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(tot.items(), key=lambda x: -x[1])},
           "launches_per_step": len(kt)}
    # the same step as one persistent launch (disco_batch_set_schedule)
    try:
        b.schedule = db.SCHED_PERSISTENT
    except db.DiscoError:
        pass
    if b.schedule == db.SCHED_PERSISTENT:
        b.run(args.warmup)
        b.sync()
        ktot, _ = kernel_table(b.kernel_times())
        kms, _ = timed_run(b, stream, args.steps, barrier, allmax)
        out["persistent_schedule"] = {
            "schedule": "persistent one-launch step", "ms_per_step": kms / args.steps,
            "value": world * nreal * args.steps / (kms / 1e3),
            "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(ktot.items(), key=lambda x: -x[1])}}
        b.schedule = db.SCHED_KERNELS
    b.close()
    if not args.no_mixed:
        bm = db.Batch(disks, device=local, precision=db.PREC_MIXED)
        bm.set_stream(stream.cuda_stream)
        bm.run(args.warmup)
        bm.sync()
        mms, _ = timed_run(bm, stream, args.steps, barrier, allmax)
        mv = world * nreal * args.steps / (mms / 1e3)
        out["mixed_form"] = {"value": mv, "unit": "zone-updates/s", "ms_per_step": mms / args.steps,
                             "speedup_vs_fp64": mv / value,
                             "precision": "FP32 prim/slopes/fluxes, FP64 mesh/dt/Kahan cons"}
        bm.close()
    if rank0_cpu(args) and world == 1:
        try:
            v, cores, sample, _ = time_reference("ragged64", 1)
            out["cpu_baseline"] = {"value": v, "unit": "zone-updates/s", "cores": cores, "kind": "reference",
                                   "sample": sample}
        except Exception as ex:
            out["cpu_baseline"] = {"value": None, "sample": "unavailable: %s" % ex}
    return out


# dram__bytes_read.sum + dram__bytes_write.sum of one k_update launch of the
# mixed form on the config-4 slab of 12 z layers (4,995,072 cells with
# ghosts), from an ncu capture: (bytes, cells of that slab)
DRAM_UPDATE_C4 = (1675015000 + 503760128, 4995072)


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

    from disco_b200.replicas import max_over_ranks

    def allmax(x):
        return max_over_ranks(x, pg, device="cuda")

    c4 = args.workload == "config4"
    disks = make_disks(args.workload, rank, args.c4_nz)
    prec = db.PREC_MIXED if c4 else db.PREC_FP64
    b = db.Batch(disks, device=local, precision=prec)
    nreal = sum(d.nreal for d in disks)
    ncell = b.ncell
    nfr, nfz = face_counts(disks)
    na = sum(d.Nr * d.Nz for d in disks)

    stream = torch.cuda.Stream(device=local)
    b.set_stream(stream.cuda_stream)
    b.run(args.warmup)
    b.sync()
    # per-kernel device times of one step (events between launches, same stream)
    kt = b.kernel_times(cap=128)
    launches_per_step = len(kt)
    clocks = Clocks(local)
    ms, ck = timed_run(b, stream, args.steps, barrier, allmax, clocks)
    value = world * nreal * args.steps / (ms / 1e3)
    hbm, peak_kind = peaks()

    if c4:
        def bytes_of(name, first):
            return kernel_bytes_mhd(name, first, ncell, nfr, nfz, mixed=True)

        def traffic_of(dom, n):
            if dom != "k_update" or DRAM_UPDATE_C4 is None:
                return None, None
            bb, cells = DRAM_UPDATE_C4
            return bb / cells * ncell, ("ncu capture of one k_update launch on the 12-layer config-4 "
                                        "slab, scaled by the cells processed")
        b_step = B_ALG_MHD_CT["mixed"]
    else:
        def bytes_of(name, first):
            return kernel_bytes(name, first, ncell, nfr, na, nreal)

        def traffic_of(dom, n):
            per_unit = {"k_update": (DRAM_UPDATE_RAGGED8, ncell), "k_flux_r": (DRAM_FLUX_RAGGED8, nfr)}
            if dom not in per_unit or not args.workload.startswith("ragged"):
                return None, None
            (b8, u8), units = per_unit[dom]
            return b8 / u8 * units, ("ncu capture on ragged8 (dram bytes of one %s launch), scaled by "
                                     "the units processed" % dom)
        b_step = B_ALG_STEP
    roof, tot = dominant_roofline(kt, bytes_of, traffic_of)
    step_gbs = b_step * (value / world) / 1e9

    # the FP64 plain path on the same set-up and the same step sequence
    # (config 4): its throughput and roofline, and the FP32 form's error and
    # drifts against it
    fp64 = None
    if c4:
        r = np.concatenate([d.real for d in disks]) == 1
        sm = b.get_cells()
        b64 = db.Batch(disks, device=local)
        b64.set_stream(stream.cuda_stream)
        s0 = b64.get_cells()
        tot0 = {q: float(s0["cons"][r, q].sum()) for q in (0, 3)}
        del s0
        b64.run(args.warmup)
        b64.sync()
        kt64 = b64.kernel_times(cap=128)
        ms64, _ = timed_run(b64, stream, args.steps, barrier, allmax)
        v64 = world * nreal * args.steps / (ms64 / 1e3)
        roof64, tot64 = dominant_roofline(kt64, lambda nm, first: kernel_bytes_mhd(nm, first, ncell, nfr, nfz,
                                                                                   mixed=False),
                                          lambda dom, n: (None, None))
        sa = b64.get_cells()
        b64.close()
        names = ["rho", "P", "v_r", "omega", "v_z", "B_r", "B_phi", "B_z", "X"]
        err = {}
        for q, nm in enumerate(names):
            den = np.abs(sa["prim"][r, q]).sum()
            err[nm] = float(np.abs(sm["prim"][r, q] - sa["prim"][r, q]).sum() / den) if den > 0 else None
        ctot = lambda st, q: float(st["cons"][r, q].sum())
        g64 = B_ALG_MHD_CT["fp64"] * (v64 / world) / 1e9
        fp64 = {"value": v64, "unit": "zone-updates/s", "ms_per_step": ms64 / args.steps,
                "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(tot64.items(), key=lambda x: -x[1])},
                "roofline": roof64,
                "step_roofline": {"bytes_per_zone_update": B_ALG_MHD_CT["fp64"], "achieved": g64, "peak": hbm,
                                  "unit": "GB/s", "frac": g64 / hbm},
                "mixed_speedup_vs_fp64": value / v64,
                "mixed_rel_l1_vs_fp64": err,
                "drift": {"mass_fp64": ctot(sa, 0) / tot0[0] - 1.0, "mass_mixed": ctot(sm, 0) / tot0[0] - 1.0,
                          "ang_mom_fp64": ctot(sa, 3) / tot0[3] - 1.0,
                          "ang_mom_mixed": ctot(sm, 3) / tot0[3] - 1.0},
                "note": "both forms from the same set-up after %d warm-up + 1 instrumented + %d timed steps"
                        % (args.warmup, args.steps)}
        del sa, sm

    # end to end through the C ABI with host buffers: upload the state from
    # pinned host memory, K x {dt = getmindt() -> host; timestep(dt) from
    # host}, download the state into the same buffers.
    keep = []

    def pinned(a):
        t = torch.empty(a.shape, dtype=torch.from_numpy(np.ascontiguousarray(a)).dtype, pin_memory=True)
        keep.append(t)
        n = t.numpy()
        n[...] = a
        return n
    st = {k: pinned(v) for k, v in b.get_cells().items()}
    real = pinned(np.concatenate([d.real for d in disks]).astype(np.int32))
    h2d = sum(st[k].nbytes for k in st) + real.nbytes
    d2h = sum(st[k].nbytes for k in st)
    barrier()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    t_wall = time.perf_counter()
    b.set_cells(st["prim"], st["cons"], st["piph"], st["dphi"], st["wiph"], real, Phi=st.get("Phi"))
    for _ in range(args.steps):
        dt = b.mindt()
        b.timestep(dt)
    b.get_cells(out=st)
    f1.record(stream)
    f1.synchronize()
    t_wall = time.perf_counter() - t_wall
    e2e_ms = allmax(max(f0.elapsed_time(f1), t_wall * 1e3))
    e2e = world * nreal * args.steps / (e2e_ms / 1e3)
    del st, keep
    b.close()

    mixed = None
    if not c4 and not args.no_mixed:
        bm = db.Batch(disks, device=local, precision=db.PREC_MIXED)
        bm.set_stream(stream.cuda_stream)
        bm.run(args.warmup)
        bm.sync()
        mms, _ = timed_run(bm, stream, args.steps, barrier, allmax)
        mv = world * nreal * args.steps / (mms / 1e3)
        mixed = {"value": mv, "unit": "zone-updates/s", "ms_per_step": mms / args.steps,
                 "speedup_vs_fp64": mv / value,
                 "precision": "FP32 prim/slopes/fluxes, FP64 mesh/dt/Kahan cons"}
        bm.close()

    side = {}
    if c4 and not args.no_config2:
        side["config2_ragged64"] = ragged_leg(args, local, stream, barrier, allmax, rank, world)
        barrier()
    if not args.no_config1:
        side["config1_mhd3d"] = config1_leg(args, local, stream)
        barrier()
    if not c4 and not args.no_config4:
        side["config4_binary3d"] = config4_leg(args, local, stream)
        barrier()
    if not args.no_config3:
        side["config3_grtorus"] = config3_leg(args, local, stream)
        barrier()
    if not args.no_c2p:
        side["c2p"] = c2p_leg(args, local, stream)
        barrier()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            if c4:
                v, cores, sample, _ = time_reference_c4(1)
            else:
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
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if c4 else "f64", "data": "synthetic",
            "config": workload_config(args.workload, nreal, args.c4_nz),
            "layout": {"cells_per_gpu_incl_ghosts": ncell, "r_faces_per_gpu": nfr, "z_faces_per_gpu": nfz,
                       "precision": "mixed form" if c4 else "fp64 plain path"},
            "parallelism": "independent disks per GPU" if world > 1 else "single GPU",
            "roofline": roof,
            "step_roofline": {"bytes_per_zone_update": b_step, "achieved": step_gbs, "peak": hbm,
                              "unit": "GB/s", "frac": step_gbs / hbm},
            "kernels_ms_per_step": {k: round(v, 4) for k, v in sorted(tot.items(), key=lambda x: -x[1])},
            "schedule": "one kernel per pass, CUDA-graph replay",
            "e2e": {"value": e2e, "unit": "zone-updates/s",
                    "h2d_bytes_per_step": (h2d + 8 * len(disks) * args.steps) / args.steps,
                    "d2h_bytes_per_step": (d2h + 8 * len(disks) * args.steps) / args.steps},
            "gpu_launches": launches_per_step * args.steps,
            "fp64_plain": fp64,
            "mixed_form": mixed,
            "clocks": ck,
            "cpu_baseline": cpu,
        }
        line.update(side)
        print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="config4", choices=["config4", "ragged64", "ragged8", "config0"])
    ap.add_argument("--c4-nz", type=int, default=C4_NZ,
                    help="z layers of the config-4 disk (128; fewer for profiling captures)")
    ap.add_argument("--no-config2", action="store_true", help="skip the ragged64 (config 2) leg")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    ap.add_argument("--no-c2p", action="store_true", help="skip the GRMHD cons->prim leg")
    ap.add_argument("--no-config1", action="store_true", help="skip the 3D MHD (config 1) leg")
    ap.add_argument("--no-config3", action="store_true", help="skip the GRMHD torus (config 3) leg")
    ap.add_argument("--c3-nz", type=int, default=96, help="z layers of the config-3 torus (96)")
    ap.add_argument("--only-config3", action="store_true",
                    help="run the config-3 leg alone (no headline line), e.g. for profiling")
    ap.add_argument("--only-c2p", action="store_true",
                    help="run the cons->prim leg alone (no headline line)")
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
    if args.only_c2p:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"c2p": c2p_leg(args, local, torch.cuda.Stream(device=local))}), flush=True)
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)


if __name__ == "__main__":
    main()
