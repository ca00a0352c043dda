"""disco_b200: B200-native Disco RK timestep, Python host mirror.

The product is the C ABI in include/disco_b200.h (kernels + batch API) and
include/disco_host.h (in.par / Makefile_opt.in parsing and grid set-up),
built into disco_b200/libdisco_b200.so.  This module binds it with ctypes and
mirrors the reference's host flow (main.c:31-83):

    disk = Disk.from_files("in.par", "Makefile_opt.in")   # read_par_file, setupGrid,
                                                          # setupDomain, setupCells
    batch = Batch([disk])                                 # device-resident state
    dt = batch.mindt()                                    # getmindt
    batch.timestep(dt)                                    # timestep
    batch.run(100)                                        # 100 x {getmindt; timestep}

There is no CPU fallback: without the built library or a CUDA device every
entry point raises DiscoError.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libdisco_b200.so")
TEMPLATES = os.path.join(HERE, "templates")

OK = 0
PLANET_COLS = 7
STATUS = {0: "ok", 1: "bad argument", 2: "CUDA runtime error", 3: "module combination not built",
          4: "phi wrap loop hit its cap (non-finite piph)", 5: "non-finite or non-positive dt",
          6: "no CUDA device", 7: "call out of order", 8: "device consistency check failed",
          9: "file not written, read or parsed"}
HYDRO = {"euler": 0, "mhd": 1, "grmhd2": 2}
METRIC = {"schw_ks_rpz": 0, "kerr_ks_rpz": 1}
BOUNDARY = {"fixed": 0, "zerograd": 1, "fixed3d": 2, "polar": 3, "outflow3d": 4, "zerograd_omk": 5,
            "accrete3d": 6, "polar3d": 7, "horizon": 8, "horizon3d": 9, "horizon_bin": 10,
            "fixRrefZ": 11, "tube": 12, "surfaceGravBox": 13, "fixed_gap": 14, "flowthrough": 15}
PLANETS = {"none": 0, "sun": 1, "cm2": 2, "binary_soft": 3, "circular": 4, "cm": 5}
INITIAL = {"kepler_noise": 0, "mhd_shear_noise": 1, "host": 2, "gr_torus_noise": 3}
PREC_FP64, PREC_MIXED = 0, 1
SCHED_KERNELS, SCHED_PERSISTENT = 0, 1
GR_DUMP_ROWS = 21                 # DISCO_GR_DUMP_ROWS: cons / dV (9), warm-start prims (9), x (3)


class DiscoError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)} (status {status})")


class Params(C.Structure):
    """Mirror of disco_params (include/disco_b200.h)."""
    _fields_ = [
        ("Num_R", C.c_int), ("Num_Z", C.c_int), ("aspect", C.c_double),
        ("rmin", C.c_double), ("rmax", C.c_double), ("zmin", C.c_double), ("zmax", C.c_double),
        ("phimax", C.c_double),
        ("NoBC_Rmin", C.c_int), ("NoBC_Rmax", C.c_int), ("NoBC_Zmin", C.c_int), ("NoBC_Zmax", C.c_int),
        ("LogZoning", C.c_int), ("R_Periodic", C.c_int), ("Z_Periodic", C.c_int),
        ("LogRadius", C.c_double),
        ("Mesh_Motion", C.c_int), ("Riemann_Solver", C.c_int), ("Timestep", C.c_int),
        ("CFL", C.c_double), ("PLM", C.c_double), ("maxDT", C.c_double),
        ("Density_Floor", C.c_double), ("Pressure_Floor", C.c_double),
        ("Exact_Mesh_Omega", C.c_int), ("Exact_Mesh_Omega_Par", C.c_double),
        ("Energy_Omega", C.c_int), ("Energy_Omega_Par", C.c_double),
        ("RotFrame", C.c_int), ("RotOmega", C.c_double), ("RotD", C.c_double),
        ("Adiabatic_Index", C.c_double), ("viscosity", C.c_double),
        ("visc_flag", C.c_int), ("alpha_flag", C.c_int), ("isothermal_flag", C.c_int),
        ("Cs2_Profile", C.c_int), ("Cs2_Par", C.c_double),
        ("Disk_Mach", C.c_double), ("Mass_Ratio", C.c_double),
        ("grav2D", C.c_int), ("CT", C.c_int), ("initPar0", C.c_int),
        ("initPar", C.c_double * 9), ("metricPar", C.c_double * 5), ("t_min", C.c_double),
        ("include_atmos", C.c_int), ("noiseType", C.c_int), ("noiseAbs", C.c_double),
        ("noiseRel", C.c_double),
    ]


class Modules(C.Structure):
    """Mirror of disco_modules."""
    _fields_ = [("hydro", C.c_int), ("boundary", C.c_int), ("planets", C.c_int),
                ("initial", C.c_int), ("analysis", C.c_int),
                ("num_c", C.c_int), ("num_n", C.c_int), ("ct_mode", C.c_int), ("metric", C.c_int)]


_lib = None

_I = C.c_int
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_IP = C.POINTER(C.c_int)


def library():
    """Load libdisco_b200.so (raises DiscoError if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIBPATH):
        raise DiscoError(6, "libdisco_b200.so not built (run disco_b200.build.build())")
    lib = C.CDLL(LIBPATH)
    sig = {
        "disco_abi_version": (_I, []),
        "disco_strerror": (C.c_char_p, [_I]),
        "disco_batch_create": (_I, [_I, C.POINTER(Modules), _I, _I, C.POINTER(Params), _IP, _IP, _IP,
                                    _IP, _D, _D, C.POINTER(_P)]),
        "disco_batch_destroy": (None, [_P]),
        "disco_batch_sizes": (_I, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _IP]),
        "disco_batch_set_cells": (_I, [_P, _D, _D, _D, _D, _D, _IP, _D]),
        "disco_batch_get_cells": (_I, [_P, _D, _D, _D, _D, _D, _D]),
        "disco_batch_setup_cells": (_I, [_P]),
        "disco_batch_mindt": (_I, [_P, _D]),
        "disco_batch_timestep": (_I, [_P, _D]),
        "disco_batch_run": (_I, [_P, _I]),
        "disco_batch_report": (_I, [_P, _I, _D]),
        "disco_batch_time": (_I, [_P, _I, _D, _IP]),
        "disco_batch_get_faces": (_I, [_P, _I, _I, _IP, _IP, _IP, _IP, _IP, _D]),
        "disco_batch_get_diagnostics": (_I, [_P, _I, _D, _IP, _D]),
        "disco_batch_last_error": (_I, [_P]),
        "disco_batch_kernel_times": (_I, [_P, C.POINTER(C.c_float), C.POINTER(C.c_char_p), _I, _IP]),
        "disco_batch_set_stream": (_I, [_P, _P]),
        "disco_batch_set_schedule": (_I, [_P, _I]),
        "disco_batch_set_gr_dump": (_I, [_P, _P]),
        "disco_batch_get_schedule": (_I, [_P, _IP]),
        "disco_batch_debug_get": (_I, [_P, _I, _D]),
        "disco_read_par": (_I, [C.c_char_p, C.POINTER(Params), _IP]),
        "disco_read_opt": (_I, [C.c_char_p, C.POINTER(Modules)]),
        "disco_setup_grid": (_I, [C.POINTER(Params), _IP, _IP, _IP, _IP, _D, _D]),
        "disco_setup_phi": (_I, [C.POINTER(Params), _I, _I, _IP, _IP, _D, _D, _IP]),
        "disco_sizeof": (_I, [_I]),
        "disco_batch_set_time": (_I, [_P, _I, C.c_double]),
        "disco_batch_set_noise": (_I, [_P, _D]),
        "disco_setup_noise": (_I, [C.POINTER(Params), _I, _I, _IP, _IP, _D]),
        "disco_batch_get_planets": (_I, [_P, _I, _D, _I, _IP]),
        "disco_batch_set_planets": (_I, [_P, _I, _D, _I]),
        "disco_batch_restart_cells": (_I, [_P, _D, _D, _D]),
        "disco_batch_write_checkpoint": (_I, [_P, _I, C.c_char_p]),
        "disco_batch_write_ascii": (_I, [_P, _I, C.c_char_p]),
        "disco_batch_restart": (_I, [_P, C.POINTER(C.c_char_p)]),
        "disco_npz_create": (_I, [C.c_char_p, C.POINTER(_P)]),
        "disco_npz_put": (_I, [_P, C.c_char_p, C.c_char_p, _I, C.POINTER(C.c_int64), _P]),
        "disco_npz_begin": (_I, [_P, C.c_char_p, C.c_char_p, _I, C.POINTER(C.c_int64)]),
        "disco_npz_append": (_I, [_P, _P, C.c_size_t]),
        "disco_npz_end": (_I, [_P]),
        "disco_npz_open": (_I, [C.c_char_p, C.POINTER(_P)]),
        "disco_npz_info": (_I, [_P, C.c_char_p, C.c_char_p, _IP, C.POINTER(C.c_int64)]),
        "disco_npz_read": (_I, [_P, C.c_char_p, C.c_uint64, _P, C.c_size_t]),
        "disco_npz_close": (_I, [_P]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(status, where):
    if status != OK:
        raise DiscoError(status, where)


def dptr(a):
    return a.ctypes.data_as(_D) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(_IP) if a is not None else None


def read_par(path):
    """read_par_file (readpar.c:44-188) -> Params."""
    p = Params()
    miss = C.c_int(0)
    _check(library().disco_read_par(path.encode(), C.byref(p), C.byref(miss)), "disco_read_par")
    return p


def read_opt(path):
    """Makefile_opt.in module selection -> Modules."""
    m = Modules()
    _check(library().disco_read_opt(path.encode(), C.byref(m)), "disco_read_opt")
    return m


class Disk:
    """One disk's grid and initial phi layout, built as setupGrid/setupDomain do."""

    def __init__(self, params, modules):
        lib = library()
        self.params, self.modules = params, modules
        Nr, Nz = C.c_int(), C.c_int()
        Ng = np.zeros(4, np.int32)
        _check(lib.disco_setup_grid(C.byref(params), C.byref(Nr), C.byref(Nz), iptr(Ng),
                                    None, None, None), "disco_setup_grid")
        self.Nr, self.Nz, self.Ng = Nr.value, Nz.value, Ng
        self.Np = np.zeros(self.Nr * self.Nz, np.int32)
        self.r_jph = np.zeros(self.Nr + 1)
        self.z_kph = np.zeros(self.Nz + 1)
        _check(lib.disco_setup_grid(C.byref(params), C.byref(Nr), C.byref(Nz), iptr(Ng),
                                    iptr(self.Np), dptr(self.r_jph), dptr(self.z_kph)),
               "disco_setup_grid")
        self.ncell = int(self.Np.sum())
        self.piph = np.zeros(self.ncell)
        self.dphi = np.zeros(self.ncell)
        self.real = np.zeros(self.ncell, np.int32)
        _check(lib.disco_setup_phi(C.byref(params), self.Nr, self.Nz, iptr(self.Ng), iptr(self.Np),
                                   dptr(self.piph), dptr(self.dphi), iptr(self.real)),
               "disco_setup_phi")
        # addNoise's draws (Noise_Type 1-3), from the same rand() stream
        self.noise = None
        if params.noiseType in (1, 2, 3):
            self.noise = np.zeros((self.ncell, 4))
            _check(lib.disco_setup_noise(C.byref(params), self.Nr, self.Nz, iptr(self.Ng),
                                         iptr(self.Np), dptr(self.noise)), "disco_setup_noise")

    @classmethod
    def from_files(cls, par_path, opt_path):
        return cls(read_par(par_path), read_opt(opt_path))

    @property
    def q(self):
        return self.modules.num_c + self.modules.num_n

    @property
    def nreal(self):
        return int(self.real.sum())


class Batch:
    """Device-resident batch of disks (disco_batch_*)."""

    def __init__(self, disks, device=0, precision=PREC_FP64, setup=True):
        lib = library()
        self.disks = list(disks)
        n = len(self.disks)
        m = self.disks[0].modules
        key = lambda mm: tuple(getattr(mm, f) for f, _ in Modules._fields_)
        if any(key(d.modules) != key(m) for d in self.disks):
            # one Makefile_opt.in module selection per batch, as one Disco build has
            raise DiscoError(1, "Batch: all disks must share one module selection")
        par = (Params * n)(*[d.params for d in self.disks])
        Nr = np.array([d.Nr for d in self.disks], np.int32)
        Nz = np.array([d.Nz for d in self.disks], np.int32)
        Ng = np.concatenate([d.Ng for d in self.disks]).astype(np.int32)
        Np = np.concatenate([d.Np for d in self.disks]).astype(np.int32)
        rj = np.concatenate([d.r_jph for d in self.disks])
        zk = np.concatenate([d.z_kph for d in self.disks])
        h = C.c_void_p()
        _check(lib.disco_batch_create(device, C.byref(m), precision, n, par, iptr(Nr), iptr(Nz),
                                      iptr(Ng), iptr(Np), dptr(rj), dptr(zk), C.byref(h)),
               "disco_batch_create")
        self.h = h
        self.q = self.disks[0].q
        self.offsets = np.concatenate([[0], np.cumsum([d.ncell for d in self.disks])]).astype(np.int64)
        self.ncell = int(self.offsets[-1])
        if setup:
            piph = np.concatenate([d.piph for d in self.disks])
            dphi = np.concatenate([d.dphi for d in self.disks])
            real = np.concatenate([d.real for d in self.disks]).astype(np.int32)
            _check(lib.disco_batch_set_cells(self.h, None, None, dptr(piph), dptr(dphi), None,
                                             iptr(real), None), "disco_batch_set_cells")
            self._upload_noise()
            _check(lib.disco_batch_setup_cells(self.h), "disco_batch_setup_cells")

    def close(self):
        if getattr(self, "h", None):
            library().disco_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def ct(self):
        """Constrained transport on (in.par Constrained_Transport)."""
        return bool(self.disks[0].params.CT)

    @property
    def num_faces(self):
        """Face-flux slots per cell under CT (the reference's NUM_FACES)."""
        return 5 if self.disks[0].modules.ct_mode == 2 else 3

    def set_cells(self, prim, cons, piph, dphi, wiph=None, real=None, Phi=None):
        """Upload a state; Phi (ncell x num_faces face fluxes) is the
        constrained-transport state and is taken only when CT is on (zeros when
        omitted)."""
        prim = None if prim is None else np.ascontiguousarray(prim, np.float64)
        cons = None if cons is None else np.ascontiguousarray(cons, np.float64)
        piph = np.ascontiguousarray(piph, np.float64)
        dphi = np.ascontiguousarray(dphi, np.float64)
        wiph = None if wiph is None else np.ascontiguousarray(wiph, np.float64)
        real = None if real is None else np.ascontiguousarray(real, np.int32)
        Phi = None if Phi is None else np.ascontiguousarray(Phi, np.float64)
        if Phi is not None and Phi.shape != (self.ncell, self.num_faces):
            raise ValueError("Phi must be ncell x %d" % self.num_faces)
        _check(library().disco_batch_set_cells(self.h, dptr(prim), dptr(cons), dptr(piph),
                                               dptr(dphi), dptr(wiph), iptr(real), dptr(Phi)),
               "disco_batch_set_cells")

    def get_cells(self, out=None):
        """Download the state; `out` may supply the arrays (e.g. pinned host
        memory) as a dict with the keys this returns."""
        n, q = self.ncell, self.q
        o = out or {}
        prim = o.get("prim"); cons = o.get("cons")
        piph = o.get("piph"); dphi = o.get("dphi"); wiph = o.get("wiph")
        prim = np.zeros((n, q)) if prim is None else prim
        cons = np.zeros((n, q)) if cons is None else cons
        piph = np.zeros(n) if piph is None else piph
        dphi = np.zeros(n) if dphi is None else dphi
        wiph = np.zeros(n) if wiph is None else wiph
        for a, shape in ((prim, (n, q)), (cons, (n, q)), (piph, (n,)), (dphi, (n,)), (wiph, (n,))):
            if a.shape != shape or a.dtype != np.float64 or not a.flags.c_contiguous:
                raise ValueError("get_cells: output arrays must be C-contiguous float64 of the state's shape")
        Phi = (o.get("Phi") if o.get("Phi") is not None else np.zeros((n, self.num_faces))) \
            if self.ct else None
        _check(library().disco_batch_get_cells(self.h, dptr(prim), dptr(cons), dptr(piph),
                                               dptr(dphi), dptr(wiph), dptr(Phi)),
               "disco_batch_get_cells")
        out = dict(prim=prim, cons=cons, piph=piph, dphi=dphi, wiph=wiph)
        if Phi is not None:
            out["Phi"] = Phi
        return out

    def mindt(self):
        dt = np.zeros(len(self.disks))
        _check(library().disco_batch_mindt(self.h, dptr(dt)), "disco_batch_mindt")
        return dt

    def timestep(self, dt=None):
        a = None if dt is None else np.ascontiguousarray(np.broadcast_to(dt, len(self.disks)), np.float64)
        _check(library().disco_batch_timestep(self.h, dptr(a)), "disco_batch_timestep")

    def run(self, nsteps):
        _check(library().disco_batch_run(self.h, int(nsteps)), "disco_batch_run")

    def set_stream(self, stream_handle):
        """Launch on an external cudaStream_t (an int handle; 0/None = own stream)."""
        _check(library().disco_batch_set_stream(self.h, C.c_void_p(stream_handle or None)),
               "disco_batch_set_stream")

    @property
    def schedule(self):
        """SCHED_PERSISTENT (the step as one launch) or SCHED_KERNELS."""
        x = C.c_int()
        _check(library().disco_batch_get_schedule(self.h, C.byref(x)), "disco_batch_get_schedule")
        return x.value

    @schedule.setter
    def schedule(self, sched):
        _check(library().disco_batch_set_schedule(self.h, int(sched)), "disco_batch_set_schedule")

    def set_gr_dump(self, buf):
        """GRMHD batches: each cons->prim of the following steps writes its
        inputs (cons / dV, warm-start prims, x: GR_DUMP_ROWS x ncell float64,
        a CUDA tensor on the batch's device, e.g. torch.zeros) for the real
        cells into `buf`; None stops it.  The buffer must outlive its use."""
        if buf is None:
            ptr = None
        else:
            if tuple(buf.shape) != (GR_DUMP_ROWS, self.ncell) or not buf.is_contiguous() \
                    or str(buf.dtype) != "torch.float64" or not buf.is_cuda:
                raise ValueError("dump buffer must be a contiguous float64 CUDA tensor of shape (%d, %d)"
                                 % (GR_DUMP_ROWS, self.ncell))
            ptr = C.c_void_p(buf.data_ptr())
        _check(library().disco_batch_set_gr_dump(self.h, ptr), "disco_batch_set_gr_dump")
        self._gr_dump = buf

    def kernel_times(self, cap=64):
        """One instrumented step: [(kernel name, device ms), ...] in launch order."""
        ms = (C.c_float * cap)()
        names = (C.c_char_p * cap)()
        n = C.c_int()
        _check(library().disco_batch_kernel_times(self.h, ms, names, cap, C.byref(n)),
               "disco_batch_kernel_times")
        return [(names[i].decode(), float(ms[i])) for i in range(n.value)]

    def debug_array(self, which):
        """Internal per-cell array after the last step: 0 gradp, 1 gradr, 2 RKcons."""
        out = np.zeros((self.ncell, self.q))
        _check(library().disco_batch_debug_get(self.h, which, dptr(out)), "disco_batch_debug_get")
        return out

    def last_error(self):
        return library().disco_batch_last_error(self.h)

    def sync(self):
        _check(self.last_error(), "device")

    def time(self, disk=0):
        t = C.c_double(); cnt = C.c_int()
        _check(library().disco_batch_time(self.h, disk, C.byref(t), C.byref(cnt)), "disco_batch_time")
        return t.value, cnt.value

    def faces(self, disk=0, dim=1, geom=False):
        d = self.disks[disk]
        ntr = (d.Nr - 1) * d.Nz if dim == 1 else (d.Nz - 1) * d.Nr
        nf_max = int(sum(d.Np)) * 2 + 16
        fI = np.zeros(ntr + 1, np.int32)
        iL = np.zeros(nf_max, np.int32); iR = np.zeros(nf_max, np.int32)
        LR = np.zeros(nf_max, np.int32)
        g = np.zeros((nf_max, 8)) if geom else None
        nf = C.c_int()
        _check(library().disco_batch_get_faces(self.h, disk, dim, C.byref(nf), iptr(fI), iptr(iL),
                                               iptr(iR), iptr(LR), dptr(g)), "disco_batch_get_faces")
        n = nf.value
        out = dict(fIndex=fI, iL=iL[:n], iR=iR[:n], LRtype=LR[:n])
        if geom:
            out["geom"] = g[:n]
        return out

    REPORT_FIELDS = ("t", "Torque", "Power", "Fr", "rho_min", "rhoavg_min", "PsiR", "PsiI", "Mass",
                     "Mdot", "S_R", "L1_rho", "L1_isen", "L1_B", "Br2", "aM", "bM")

    def report(self, disk=0):
        """report() on the device: the 17 numbers of the disk's report.dat line
        (names in REPORT_FIELDS)."""
        out = np.zeros(17)
        _check(library().disco_batch_report(self.h, disk, dptr(out)), "disco_batch_report")
        return out

    def _upload_noise(self):
        """addNoise's draws of every disk with Noise_Type 1-3 (zeros for the others)."""
        if all(d.noise is None for d in self.disks):
            return
        nz = np.concatenate([d.noise if d.noise is not None else np.zeros((d.ncell, 4))
                             for d in self.disks])
        _check(library().disco_batch_set_noise(self.h, dptr(np.ascontiguousarray(nz))),
               "disco_batch_set_noise")

    def set_time(self, t, disk=0):
        """Set the disk's simulation time (a restart's T)."""
        _check(library().disco_batch_set_time(self.h, disk, float(t)), "disco_batch_set_time")

    def planets(self, disk=0):
        """The disk's planets: rows of M, vr, omega, r, phi, eps, type (the
        checkpoint's Data/Planets columns)."""
        n = C.c_int()
        lib = library()
        _check(lib.disco_batch_get_planets(self.h, disk, None, 0, C.byref(n)), "disco_batch_get_planets")
        rows = np.zeros((n.value, PLANET_COLS))
        _check(lib.disco_batch_get_planets(self.h, disk, dptr(rows), n.value, C.byref(n)),
               "disco_batch_get_planets")
        return rows

    def set_planets(self, rows, disk=0):
        rows = np.ascontiguousarray(rows, np.float64)
        if rows.ndim != 2 or rows.shape[1] != PLANET_COLS:
            raise ValueError("planet rows must be npl x %d" % PLANET_COLS)
        _check(library().disco_batch_set_planets(self.h, disk, dptr(rows), rows.shape[0]),
               "disco_batch_set_planets")

    def restart_cells(self, prim, piph, Phi=None):
        """setupCells after a restart from prim / Phi / piph of every cell
        (disco_batch_restart_cells)."""
        prim = np.ascontiguousarray(prim, np.float64)
        piph = np.ascontiguousarray(piph, np.float64)
        Phi = None if Phi is None else np.ascontiguousarray(Phi, np.float64)
        if prim.shape != (self.ncell, self.q) or piph.shape != (self.ncell,):
            raise ValueError("restart_cells: prim must be ncell x q, piph ncell")
        self._upload_noise()
        _check(library().disco_batch_restart_cells(self.h, dptr(prim), dptr(Phi), dptr(piph)),
               "disco_batch_restart_cells")

    def write_checkpoint(self, filestart, disk=0):
        """Write the disk's checkpoint, <filestart>.npz (the datasets of the
        reference's HDF5 checkpoint under their paths); returns the path."""
        _check(library().disco_batch_write_checkpoint(self.h, disk, os.fsencode(filestart)),
               "disco_batch_write_checkpoint")
        return os.fsdecode(filestart) + ".npz"

    def write_ascii(self, filestart, disk=0):
        """Write the ascii output module's <filestart>.dat; returns the path."""
        _check(library().disco_batch_write_ascii(self.h, disk, os.fsencode(filestart)),
               "disco_batch_write_ascii")
        return os.fsdecode(filestart) + ".dat"

    def restart(self, paths):
        """Restart every disk from its checkpoint file (one path per disk, or
        one path for a one-disk batch)."""
        if isinstance(paths, (str, bytes, os.PathLike)):
            paths = [paths]
        if len(paths) != len(self.disks):
            raise ValueError("restart: one checkpoint per disk")
        arr = (C.c_char_p * len(paths))(*[os.fsencode(p) for p in paths])
        _check(library().disco_batch_restart(self.h, arr), "disco_batch_restart")

    def diagnostics(self, disk=0):
        d = self.disks[disk]
        Qrz = np.zeros(d.Nr * d.Nz * 18)
        nq = C.c_int(); tav = C.c_double()
        _check(library().disco_batch_get_diagnostics(self.h, disk, dptr(Qrz), C.byref(nq),
                                                     C.byref(tav)), "disco_batch_get_diagnostics")
        return Qrz[: d.Nr * d.Nz * nq.value], tav.value


def template_paths(name):
    """(in.par, Makefile_opt.in) of a bundled configuration template."""
    return (os.path.join(TEMPLATES, name + ".par"), os.path.join(TEMPLATES, name + ".in"))
