/*
 * disco_b200 -- C ABI of the B200-native Disco RK timestep.
 *
 * This is the drop-in boundary for the serial (USE_MPI=0) Disco hot path.
 * In the reference, main.c calls two functions per step:
 *
 *     double getmindt( struct domain * );          misc.c:39-84   (main.c:12,72)
 *     void   timestep( struct domain * , double ); timestep.c:7-45 (main.c:7,81)
 *
 * and timestep() calls onestep() twice (onestep.c:84-229).  Physics modules
 * are link-time selected C files (hydro.h, geometry.h, boundary.h, omega.h,
 * Planets/<name>.c, Initial/<name>.c) chosen in Makefile_opt.in; run-time parameters
 * come from in.par (readpar.c:44-188).
 *
 * Here the whole state lives on one GPU between calls, laid out as ragged
 * structure-of-arrays (cells in annulus order jk = j + Nr*k, i = 0..Np-1).
 * The functions below take plain pointers and sizes; no struct of the
 * reference crosses the boundary, so a C, cgo, ctypes or JNI caller can bind
 * them directly.  Every function returns an int status: DISCO_OK (0) or one
 * of the DISCO_ERR_* codes; disco_strerror() names it.  Device-side failures
 * that the reference would hang or NaN on (unbounded phi-wrap loops on a
 * non-finite piph, misc.c:22-23 / cylindrical.c:12-13) set an error word
 * that the next call reports as DISCO_ERR_PHI_WRAP or DISCO_ERR_NONFINITE.
 *
 * A "batch" holds one or more independent disks (each its own in.par grid,
 * parameters and dt) advanced together in the same kernels.  A single-disk
 * batch is exactly the reference's serial domain.
 */
#ifndef DISCO_B200_H
#define DISCO_B200_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DISCO_ABI_VERSION 3

enum disco_status {
   DISCO_OK = 0,
   DISCO_ERR_ARG = 1,          /* bad argument (null pointer, size, unknown module) */
   DISCO_ERR_CUDA = 2,         /* a CUDA runtime call failed */
   DISCO_ERR_UNSUPPORTED = 3,  /* module combination not built */
   DISCO_ERR_PHI_WRAP = 4,     /* phi wrap loop hit its iteration cap (non-finite piph) */
   DISCO_ERR_NONFINITE = 5,    /* non-finite dt or state detected */
   DISCO_ERR_NO_DEVICE = 6,    /* no CUDA device / library built without one */
   DISCO_ERR_STATE = 7,        /* call out of order (e.g. step before set_cells) */
   DISCO_ERR_INTERNAL = 8,     /* a device-side consistency check failed */
   DISCO_ERR_IO = 9            /* a file could not be written, read or parsed */
};

/* Module choices, one per Makefile_opt.in line (Makefile:11-26).  The names
 * match the reference's module file names. */
enum disco_hydro    { DISCO_HYDRO_EULER = 0, DISCO_HYDRO_MHD = 1, DISCO_HYDRO_GRMHD = 2 };
/* METRIC of a grmhd2 build: Hydro/Metric/schw_ks_rpz.c, or the new Kerr-Schild
 * module kerr_ks_rpz (spin Metric_Par3; the reference has no Kerr metric) */
enum disco_metric   { DISCO_METRIC_SCHW_KS_RPZ = 0, DISCO_METRIC_KERR_KS_RPZ = 1 };
enum disco_boundary { DISCO_BC_FIXED = 0, DISCO_BC_ZEROGRAD = 1, DISCO_BC_FIXED3D = 2,
                      DISCO_BC_POLAR = 3, DISCO_BC_OUTFLOW3D = 4, DISCO_BC_ZEROGRAD_OMK = 5,
                      DISCO_BC_ACCRETE3D = 6, DISCO_BC_POLAR3D = 7, DISCO_BC_HORIZON = 8,
                      DISCO_BC_HORIZON3D = 9, DISCO_BC_HORIZON_BIN = 10, DISCO_BC_FIXRREFZ = 11,
                      DISCO_BC_TUBE = 12, DISCO_BC_SURFACEGRAVBOX = 13, DISCO_BC_FIXED_GAP = 14,
                      DISCO_BC_FLOWTHROUGH = 15 };
enum disco_planets  { DISCO_PLANETS_NONE = 0, DISCO_PLANETS_SUN = 1, DISCO_PLANETS_CM2 = 2,
                      DISCO_PLANETS_BINARY_SOFT = 3, DISCO_PLANETS_CIRCULAR = 4,
                      DISCO_PLANETS_CM = 5 };
/* DISCO_IC_HOST: the Initial module is the host's own (a drop-in evaluating
 * any reference IC in setupCells): the state must come from set_cells, and
 * only boundaries that never re-evaluate initial() during the steps
 * (zerograd, outflow3d) are accepted. */
enum disco_initial  { DISCO_IC_KEPLER_NOISE = 0, DISCO_IC_MHD_SHEAR_NOISE = 1, DISCO_IC_HOST = 2,
                      DISCO_IC_GR_TORUS_NOISE = 3 };
enum disco_analysis { DISCO_DIAG_NONE = 0, DISCO_DIAG_DISK2D = 1, DISCO_DIAG_EULER = 2,
                      DISCO_DIAG_MHDMRI = 3 };
enum disco_precision{ DISCO_PREC_FP64 = 0, DISCO_PREC_MIXED = 1 };
/* How a batch's step is launched (disco_batch_set_schedule): one kernel per
 * pass of onestep(), or the whole RK2 step as one persistent launch whose
 * blocks wait only for the blocks they read from.  Both run the same block
 * bodies, so their results are identical bit for bit. */
enum disco_schedule { DISCO_SCHED_KERNELS = 0, DISCO_SCHED_PERSISTENT = 1 };

/* Compile-time module selection (Makefile_opt.in).  num_c/num_n/ct_mode are
 * the reference's NUM_C, NUM_N and CT_MODE (paul.h:26-49). */
typedef struct disco_modules {
   int hydro, boundary, planets, initial, analysis;
   int num_c, num_n, ct_mode;
   int metric;                 /* enum disco_metric, for HYDRO = grmhd2 */
} disco_modules;

/* Run-time parameters: the subset of struct param_list (paul.h:51-127) that
 * the step reads, with read_par_file's 2*pi scalings already applied
 * (readpar.c:162-172).  Field names follow param_list. */
typedef struct disco_params {
   int    Num_R, Num_Z;
   double aspect;
   double rmin, rmax, zmin, zmax, phimax;
   int    NoBC_Rmin, NoBC_Rmax, NoBC_Zmin, NoBC_Zmax;
   int    LogZoning, R_Periodic, Z_Periodic;
   double LogRadius;
   int    Mesh_Motion, Riemann_Solver, Timestep;
   double CFL, PLM, maxDT;
   double Density_Floor, Pressure_Floor;
   int    Exact_Mesh_Omega;
   double Exact_Mesh_Omega_Par;
   int    Energy_Omega;
   double Energy_Omega_Par;
   int    RotFrame;
   double RotOmega, RotD;
   double Adiabatic_Index;
   double viscosity;
   int    visc_flag, alpha_flag;
   int    isothermal_flag;
   int    Cs2_Profile;
   double Cs2_Par;
   double Disk_Mach;
   double Mass_Ratio;
   int    grav2D;
   int    CT;
   int    initPar0;
   double initPar[9];          /* initPar[1..8] = Init_Par1..8; [0] unused */
   double metricPar[5];        /* metricPar[1..4] = Metric_Par1..4 */
   double t_min;
   /* set-up options of setupCells (domain.c:144-205): Include_Atmos
    * (adjust_gas, planet.c:76-96) and Noise_Type / Noise_Abs / Noise_Rel
    * (addNoise, noise.c:15-50) */
   int    include_atmos;
   int    noiseType;
   double noiseAbs, noiseRel;
} disco_params;

typedef struct disco_batch disco_batch;   /* opaque device-resident batch */

/* Version of this ABI (DISCO_ABI_VERSION). */
int disco_abi_version(void);
const char *disco_strerror(int status);

/*
 * Create a batch of `ndisk` independent disks on CUDA device `device`.
 *
 * Per disk d: params[d], and its grid exactly as setupGrid() builds it
 * (gridsetup.c:15-142): Nr[d], Nz[d] (annuli incl. ghosts), Ng[4*d+0..3] =
 * NgRa, NgRb, NgZa, NgZb, and concatenated arrays
 *   Np      : Nr*Nz ints per disk            (cells per annulus)
 *   r_jph   : Nr+1 doubles per disk, element 0 is the reference's r_jph[-1]
 *   z_kph   : Nz+1 doubles per disk, element 0 is z_kph[-1]
 * All disks share one module selection `mods` and one precision.
 * Replaces: setupGrid + setupDomain allocation (gridsetup.c:90-95,
 * domain.c:34-38,112-113).
 */
int disco_batch_create(int device, const disco_modules *mods, int precision,
                       int ndisk, const disco_params *params,
                       const int *Nr, const int *Nz, const int *Ng,
                       const int *Np, const double *r_jph, const double *z_kph,
                       disco_batch **out);
void disco_batch_destroy(disco_batch *b);

/* Total cells (incl. ghosts) and real cells of the batch; Q = num_c+num_n. */
int disco_batch_sizes(const disco_batch *b, int64_t *ncell, int64_t *nreal, int *q);

/*
 * Upload cell state from host memory.  All arrays hold ncell entries in
 * annulus order (disk-major); prim/cons are cell-major, Q doubles per cell
 * (the reference's struct cell prim[NUM_Q] / cons[NUM_Q], paul.h:185-186).
 * real[] is the reference's cell->real flag.  cons may be NULL (then cons is
 * rebuilt from prim with prim2cons on the device, as setupCells does,
 * domain.c:205).  Phi is the constrained-transport state (in.par
 * Constrained_Transport 1; CT_MODE 1 for 2D disks, CT_MODE 2 in 2D or 3D):
 * NUM_FACES doubles per cell (3 or 5), the reference's cell->Phi[NUM_FACES]
 * (paul.h:198) -- Phi[0] the magnetic flux through the phi face at piph,
 * Phi[1] / Phi[2] that through the r face the cell owns in the track inside
 * / outside it, Phi[3] / Phi[4] the z face it owns below / above it
 * (bfields.c:734-758).  It is ignored when CT is off and may be NULL (zeros)
 * when CT is on.
 */
int disco_batch_set_cells(disco_batch *b, const double *prim, const double *cons,
                          const double *piph, const double *dphi, const double *wiph,
                          const int *real, const double *Phi);

/* Download cell state (same layout; Phi only when CT is on); any pointer
 * may be NULL to skip it. */
int disco_batch_get_cells(disco_batch *b, double *prim, double *cons,
                          double *piph, double *dphi, double *wiph, double *Phi);

/*
 * Device set-up of a fresh batch after set_cells with prim unset: evaluates
 * the Initial module on every real cell, prim2cons, cons2prim, set_wcell
 * (domain.c:283-386) and the boundary (main.c:53-62).  piph/dphi must have
 * been uploaded (the reference draws them from rand(), domain.c:206-233).
 */
int disco_batch_setup_cells(disco_batch *b);

/*
 * The random numbers of addNoise (noise.c:15-50) for in.par Noise_Type 1-3:
 * 4 doubles per cell (annulus order, disk-major), made on the host by
 * disco_setup_noise (include/disco_host.h) from glibc's rand() stream in
 * the reference's cell order.  setupCells applies them after the Initial
 * module (and adjust_gas), and again on restart, so set them before
 * disco_batch_setup_cells / _restart_cells of a batch with noise (those
 * return DISCO_ERR_STATE otherwise); disco_batch_restart makes them itself.
 * NULL clears them.
 */
int disco_batch_set_noise(disco_batch *b, const double *noise);

/* getmindt (misc.c:39-84) for every disk: dt[d] = CFL * min over real cells. */
int disco_batch_mindt(disco_batch *b, double *dt);

/*
 * One full step of every disk: timestep() (timestep.c:7-45) with the given
 * per-disk dt (NULL = use the dt that the last mindt/step left on the
 * device, i.e. getmindt of the current state, with no host round trip).
 */
int disco_batch_timestep(disco_batch *b, const double *dt);

/*
 * nsteps repetitions of { dt = getmindt; timestep(dt) } (main.c:69-83
 * without output), all on the device, replayed from a CUDA graph.
 */
int disco_batch_run(disco_batch *b, int nsteps);

/* Simulation time and step count of disk d (theDomain->t, count_steps). */
int disco_batch_time(const disco_batch *b, int disk, double *t, int *count_steps);

/* Set disk d's simulation time (theDomain->t; restart sets it from the
 * checkpoint, h5in.c:159). */
int disco_batch_set_time(disco_batch *b, int disk, double t);

/*
 * Planets of disk d as rows of DISCO_PLANET_COLS doubles -- M, vr, omega, r,
 * phi, eps, type -- the columns of the checkpoint's Data/Planets
 * (h5out.c:444-455) and of restart (h5in.c:305-317).  get: *npl receives the
 * module's planet count (theDomain->Npl); rows (may be NULL) needs cap >= it.
 * set: npl must equal that count; type must be 0 (PLPOINTMASS, the only
 * planet force built), else DISCO_ERR_UNSUPPORTED.  Set after a restart, or
 * by a drop-in whose host domain has moved the planets.
 */
#define DISCO_PLANET_COLS 7
int disco_batch_get_planets(disco_batch *b, int disk, double *rows, int cap, int *npl);
int disco_batch_set_planets(disco_batch *b, int disk, const double *rows, int npl);

/*
 * Restart set-up (setupCells with restart_flag set, domain.c:139-240, after
 * restart()'s Doub2Cell, h5in.c:72-77): uploads, for every cell of the batch
 * in annulus order, prim (NUM_Q per cell), Phi (NUM_FACES per cell; required
 * when constrained transport is on, ignored otherwise) and piph, then on the
 * device: dphi by calc_dp, wiph = 0, prim2cons and cons2prim on real cells,
 * ghosts' boundary values (main.c:53-62), the mesh velocities, and getmindt.
 * Diagnostics and step counts restart from zero (h5in.c:329-333).  Time and
 * planets are set separately (disco_batch_set_time / _set_planets).
 */
int disco_batch_restart_cells(disco_batch *b, const double *prim, const double *Phi,
                              const double *piph);

/*
 * Checkpoint of disk d (Output/h5out.c:349-598, serial): the file
 * "<filestart>.npz" (the container of disco_host.h: disco_npz_*) holds the
 * reference's datasets under their HDF5 paths --
 *   Grid/T [1], Grid/r_jph [Nr+1], Grid/z_kph [Nz+1] (ghost edges included),
 *   Grid/Index, Grid/Np, Grid/Id_phi0 [Nz][Nr] (int32),
 *   Data/Cells [ncell][NUM_Q+NUM_FACES+1] (prim, Phi, piph per cell, annulus
 *   order), Data/Planets [Npl][7], Data/Diagnostics [Nz][Nr][Ntools],
 *   Pars/<in.par key> [1], Opts/<module> [1]
 * -- and, as output() does, averages the diagnostics over their window
 * (avg_diagnostics) and then zeroes them (zero_diagnostics).  NUM_FACES is
 * that of CT_MODE (0, 3 or 5), with zero face fluxes when constrained
 * transport is off.  The rows are packed on the device and streamed to the
 * file through a pinned buffer.
 */
int disco_batch_write_checkpoint(disco_batch *b, int disk, const char *filestart);

/*
 * The ascii output module (Output/ascii.c:7-77) for disk d: "<filestart>.dat"
 * with one line per cell -- r phi z dr dphi dz prim[NUM_Q], "%e " each --
 * annuli j outer, layers k inner (the ghost layers left out when
 * Z_Periodic), the same text the reference writes for the same state.
 */
int disco_batch_write_ascii(disco_batch *b, int disk, const char *filestart);

/*
 * Restart every disk of the batch from its checkpoint file (paths[d], as
 * written by disco_batch_write_checkpoint): the reads of restart()
 * (h5in.c:100-354: T, Planets, Cells by Index/Np) and the set-up of
 * disco_batch_restart_cells.  The file's grid (Np, r_jph, z_kph) must be the
 * disk's -- the reference rebuilds its grid from the file, this batch was
 * built for one -- and its column count NUM_Q+NUM_FACES+1; otherwise
 * DISCO_ERR_ARG.  A file that cannot be read gives DISCO_ERR_IO.
 */
int disco_batch_restart(disco_batch *b, const char *const *paths);

/*
 * report() (report.c:7-202) on the device, without copying the state: the
 * 17 numbers of the disk's report.dat line, in the reference's order --
 * t, Torque, Power, Fr, rho_min, rhoavg_min, PsiR, PsiI, Mass, Mdot, S_R,
 * L1_rho, L1_isen, L1_B, Br2, aM, bM (report.c:189-193).  The sums run as
 * block trees, so they agree with the reference's serial loop to rounding.
 */
int disco_batch_report(disco_batch *b, int disk, double *out);

/*
 * Face list of disk `disk` for dim 1 (r) or 2 (z), built from the current
 * state exactly as setup_faces/buildfaces build it (misc.c:512-532,
 * faces_alt.c:36-179).  fIndex has N_ftracks+1 entries (the reference's
 * fIndex_r / fIndex_z); iL/iR are cell indices within the disk (annulus
 * order); LRtype as struct face.  Any output pointer may be NULL; *nfaces
 * receives the count.  geom (8 doubles per face: dxL dxR cm0 cm1 cm2 dphi dl
 * dA) may be NULL.
 */
int disco_batch_get_faces(disco_batch *b, int disk, int dim, int *nfaces,
                          int *fIndex, int *iL, int *iR, int *LRtype, double *geom);

/* Time-averaged diagnostics Qrz of disk d (analysis.c:52-107): Nr*Nz*nq. */
int disco_batch_get_diagnostics(disco_batch *b, int disk, double *Qrz, int *nq, double *t_avg);

/* Device error word accumulated since the last call (DISCO_OK if none). */
int disco_batch_last_error(disco_batch *b);

/*
 * Diagnostic read of an internal per-cell array left by the last step, cell-
 * major Q doubles per cell: which = 0 gradp, 1 gradr (the phi and r slopes of
 * plm_phi / plm_trans, plm.c:15-195, from the last substep), 2 RKcons.
 */
int disco_batch_debug_get(disco_batch *b, int which, double *out);

/*
 * Launch all further work of the batch on `stream` (a cudaStream_t, passed
 * as void* so this header needs no CUDA include; NULL restores the batch's
 * own stream).  Lets a caller time the step with events on its own stream.
 */
int disco_batch_set_stream(disco_batch *b, void *stream);

/*
 * Choose how the step is launched (enum disco_schedule).  A new batch uses
 * DISCO_SCHED_KERNELS (the faster of the two on a B200: 4.8 against 8.3
 * ms per ragged64 step).  DISCO_SCHED_PERSISTENT needs modules it covers:
 * hydro or MHD without constrained transport, 2D disks, RK2, fixed / polar
 * boundaries, no Mesh_Motion 3, no viscosity; DISCO_ERR_UNSUPPORTED
 * otherwise.  No
 * counterpart in the reference (its onestep() is one sequence of loops);
 * disco_batch_get_schedule returns the schedule in use.
 */
int disco_batch_set_schedule(disco_batch *b, int sched);
int disco_batch_get_schedule(const disco_batch *b, int *sched);

/* GRMHD batches: from the next step on, every cons->prim of the step writes
 * its inputs for each real cell into dev (device memory of the batch's GPU,
 * DISCO_GR_DUMP_ROWS x ncell doubles, row-major: cons / dV in rows 0-8, the
 * warm-start prims -- the cell's prims before the solve -- in rows 9-17, the
 * cell centre x in rows 18-20); rows of other cells are left as they were,
 * and each substep overwrites the last.  These are exactly the arguments
 * the step's noble2d solve sees (disco_gr_cons2prim with dV = 1 solves them
 * to the same bits), so the plain solver's training pairs (include/disco_c2p.h)
 * can be written from the states of the run itself.  dev = NULL stops it.
 * Returns DISCO_ERR_UNSUPPORTED for a batch without HYDRO grmhd2. */
#define DISCO_GR_DUMP_ROWS 21
int disco_batch_set_gr_dump(disco_batch *b, double *dev);

/*
 * Run one full step with a CUDA event between every kernel launch and
 * return each launch's device time: ms[i] and the kernel's name in
 * names[i] (static strings), for i < *nlaunch (at most cap).  The
 * reference's profiler (profiler.c:188-206) labels the same phases.
 */
int disco_batch_kernel_times(disco_batch *b, float *ms, const char **names, int cap, int *nlaunch);

/*
 * getmindt for one disk whose state the caller already keeps in device
 * memory, computed without allocating any device memory.  No counterpart in
 * the reference: it exists for callers that may not call cudaMalloc (a host
 * code that owns all device memory through its own pool, or a loop that runs
 * while allocation is forbidden), since disco_batch_mindt needs a batch and
 * creating a batch allocates.
 *
 * Inputs: the disk's params, hydro module (DISCO_HYDRO_EULER only), grid as
 * for disco_batch_create (host arrays: Ng[4], Np[Nr*Nz], r_jph[Nr+1],
 * z_kph[Nz+1]) and device pointers to its cells in annulus order: prim as
 * structure-of-arrays (prim[q*ncell + c], q < 6), piph, dphi, wiph.  Work is
 * issued on `stream` (a cudaStream_t; NULL = default stream) and *dt (host)
 * receives CFL * min over real cells, the reference's getmindt value,
 * including the viscous limit of Use_Viscosity (euler.c:357-375).  The
 * arrays and the stream must belong to the current device; device arrays
 * of another device return DISCO_ERR_ARG.
 *
 * Limits: Nr*Nz <= 65536 annuli, Nr+1 and Nz+1 <= 8192, ncell <= 2^26;
 * larger grids return DISCO_ERR_ARG.  Working memory is one static device
 * array of about 3.2 MiB that every GPU using the library holds until exit.
 * The first call on a device looks up that array's device address
 * (cudaGetSymbolAddress); make it before any stream capture.  All calls share
 * the array: calls that overlap on the GPU race and must be serialised.
 */
int disco_mindt_noalloc(const disco_params *p, int hydro, int Nr, int Nz,
                        const int *Ng, const int *Np, const double *r_jph,
                        const double *z_kph, const double *prim, const double *piph,
                        const double *dphi, const double *wiph, void *stream, double *dt);

#ifdef __cplusplus
}
#endif
#endif
