"""Generate the golden fixtures of tests/golden/ by running the reference.

The reference Disco has no test vectors of its own (no tests/, no golden
data), so its behaviour is pinned by running it: oracle/Makefile compiles the
reference's unmodified serial sources with a fixed-step driver
(oracle/ref_driver.c), and this script records its state after 0 and N steps
for a few small configurations.  Run it where the reference tree is
available:

    python tests/golden/make_golden.py

Each case writes <case>.npz with the step-0 state (s0_*), the step-N state
(sN_*), the dt sequence, the r-face list after N steps and the diagnostics.
The checkpoint cases (ck_*) hold the state after N steps with its planets,
the reference's checkpoint datasets (ck_*) and ascii output of that state,
and the state after restarting from that checkpoint, 0 steps (r0_*) and M
steps (rM_*) later.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(REPO, "oracle"))
import pyoracle  # noqa: E402

TEMPLATES = os.path.join(REPO, "disco_b200", "templates")

# the 3D rigid disk of the composed boundary modules' fixtures
BC3D = {"Num_R": 10, "Num_Z": 4, "Z_Min": -0.3, "Z_Max": 0.3, "Log_Zoning": 0, "Init_Par2": 1,
        "Init_Par1": 0.05, "Energy_Omega": 0, "Mach_Number": 5.0}

# case -> (module config, in.par overrides, steps)
CASES = {
    "c0_log16": ("c0_kepler2d", {"Num_R": 16}, 8),
    "c0_lin20": ("c0_kepler2d", {"Num_R": 20, "Log_Zoning": 0, "Mach_Number": 12.0,
                                 "Init_Par0": 27}, 8),
    "c0_hll_fe_mm3": ("c0_kepler2d", {"Num_R": 10, "Riemann_Solver": 0, "Timestep": 1,
                                      "Mesh_Motion": 3, "PLM": 1.2}, 6),
    "c0_cm2": ("c0_cm2", {"Num_R": 24, "Mass_Ratio": 1.0e-3, "Energy_Omega": 0}, 6),
    # libm-free: rigid rotation held by pressure, no gravity, lab energy frame
    "c0_rigid": ("c0_nograv", {"Num_R": 20, "Log_Zoning": 0, "Init_Par2": 1,
                               "Energy_Omega": 0, "Mach_Number": 5.0}, 8),
    # Newtonian MHD (mhd.c, no CT): HLLD, HLLC-MHD and HLL + forward Euler
    "c1_mhd_hlld": ("c1_mhd2d", {}, 8),
    "c1_mhd_hllc": ("c1_mhd2d", {"Num_R": 12, "Riemann_Solver": 1, "Init_Par0": 99}, 6),
    "c1_mhd_hll_fe": ("c1_mhd2d", {"Num_R": 10, "Riemann_Solver": 0, "Timestep": 1,
                                   "Mesh_Motion": 1, "Init_Par1": 0.05}, 6),
    # libm-free MHD: rigid rotation held by pressure, no gravity, HLLD
    "c1_mhd_rigid": ("c1_mhd2d_nograv", {"Num_R": 14, "Init_Par2": 1, "Init_Par4": 10.0}, 8),
    # zero-gradient boundaries (Boundary/zerograd.c), 2D hydro
    "c0_zg": ("c0_zerograd", {"Num_R": 16, "Init_Par0": 4242}, 6),
    # 3D: z faces, z slopes and fluxes (hydro, fixed; MHD HLLD, zerograd)
    "c0_3d": ("c0_fixed3d", {"Num_R": 10, "Num_Z": 4, "Grav2D": 1, "Z_Min": -0.3,
                             "Z_Max": 0.3}, 4),
    "c1_mhd3d": ("c1_mhd3d", {"Num_R": 8, "Num_Z": 6}, 5),
    "c1_mhd3d_rigid": ("c1_mhd3d_nograv", {"Num_R": 8, "Num_Z": 6, "Init_Par2": 1,
                                           "Init_Par4": 10.0}, 6),
    # 2D constrained transport (bfields.c) with toroidal and radial field:
    # Keplerian HLLD, libm-free rigid HLLD, and HLL + forward Euler with the
    # by-cell mesh
    "c1_ct2d": ("c1_mhd2d", {"Num_R": 12, "Constrained_Transport": 1, "Init_Par5": 20.0,
                             "Init_Par6": 0.05}, 8),
    "c1_ct_rigid": ("c1_mhd2d_nograv", {"Num_R": 14, "Init_Par2": 1, "Init_Par4": 10.0,
                                        "Constrained_Transport": 1, "Init_Par5": 20.0,
                                        "Init_Par6": 0.05}, 8),
    "c1_ct_hll_fe": ("c1_mhd2d", {"Num_R": 10, "Riemann_Solver": 0, "Timestep": 1,
                                  "Mesh_Motion": 1, "Constrained_Transport": 1,
                                  "Init_Par5": 10.0, "Init_Par6": 0.1}, 6),
    # 3D constrained transport (CT_MODE 2: z faces, E_phi edges, make_edge_adjust),
    # zero-gradient boundaries: Keplerian HLLD and libm-free rigid HLLD
    "c1_ct3d": ("c1_mhd3d", {"Num_R": 8, "Num_Z": 6, "Constrained_Transport": 1,
                             "Init_Par5": 20.0, "Init_Par6": 0.05}, 5),
    "c1_ct3d_rigid": ("c1_mhd3d_nograv", {"Num_R": 8, "Num_Z": 6, "Init_Par2": 1,
                                          "Init_Par4": 10.0, "Constrained_Transport": 1,
                                          "Init_Par5": 20.0, "Init_Par6": 0.05}, 6),
    # the polar boundary module (Boundary/polar.c) on grids down to the axis
    # (NoBC_Rmin 1, R_Min 0): no inner ghosts, the axis gradient fix
    # (plm_geom_boundary -> geom_grad) and the polar source terms; rigid
    # rotation without gravity, hydro 2D, MHD 2D with CT, MHD 3D with CT
    "c0_polar": ("c0_polar", {"Num_R": 16, "R_Min": 0.0, "R_Max": 2.0, "NoBC_Rmin": 1,
                              "Log_Zoning": 0, "Init_Par2": 1, "Init_Par1": 0.05,
                              "Energy_Omega": 0, "Mach_Number": 5.0}, 8),
    "c1_polar_ct": ("c1_polar", {"Num_R": 14, "R_Min": 0.0, "R_Max": 2.0, "NoBC_Rmin": 1,
                                 "Init_Par2": 1, "Init_Par4": 10.0, "Constrained_Transport": 1,
                                 "Init_Par5": 20.0}, 8),
    "c1_polar3d": ("c1_polar3d", {"Num_R": 8, "Num_Z": 6, "R_Min": 0.0, "R_Max": 2.0,
                                  "NoBC_Rmin": 1, "Init_Par2": 1, "Init_Par4": 10.0,
                                  "Constrained_Transport": 1, "Init_Par5": 20.0}, 5),
    # boundary modules composed from boundary_functions.c: outflow3d
    # (zero-gradient, outflow diode, every side), zerograd_omk (the same with
    # Omega of the r ghosts from the Initial module), accrete3d (outflow
    # inner r, fixed outer r and z; with CT)
    "c0_outflow3d": ("c0_outflow3d", {"Num_R": 10, "Num_Z": 4, "Z_Min": -0.3, "Z_Max": 0.3,
                                      "Log_Zoning": 0, "Init_Par2": 1, "Init_Par1": 0.05,
                                      "Energy_Omega": 0, "Mach_Number": 5.0}, 5),
    "c1_omk3d": ("c1_omk3d", {"Num_R": 8, "Num_Z": 6, "Init_Par2": 1, "Init_Par4": 10.0}, 5),
    "c1_accrete3d": ("c1_accrete3d", {"Num_R": 8, "Num_Z": 6, "Init_Par2": 1, "Init_Par4": 10.0,
                                      "Constrained_Transport": 1, "Init_Par5": 20.0}, 5),
    # setupCells options: addNoise (noise.c, glibc rand() in cell order)
    # types 1 (v_r, Omega), 2 (P) and 3 (v_r, v_z from r Omega), libm-free;
    # Include_Atmos (adjust_gas with the binary's potential)
    "c0_noise1": ("c0_nograv", {"Num_R": 16, "Log_Zoning": 0, "Init_Par2": 1, "Energy_Omega": 0,
                                "Mach_Number": 5.0, "Noise_Type": 1, "Noise_Abs": 1.0e-3,
                                "Noise_Rel": 1.0e-2}, 6),
    "c0_noise2": ("c0_nograv", {"Num_R": 16, "Log_Zoning": 0, "Init_Par2": 1, "Energy_Omega": 0,
                                "Mach_Number": 5.0, "Noise_Type": 2, "Noise_Abs": 1.0e-4,
                                "Noise_Rel": 2.0e-2}, 6),
    "c1_noise3": ("c1_mhd3d_nograv", {"Num_R": 8, "Num_Z": 6, "Init_Par2": 1, "Init_Par4": 10.0,
                                      "Noise_Type": 3, "Noise_Abs": 1.0e-3,
                                      "Noise_Rel": 1.0e-2}, 5),
    "c0_atmos": ("c0_cm2", {"Num_R": 24, "Mass_Ratio": 1.0e-3, "Energy_Omega": 0,
                            "Include_Atmos": 1}, 6),
    # viscosity (euler.c visc_flux / visc_source / mindt): constant nu large
    # enough that the viscous dt limit binds (libm-free), and alpha viscosity
    # on the Keplerian disk (pow)
    "c0_visc": ("c0_nograv", {"Num_R": 16, "Log_Zoning": 0, "Init_Par2": 1, "Energy_Omega": 0,
                              "Mach_Number": 5.0, "Use_Viscosity": 1, "Viscosity": 0.5}, 6),
    "c0_visc_alpha": ("c0_kepler2d", {"Num_R": 24, "Use_Viscosity": 1, "Use_As_Alpha": 1,
                                      "Viscosity": 0.01}, 6),
    # Planets/circular.c (star + planet on a circular orbit) and Planets/cm.c
    # (binary about the centre of mass, softening relaxing as exp(-t/30))
    "c0_circular": ("c0_circular", {"Num_R": 24, "Mass_Ratio": 1.0e-3, "Energy_Omega": 0}, 6),
    # (started at t = 300, where the softening has relaxed: from t = 0 the
    # eps ~ 1 binary cannot hold the Keplerian disk and the reference blows up)
    "c0_cm": ("c0_cm", {"Num_R": 24, "Mass_Ratio": 1.0e-3, "Energy_Omega": 0, "T_Start": 300.0,
                        "Mach_Number": 5.0}, 6),
    # from t = 0, where eps = 0.5/Mach + exp(-t/30) ~ 1 changes every step: a
    # rigidly rotating, pressure-held disk that needs no Keplerian balance
    "c0_cm_t0": ("c0_cm", {"Num_R": 20, "Log_Zoning": 0, "Init_Par2": 1, "Energy_Omega": 0,
                           "Mach_Number": 5.0, "Mass_Ratio": 0.5}, 6),
    # Diagnostics/diag_euler.c (8 annulus averages: the flux of vz, the
    # angular momentum and the pressure beside diag_disk2d's), with the
    # planet torque term (cm2) and in 3D
    "c0_diag_euler": ("c0_diag_euler", {"Num_R": 24, "Mass_Ratio": 1.0e-3, "Energy_Omega": 0}, 6),
    "c0_diag_euler3d": ("c0_diag_euler3d", {"Num_R": 10, "Num_Z": 4, "Grav2D": 1, "Z_Min": -0.3,
                                            "Z_Max": 0.3}, 4),
    # Diagnostics/diag_mhdmri.c (18 annulus averages of the MHD state)
    "c1_diag_mhdmri": ("c1_diag_mhdmri", {"Num_R": 12}, 6),
    # an outer edge without ghost annuli (NoBC_Rmax 1): the last real
    # annulus has no outer track
    "c0_nobc_rmax": ("c0_nograv", {"Num_R": 16, "Log_Zoning": 0, "Init_Par2": 1,
                                   "Energy_Omega": 0, "Mach_Number": 5.0, "NoBC_Rmax": 1}, 8),
    # a reference Initial module (Initial/rigid.c), evaluated by the host
    # set-up only: the drop-in with zero-gradient boundaries (the par file is
    # what tests/test_gpu_dropin.py runs both binaries on)
    "c0_rigid_zg": ("c0_rigid_zg", {"Num_R": 32, "Log_Zoning": 0, "Energy_Omega": 0}, 8),
    # GRMHD (Hydro/grmhd2.c with the Schwarzschild Kerr-Schild metric
    # schw_ks_rpz and the normal frame, HLL): the gr_torus_noise torus with
    # its loop field and pressure noise, fixed3d ghosts; by-cell mesh motion
    # (get_omega of grmhd2) and a fixed mesh.  Only +, -, *, /, sqrt occur.
    # config 4's module set (MHD, HLLD, 3D CT, zerograd) with the softened
    # equal-mass binary (Planets/binary_soft.c of this repo, compiled into the
    # reference build): point-mass forces use libm (1e-11)
    "c4_binary3d": ("c4_binary3d", {"Num_R": 12, "Num_Z": 6, "Constrained_Transport": 1}, 5),
    "c3_grtorus": ("c3_grtorus", {"Num_R": 16, "Num_Z": 8}, 5),
    "c3_grtorus_mm0": ("c3_grtorus", {"Num_R": 12, "Num_Z": 6, "Mesh_Motion": 0,
                                      "Init_Par0": 2718}, 4),
    # the excising boundary modules: horizon3d (boundary_fixed_horizon, the
    # annuli inside R < 1 re-initialised by set_cell_init every substep and
    # left out of the dt minimum) on a 3D hydro grid down to the axis, and
    # horizon (Boundary/horizon.c: inside 0.7 r_H of M = 1, midpoint
    # re-initialisation) under the GRMHD torus with its inner edge at
    # r = 0.5 and no inner ghosts; polar3d (outer r and z ghosts from
    # set_cell_init, no inner ghosts) with 3D CT
    "c0_horizon3d": ("c0_horizon3d", {"Num_R": 10, "Num_Z": 6, "Z_Min": -0.6, "Z_Max": 0.6,
                                      "R_Min": 0.0, "R_Max": 2.0, "NoBC_Rmin": 1,
                                      "Log_Zoning": 0, "Init_Par2": 1, "Init_Par1": 0.05,
                                      "Energy_Omega": 0, "Mach_Number": 5.0}, 5),
    "c1_polar3dbc": ("c1_polar3dbc", {"Num_R": 8, "Num_Z": 6, "R_Min": 0.0, "R_Max": 2.0,
                                      "NoBC_Rmin": 1, "Init_Par2": 1, "Init_Par4": 10.0,
                                      "Constrained_Transport": 1, "Init_Par5": 20.0}, 5),
    "c3_grhorizon": ("c3_grhorizon", {"Num_R": 16, "Num_Z": 8, "R_Min": 0.5, "NoBC_Rmin": 1}, 5),
    # 3D constrained transport with z boundaries without ghost layers
    # (NoBC_Zmin / NoBC_Zmax 1): avg_Efields' z-pole branch (bfields.c:580-617)
    # averages the bottom layer's E[5] and the top layer's E[4] over each
    # annulus; libm-free rigid HLLD with zerograd r ghosts, and with the polar
    # module down to the axis (both poles of the domain at once)
    "c1_ct3d_zpole": ("c1_mhd3d_nograv", {"Num_R": 8, "Num_Z": 6, "Init_Par2": 1, "Init_Par4": 10.0,
                                          "Constrained_Transport": 1, "Init_Par5": 20.0,
                                          "Init_Par6": 0.05, "NoBC_Zmin": 1, "NoBC_Zmax": 1}, 6),
    # horizon_bin (Boundary/horizon_bin.c): two excision spheres of radius 0.8
    # at x = +-5 -- cells inside are re-initialised each substep and, once
    # excised, stay out of the dt minimum (the reference's real flag is never
    # set back); rigid rotation moves cells through them.  2D and 3D hydro,
    # no inner ghosts (the module sets none); the test is per cell with cos
    # and sin of the cell's phi
    "c0_hbin": ("c0_hbin", {"Num_R": 24, "R_Min": 3.5, "R_Max": 7.0, "NoBC_Rmin": 1, "Log_Zoning": 0,
                            "Init_Par2": 1, "Init_Par1": 0.05, "Energy_Omega": 0, "Mach_Number": 5.0}, 8),
    "c0_hbin3d": ("c0_hbin", {"Num_R": 16, "Num_Z": 6, "Z_Min": -0.6, "Z_Max": 0.6, "R_Min": 3.5,
                              "R_Max": 7.0, "NoBC_Rmin": 1, "Log_Zoning": 0, "Init_Par2": 1,
                              "Init_Par1": 0.05, "Energy_Omega": 0, "Mach_Number": 5.0}, 5),
    # the other modules composed from boundary_functions.c, with mirror
    # copies (boundary_reflect_*: the annulus as far inside as the ghost is
    # outside, normal velocity negated by reflect_prims): fixRrefZ (fixed r,
    # reflecting z), tube (reflecting outer r, zero-gradient z; no inner
    # ghosts), surfaceGravBox (reflecting r and lower z, outflow upper z),
    # fixed_gap (outflow inner r and z, fixed outer r); 3D hydro, rigid
    "c0_bc_fixRrefZ": ("c0_bc_fixRrefZ", dict(BC3D), 5),
    "c0_bc_tube": ("c0_bc_tube", dict(BC3D, NoBC_Rmin=1), 5),
    "c0_bc_surfaceGravBox": ("c0_bc_surfaceGravBox", dict(BC3D), 5),
    "c0_bc_fixed_gap": ("c0_bc_fixed_gap", dict(BC3D), 5),
    # flowthrough: a no-slip inner wall (mirror copy, all three velocity
    # components negated), outflow outer r fixed again on 0.3 pi < phi < 1.7 pi
    # after the copy, fixed z
    "c0_bc_flowthrough": ("c0_bc_flowthrough", dict(BC3D), 5),
    "c1_polar3d_zpole": ("c1_polar3d", {"Num_R": 8, "Num_Z": 6, "R_Min": 0.0, "R_Max": 2.0,
                                        "NoBC_Rmin": 1, "Init_Par2": 1, "Init_Par4": 10.0,
                                        "Constrained_Transport": 1, "Init_Par5": 20.0,
                                        "NoBC_Zmin": 1, "NoBC_Zmax": 1}, 5),
}

# the in.par template each module configuration starts from
BASE_PAR = {"c0_kepler2d": "c0_kepler2d", "c0_cm2": "c0_kepler2d", "c0_nograv": "c0_kepler2d",
            "c1_mhd2d": "c1_mhd2d", "c1_mhd2d_nograv": "c1_mhd2d", "c0_zerograd": "c0_kepler2d", "c0_fixed3d": "c0_kepler2d",
            "c1_mhd3d": "c1_mhd3d", "c1_mhd3d_nograv": "c1_mhd3d", "c0_polar": "c0_kepler2d",
            "c1_polar": "c1_mhd2d", "c1_polar3d": "c1_mhd3d", "c0_outflow3d": "c0_kepler2d",
            "c1_omk3d": "c1_mhd3d", "c1_accrete3d": "c1_mhd3d", "c0_rigid_zg": "c0_kepler2d",
            "c0_circular": "c0_kepler2d", "c0_cm": "c0_kepler2d", "c0_diag_euler": "c0_kepler2d",
            "c0_diag_euler3d": "c0_kepler2d", "c1_diag_mhdmri": "c1_mhd2d", "c3_grtorus": "c3_grtorus", "c4_binary3d": "c4_binary3d",
            "c0_horizon3d": "c0_kepler2d", "c1_polar3dbc": "c1_mhd3d", "c3_grhorizon": "c3_grtorus",
            "c0_hbin": "c0_kepler2d", "c0_bc_fixRrefZ": "c0_kepler2d", "c0_bc_tube": "c0_kepler2d",
            "c0_bc_surfaceGravBox": "c0_kepler2d", "c0_bc_fixed_gap": "c0_kepler2d",
            "c0_bc_flowthrough": "c0_kepler2d"}


def par_text(cfg_par, overrides):
    out = []
    with open(os.path.join(TEMPLATES, cfg_par + ".par")) as f:
        for line in f:
            key = line.split()[0] if line.split() else ""
            if key in overrides:
                line = "%s\t\t%s\n" % (key, repr(overrides[key]) if isinstance(overrides[key], float)
                                       else overrides[key])
            out.append(line)
    return "".join(out)


# Checkpoint and restart (Output/h5out.c, Output/ascii.c, Restart/h5in.c
# through oracle/ref_checkpoint.c): case -> (module config, in.par overrides,
# steps before the checkpoint N, steps after the restart M)
CKPT_CASES = {
    # moving binary (planets in the checkpoint), point-mass gravity, diagnostics
    "ck_cm2": ("c0_cm2", {"Num_R": 24, "Mass_Ratio": 1.0e-3, "Energy_Omega": 0}, 6, 4),
    # libm-free: hydro without face fluxes (NUM_FACES 0), 2D CT (3), 3D CT (5)
    "ck_rigid": ("c0_nograv", {"Num_R": 20, "Log_Zoning": 0, "Init_Par2": 1,
                               "Energy_Omega": 0, "Mach_Number": 5.0}, 8, 4),
    "ck_ct_rigid": ("c1_mhd2d_nograv", {"Num_R": 14, "Init_Par2": 1, "Init_Par4": 10.0,
                                        "Constrained_Transport": 1, "Init_Par5": 20.0,
                                        "Init_Par6": 0.05}, 8, 4),
    # setupCells adds noise on restart too (domain.c:202-203)
    "ck_noise": ("c0_nograv", {"Num_R": 16, "Log_Zoning": 0, "Init_Par2": 1, "Energy_Omega": 0,
                               "Mach_Number": 5.0, "Noise_Type": 1, "Noise_Abs": 1.0e-3,
                               "Noise_Rel": 1.0e-2}, 6, 3),
    "ck_ct3d_rigid": ("c1_mhd3d_nograv", {"Num_R": 6, "Num_Z": 5, "Init_Par2": 1,
                                          "Init_Par4": 10.0, "Constrained_Transport": 1,
                                          "Init_Par5": 20.0, "Init_Par6": 0.05}, 4, 3),
}

CK_FILES = (("T", "f64"), ("r_jph", "f64"), ("z_kph", "f64"), ("Index", "i32"), ("Np", "i32"),
            ("Id_phi0", "i32"), ("Cells", "f64"), ("Planets", "f64"), ("Diagnostics", "f64"))


def read_ck(d):
    """oracle/ref_checkpoint.c's raw datasets as arrays of their shapes."""
    NrT, NzT, Nc, Nq, Npl, NpDat, Nt = (int(x) for x in open(os.path.join(d, "dims.txt")).read().split())
    shapes = {"T": (1,), "r_jph": (NrT + 1,), "z_kph": (NzT + 1,), "Index": (NzT, NrT),
              "Np": (NzT, NrT), "Id_phi0": (NzT, NrT), "Cells": (Nc, Nq), "Planets": (Npl, NpDat),
              "Diagnostics": (NzT, NrT, Nt)}
    out = {}
    for name, t in CK_FILES:
        a = np.fromfile(os.path.join(d, name + "." + t), np.float64 if t == "f64" else np.int32)
        out[name] = a.reshape(shapes[name])
    return out


def run_env(cfg, text, nsteps, env):
    """Run the reference with extra environment; returns (dump, workdir)."""
    import subprocess
    import tempfile
    binary = pyoracle.build_ref(cfg)
    work = tempfile.mkdtemp(prefix="disco_ck_")
    with open(os.path.join(work, "in.par"), "w") as f:
        f.write(text)
    subprocess.run([binary, work, str(nsteps), os.path.join(work, "dump")], check=True,
                   stdout=subprocess.DEVNULL, env=dict(os.environ, **env))
    return pyoracle.load_dump(os.path.join(work, "dump")), work


def make_ckpt(case):
    import shutil
    cfg, over, n, m = CKPT_CASES[case]
    text = par_text(BASE_PAR[cfg], over)
    with open(os.path.join(HERE, case + ".par"), "w") as f:
        f.write(text)
    d0 = pyoracle.run_ref(cfg, text, 0)
    probe = os.path.join(HERE, "_ck_tmp")
    os.makedirs(probe, exist_ok=True)
    dn, w = run_env(cfg, text, n, {"DISCO_REF_CHECKPOINT": os.path.join(probe, "ck"),
                                   "DISCO_REF_ASCII": os.path.join(probe, "ascii")})
    ck = read_ck(os.path.join(probe, "ck"))
    with open(os.path.join(probe, "ascii.dat"), "rb") as f:
        ascii_bytes = np.frombuffer(f.read(), np.uint8)
    rtext = par_text(BASE_PAR[cfg], dict(over, Restart=1))
    r0, w0 = run_env(cfg, rtext, 0, {"DISCO_REF_RESTART": os.path.join(probe, "ck")})
    rm, wm = run_env(cfg, rtext, m, {"DISCO_REF_RESTART": os.path.join(probe, "ck")})
    for x in (w, w0, wm):
        shutil.rmtree(x, ignore_errors=True)
    shutil.rmtree(probe, ignore_errors=True)
    # the step-N prim, Phi and piph are the checkpoint's Cells columns
    keep = {"s0_": ("prim", "cons", "piph", "dphi", "wiph", "Phi"), "sN_": ("dphi", "wiph"),
            "r0_": ("prim", "cons", "piph", "dphi", "wiph", "Phi"), "rM_": ("prim", "cons", "piph", "Phi")}
    extra = {}
    for p, d in (("s0_", d0), ("sN_", dn), ("r0_", r0), ("rM_", rm)):
        for k in keep[p]:
            if k in d and (k != "Phi" or over.get("Constrained_Transport")):
                extra[p + k] = d[k]
    np.savez_compressed(
        os.path.join(HERE, case + ".npz"), cfg=cfg, nsteps=n, msteps=m, real=d0["real"],
        Np=d0["Np"], r_jph=d0["r_jph"], z_kph=d0["z_kph"],
        sN_t=dn["meta"]["t"], sN_planets=dn["planets"], sN_t_avg=dn["meta"]["t_avg"], sN_Qrz=dn["Qrz"],
        r0_dt_next=r0["dt_next"], r0_planets=r0["planets"], r0_t=r0["meta"]["t"],
        rM_dt=rm["dt"], rM_dt_next=rm["dt_next"], rM_t=rm["meta"]["t"], rM_planets=rm["planets"],
        ascii=ascii_bytes, **{"ck_" + k: v for k, v in ck.items()}, **extra)
    print(case, "cells", d0["meta"]["Ncell"], "ascii bytes", ascii_bytes.size)


def main():
    only = set(sys.argv[1:])
    for case in CKPT_CASES:
        if not only or case in only:
            make_ckpt(case)
    for case, (cfg, over, n) in CASES.items():
        if only and case not in only:
            continue
        text = par_text(BASE_PAR[cfg], over)
        with open(os.path.join(HERE, case + ".par"), "w") as f:
            f.write(text)
        d0 = pyoracle.run_ref(cfg, text, 0)
        dn = pyoracle.run_ref(cfg, text, n)
        F = dn["faces_1"]
        extra = {}
        if "Phi" in d0 and over.get("Constrained_Transport"):
            extra.update(s0_Phi=d0["Phi"], sN_Phi=dn["Phi"])
        if "faces_2" in dn:
            Z = dn["faces_2"]
            extra.update(z_fIndex=Z["fIndex"], z_iL=Z["iL"], z_iR=Z["iR"], z_LRtype=Z["LRtype"],
                         z_fgeom=Z["geom"])
        np.savez_compressed(
            os.path.join(HERE, case + ".npz"), cfg=cfg, nsteps=n,
            s0_prim=d0["prim"], s0_cons=d0["cons"], s0_piph=d0["piph"], s0_dphi=d0["dphi"],
            s0_wiph=d0["wiph"], real=d0["real"], s0_dt_next=d0["dt_next"],
            sN_prim=dn["prim"], sN_cons=dn["cons"], sN_piph=dn["piph"], sN_dphi=dn["dphi"],
            sN_wiph=dn["wiph"], dt=dn["dt"], sN_dt_next=dn["dt_next"], Qrz=dn["Qrz"],
            t=dn["meta"]["t"], fIndex=F["fIndex"], iL=F["iL"], iR=F["iR"], LRtype=F["LRtype"],
            fgeom=F["geom"], Np=d0["Np"], r_jph=d0["r_jph"], z_kph=d0["z_kph"], **extra)
        print(case, "cells", d0["meta"]["Ncell"], "faces", len(F["iL"]))


if __name__ == "__main__":
    main()
