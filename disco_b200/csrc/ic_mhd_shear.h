/*
 * Magnetised Keplerian shearing disk with seeded, hash-based velocity noise.
 *
 * A new initial-condition module for the MHD workloads (the reference's MHD
 * disk ICs, e.g. Initial/flock.c, draw their noise from rand() in cell
 * order, which a device cannot evaluate per cell).  Like kepler_noise, the
 * noise is a pure function of the cell position, so the host build, the
 * device set-up and the boundary kernels agree for the same x.
 *
 *   rho   = 1
 *   P     = rho cs^2 / gamma                      (sound speed cs)
 *   Omega = r^-3/2 + amp cs u_phi / r
 *   v_r   = amp cs u_r,   v_z = amp cs u_z        (u in [-1,1), hashed)
 *   B     = (Br, Bphi, Bz)
 *           Bz   = sqrt(2 P / beta)               (vertical field, plasma beta)
 *           Bphi = sqrt(2 P / beta_phi)           (uniform toroidal field; 0 when
 *                                                  beta_phi = 0)
 *           Br   = b_r (rmin / r) u(phi),  u = 4 s (1 - s) - 2/3,  s = phi/phimax
 *                                                 (mod 1): r Br is independent of r
 *                                                  and Bphi of phi, so div B = 0
 *   X     = (z - zmin)/(zmax - zmin)              (passive scalar, NUM_N>0)
 *
 * With Init_Par2 = 1 the disk rotates rigidly instead (Omega = 1 + noise),
 * held by pressure, P = rho cs^2/gamma + r^2/2, so no gravity is needed:
 * with PLANETS = none and Energy_Omega 0 a step calls no libm function
 * whose value matters, and a CPU and a GPU build agree bit for bit.
 * With Init_Par2 = 2 it is a circumbinary disk: surface density
 * rho = (rmin/r)^(1/2) (1 + amp u_rho), P = rho cs^2/gamma, Keplerian Omega
 * about the unit total mass, no velocity noise (Bphi's beta then follows the
 * local pressure).
 *
 * Noise only inside [rmin, rmax] x [zmin, zmax] (ghost cells stay smooth).
 * Uses +,-,*,/, sqrt and floor only, so host and device values are
 * bit-identical.
 *
 * Parameters (in.par): Init_Par0 = seed, Init_Par1 = amp (fraction of cs),
 * Init_Par2 = kind (0 Keplerian, 1 rigid, 2 circumbinary), Init_Par3 = cs, Init_Par4 = beta,
 * Init_Par5 = beta_phi, Init_Par6 = b_r, Adiabatic_Index, R_Min/R_Max,
 * Z_Min/Z_Max, Phi_Max.
 */
#ifndef DISCO_IC_MHD_SHEAR_H
#define DISCO_IC_MHD_SHEAR_H

#include "ic_kepler_noise.h"

typedef struct {
   double cs, beta, amp, gam;
   double beta_phi, b_r;
   double rmin, rmax, zmin, zmax, phimax;
   uint64_t seed;
   int kind;
   int pad;
} disco_ic_mhd_shear;

/* Uniform in [-1,1) from the seed, a salt and the cell position (r, phi, z
 * bucketed as disco_hash_unit does). */
DISCO_HD double disco_hash_unit3(uint64_t seed, uint64_t salt, double r, double phi, double z,
                                 double phimax){
   int64_t qr = (int64_t)(r * 1048576.0);
   int64_t qp = (int64_t)((phi / phimax) * 16777216.0);
   int64_t qz = (int64_t)((z + 1024.0) * 1048576.0);
   uint64_t h = disco_mix64(seed ^ disco_mix64(salt * 0x9E3779B97F4A7C15ull
                                               ^ (uint64_t)qr * 0x100000001B3ull
                                               ^ ((uint64_t)qp << 1)
                                               ^ ((uint64_t)qz << 29)));
   double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
   return 2.0 * u - 1.0;
}

/* prim layout: RHO, PPP, URR, UPP, UZZ, BRR, BPP, BZZ, passive... */
DISCO_HD void disco_ic_mhd_shear_eval(const disco_ic_mhd_shear *p, int num_c, int num_q,
                                      double *prim, const double *x){
   double r = x[0], phi = x[1], z = x[2];
   double sr = sqrt(r);
   double omega = 1.0 / (r * sr);
   double rho = 1.0;
   double press = rho * p->cs * p->cs / p->gam;
   if( p->kind == 1 ){
      omega = 1.0;
      press = press + 0.5 * r * r;
   }
   double vr = 0.0, vz = 0.0;
   int inside = r >= p->rmin && r <= p->rmax && z >= p->zmin && z <= p->zmax;
   if( p->kind == 2 ){
      rho = sqrt(p->rmin / r);
      if( inside && p->amp != 0.0 ) rho *= 1.0 + p->amp * disco_hash_unit3(p->seed, 4, r, phi, z, p->phimax);
      press = rho * p->cs * p->cs / p->gam;
   }else if( inside && p->amp != 0.0 ){
      double a = p->amp * p->cs;
      vr = a * disco_hash_unit3(p->seed, 1, r, phi, z, p->phimax);
      vz = a * disco_hash_unit3(p->seed, 2, r, phi, z, p->phimax);
      omega += a * disco_hash_unit3(p->seed, 3, r, phi, z, p->phimax) / r;
   }
   prim[0] = rho;
   prim[1] = press;
   prim[2] = vr;
   prim[3] = omega;
   prim[4] = vz;
   int q;
   for( q=5 ; q<num_c ; ++q ) prim[q] = 0.0;
   if( num_c >= 8 ){
      double p0 = rho * p->cs * p->cs / p->gam;     /* the disk's gas pressure */
      prim[7] = sqrt(2.0 * p0 / p->beta);
      if( p->beta_phi > 0.0 ) prim[6] = sqrt(2.0 * p0 / p->beta_phi);
      if( p->b_r != 0.0 ){
         double s = phi / p->phimax;
         s = s - floor(s);
         prim[5] = p->b_r * (p->rmin / r) * (4.0 * s * (1.0 - s) - 2.0 / 3.0);
      }
   }
   if( num_q > num_c ){
      double zr = p->zmax > p->zmin ? (z - p->zmin) / (p->zmax - p->zmin) : 0.5;
      prim[num_c] = zr;
      for( q=num_c+1 ; q<num_q ; ++q ) prim[q] = 0.0;
   }
}

#endif
