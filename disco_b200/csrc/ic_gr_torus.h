/*
 * GRMHD torus with seeded, hash-based pressure noise: a new Initial module
 * for the GRMHD timestep (the reference has no cylindrical torus IC: its
 * Fishbone-Moncrief torus, Initial/torus_fm_grmhd.c, is written in the
 * spherical coordinates of schw_ks_rpt).  It is a state with the features
 * a torus run exercises -- a dense, hot, rotating ring with a weak poloidal
 * loop field inside a thin infalling atmosphere -- not an exact equilibrium:
 *
 *   R = sqrt(r^2 + z^2),  d2 = ((R - rc)/wr)^2 + (z/(hr R))^2
 *   s = (1 - d2)^2 for d2 < 1, else 0              (compact bump, C^1)
 *   rho = rho_atm R^-3/2 + s
 *   P   = p_atm R^-5/2 + K s^2 (1 + amp u),  K = hr^2 M / rc,
 *         u in [-1,1) hashed from (seed, r, phi, z), inside the real domain only
 *   u_phi = s r^2 sqrt(M) / (R^3/2 + a sqrt(M))    (covariant, prograde)
 *   u_r   = -(1 - s) sqrt(M / (2R)),  u_z = u_r z / R   (atmosphere infall)
 *   A_phi = (s - s_cut) for s > s_cut, else 0;  B^r = -B0 dA/dz,
 *   B^z = B0 (1/r) d(r A)/dr  (divergence free),  B0 = sqrt(2 K / beta) wr / 2
 *   X = s                                           (passive scalar)
 *
 * The prim slots are the grmhd2 module's (Hydro/grmhd2.c:88-180): RHO, PPP,
 * the covariant u_r, u_phi, u_z, then the field slots BRR, BPP, BZZ, then X.
 *
 * Only +, -, *, / and sqrt appear (each correctly rounded in IEEE double
 * on gcc/x86-64 and CUDA), so host and device give the same bits for the
 * same x, and the fixed3d boundary's re-evaluation every substep is
 * idempotent.  The noise is applied only inside [rmin, rmax] x [zmin, zmax]
 * (ghost cells lie outside, so their values stay smooth in x).
 *
 * Parameters (in.par): Init_Par0 seed, Init_Par1 noise amplitude,
 * Init_Par2 rc, Init_Par3 wr, Init_Par4 hr, Init_Par5 beta, Init_Par6
 * rho_atm, Init_Par7 p_atm, Init_Par8 s_cut; Metric_Par2 M, Metric_Par3 a;
 * R_Min/R_Max, Z_Min/Z_Max, Phi_Max.
 */
#ifndef DISCO_IC_GR_TORUS_H
#define DISCO_IC_GR_TORUS_H

#include "ic_kepler_noise.h"      /* DISCO_HD, disco_mix64 */

typedef struct {
   double M, a;
   double rc, wr, hr, beta;
   double rho_atm, p_atm, s_cut, amp;
   double rmin, rmax, zmin, zmax, phimax;
   uint64_t seed;
} disco_ic_gr_torus;

/* uniform in [-1, 1) from the seed and the cell position (r, z bucketed at
 * 2^-20, phi at Pmax 2^-24, as disco_hash_unit) */
DISCO_HD double disco_hash_unit3(uint64_t seed, double r, double phi, double z, double phimax){
   int64_t qr = (int64_t)(r * 1048576.0);
   int64_t qz = (int64_t)(z * 1048576.0);
   int64_t qp = (int64_t)((phi / phimax) * 16777216.0);
   uint64_t h = disco_mix64(seed ^ disco_mix64((uint64_t)qr * 0x100000001B3ull
                                               ^ ((uint64_t)qp << 1)
                                               ^ ((uint64_t)qz * 0x9E3779B97F4A7C15ull)));
   double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
   return 2.0 * u - 1.0;
}

DISCO_HD void disco_ic_gr_torus_eval(const disco_ic_gr_torus *p, int num_c, int num_q,
                                     double *prim, const double *x){
   const double r = x[0], phi = x[1], z = x[2];
   const double R = sqrt(r*r + z*z);
   const double sR = sqrt(R);
   const double dR = (R - p->rc)/p->wr;
   const double zh = z/(p->hr*R);
   const double d2 = dR*dR + zh*zh;
   const double one_m = 1.0 - d2;
   const double s = d2 < 1.0 ? one_m*one_m : 0.0;
   const double K = p->hr*p->hr*p->M/p->rc;
   double P = p->p_atm/(R*R*sR) + K*s*s;
   if( r >= p->rmin && r <= p->rmax && z >= p->zmin && z <= p->zmax && p->amp != 0.0 && s > 0.0 )
      P = p->p_atm/(R*R*sR) + K*s*s*(1.0 + p->amp*disco_hash_unit3(p->seed, r, phi, z, p->phimax));
   const double rho = p->rho_atm/(R*sR) + s;
   const double sM = sqrt(p->M);
   const double uphi = s*r*r*sM/(R*sR + p->a*sM);
   const double ur = -(1.0 - s)*sqrt(p->M/(2.0*R));
   const double uz = ur*z/R;
   /* the loop field: A = s - s_cut inside, dA = ds = -2 (1 - d2) dd2 */
   double Br = 0.0, Bz = 0.0;
   if( s > p->s_cut && d2 < 1.0 ){
      const double B0 = sqrt(2.0*K/p->beta)*p->wr*0.5;
      const double A = s - p->s_cut;
      /* d(d2)/dR = 2 dR / wr + 2 zh * (-z/(hr R^2)); d(zh)/dz at fixed R part */
      const double dd2_dR = 2.0*dR/p->wr - 2.0*zh*z/(p->hr*R*R);
      const double dd2_dr = dd2_dR*r/R;
      const double dd2_dz = dd2_dR*z/R + 2.0*zh/(p->hr*R);
      const double ds_dr = -2.0*one_m*dd2_dr;
      const double ds_dz = -2.0*one_m*dd2_dz;
      Br = -B0*ds_dz;
      Bz = B0*(A/r + ds_dr);
   }
   prim[0] = rho;
   prim[1] = P;
   prim[2] = ur;
   prim[3] = uphi;
   prim[4] = uz;
   int q;
   for( q=5 ; q<num_c ; ++q ) prim[q] = 0.0;
   if( num_c >= 8 ){ prim[5] = Br; prim[6] = 0.0; prim[7] = Bz; }
   if( num_q > num_c ){
      prim[num_c] = s;
      for( q=num_c+1 ; q<num_q ; ++q ) prim[q] = 0.0;
   }
}

#endif
