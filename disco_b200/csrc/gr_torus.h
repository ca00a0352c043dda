/*
 * GRMHD torus state: a new Initial-style module (the reference has no torus
 * IC for grmhd2), shared by the device code and the CPU oracle so both build
 * the same cell states.  It stands in for a Fishbone-Moncrief torus in
 * Kerr-Schild coordinates with the qualitative features the cons->prim solve
 * sees (a dense, hot, rotating torus with a poloidal loop field inside a thin
 * infalling atmosphere), not an exact equilibrium:
 *
 *   R = sqrt(r^2+z^2),  s = exp(-((R-rc)/wr)^2 - (z/(hr R))^2)
 *   rho = rho_atm R^-3/2 + s
 *   P   = p_atm R^-5/2 + K s^gam (1 + amp u),  u in [-1,1) hashed per cell
 *   u_phi = s r^2 sqrt(M)/(R^3/2 + a sqrt(M))     (covariant, prograde)
 *   u_r = -(1-s) sqrt(M/(2R)),  u_z = u_r z/R     (atmosphere infall)
 *   A_phi = B0 (s - s_cut) for s > s_cut:  B^r = -dA/dz, B^z = dA/dr
 *   X = s (passive)
 *
 * The perturbation gr_perturb multiplies every primitive by (1 + eps u_q),
 * u_q hashed from (seed, cell, q): one step's change of a run, with eps
 * setting how far the previous prims (the Newton warm start) lie from the
 * solution.  Only +, -, *, /, sqrt and exp appear; the hash is integer.
 */
#pragma once
#include <stdint.h>
#include <math.h>

#ifdef __CUDACC__
#define GRT_HD __host__ __device__ __forceinline__
#else
#define GRT_HD static inline
#endif

typedef struct gr_torus_par {
   double M, a, gam;
   double rc, wr, hr, K;
   double rho_atm, p_atm, B0, s_cut, amp;
   uint64_t seed;
} gr_torus_par;

GRT_HD uint64_t grt_mix(uint64_t z){
   z += 0x9e3779b97f4a7c15ULL;
   z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
   z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
   return z ^ (z >> 31);
}

/* uniform in [-1, 1) from 53 hashed bits */
GRT_HD double grt_unit(uint64_t seed, uint64_t cell, uint64_t q){
   uint64_t h = grt_mix(seed ^ grt_mix(cell * 16 + q));
   return (double)(h >> 11) * (1.0/4503599627370496.0) - 1.0;
}

/* prim layout: RHO 0, PPP 1, URR 2, UPP 3, UZZ 4, BRR 5, BPP 6, BZZ 7, X 8 */
GRT_HD void gr_torus_prim(const gr_torus_par *tp, const double *x, uint64_t cell, double *prim){
   double r = x[0], z = x[2];
   double R = sqrt(r*r + z*z);
   double dR = (R - tp->rc)/tp->wr;
   double zh = z/(tp->hr*R);
   double s = exp(-dR*dR - zh*zh);
   double sR = 1.0/sqrt(R);
   double rho = tp->rho_atm*sR*sR*sR + s;
   double Ps = tp->K*exp(tp->gam*log(s > 1e-300 ? s : 1e-300));
   double P = tp->p_atm*sR*sR*sR*sR*sR + Ps*(1.0 + tp->amp*grt_unit(tp->seed, cell, 0));
   double sM = sqrt(tp->M);
   double uphi = s*r*r*sM/(R*sqrt(R) + tp->a*sM);
   double ur = -(1.0 - s)*sqrt(tp->M/(2.0*R));
   double uz = ur*z/R;
   /* dq/dr and dq/dz of q = -dR^2 - zh^2 */
   double dqdR = -2.0*dR/tp->wr + 2.0*zh*zh/R;
   double dqdr = dqdR*r/R;
   double dqdz = dqdR*z/R - 2.0*zh/(tp->hr*R);
   double Br = 0.0, Bz = 0.0;
   if( s > tp->s_cut ){
      Br = -tp->B0*s*dqdz;
      Bz =  tp->B0*s*dqdr;
   }
   prim[0] = rho; prim[1] = P;
   prim[2] = ur; prim[3] = uphi; prim[4] = uz;
   prim[5] = Br; prim[6] = 0.0; prim[7] = Bz;
   prim[8] = s;
}

GRT_HD void gr_perturb(const double *prim, double *out, uint64_t seed, uint64_t cell, double eps){
   int q;
   for( q=0 ; q<9 ; ++q ) out[q] = prim[q]*(1.0 + eps*grt_unit(seed, cell, (uint64_t)q + 1));
}
