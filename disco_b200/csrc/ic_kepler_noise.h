/*
 * Keplerian disk with seeded, hash-based density noise.
 *
 * A new initial-condition module (the reference has no density-noise IC:
 * its Noise_Type options perturb only velocities or pressure, noise.c:17-49,
 * and they draw from glibc rand() in cell order, which cannot be evaluated
 * per cell on a device).  The noise here is a pure function of the cell
 * position, so the host build and the device boundary kernels give the same
 * value for the same x, and re-evaluating initial() (as the `fixed` boundary
 * does every substep, Boundary/fixed.c:11-60) is idempotent.
 *
 *   Sigma = 1 * (1 + amp * u),  u in [-1,1) hashed from (seed, r, phi)
 *   Omega = r^-3/2,  v_r = v_z = 0
 *   P     = Sigma * (v_phi / Mach)^2 ,  v_phi = r^-1/2
 *   X     = 4 (phi/Pmax)(1 - phi/Pmax)          (passive scalar, NUM_N>0)
 *
 * With Init_Par2 = 1 the disk instead rotates rigidly (Omega = 1) and is
 * held by pressure, P = 1/Mach^2 + r^2/2, with no gravity needed: run with
 * PLANETS = none and Energy_Omega 0, a step then calls no libm function
 * whose value matters, which makes a CPU and a GPU build comparable bit for
 * bit.
 *
 * Noise is applied only inside [rmin, rmax]: ghost annuli lie outside, so
 * their boundary values stay a smooth function of x and cannot flip a hash
 * bucket when a ghost cell's phi differs by an ulp between two builds.
 *
 * Everything uses +,-,*,/ and sqrt only (all correctly rounded in IEEE-754
 * double on both gcc/x86-64 and CUDA), so host and device values are
 * bit-identical for bit-identical x.
 *
 * Parameters (in.par): Mach_Number, Init_Par0 = seed, Init_Par1 = amp,
 * R_Min / R_Max, Phi_Max.
 */
#ifndef DISCO_IC_KEPLER_NOISE_H
#define DISCO_IC_KEPLER_NOISE_H

#ifdef __CUDACC__
#define DISCO_HD __host__ __device__ __forceinline__
#else
#define DISCO_HD static inline
#endif

#include <stdint.h>
#ifndef __CUDACC__
#include <math.h>
#endif

typedef struct {
   double mach;
   double amp;
   double rmin, rmax;
   double phimax;
   uint64_t seed;
   int kind;          /* Init_Par2: 0 Keplerian, 1 rigid rotation held by pressure */
   int pad;
} disco_ic_kepler_noise;

/* splitmix64 finaliser (Steele, Lea & Flood 2014). */
DISCO_HD uint64_t disco_mix64(uint64_t z){
   z += 0x9E3779B97F4A7C15ull;
   z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
   z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
   return z ^ (z >> 31);
}

/* Uniform in [-1,1) from the seed and the cell position.  r and phi are
 * bucketed at 2^-20 and Pmax*2^-24 so that the value is a function of the
 * cell, not of the last bit of its centroid. */
DISCO_HD double disco_hash_unit(uint64_t seed, double r, double phi, double phimax){
   int64_t qr = (int64_t)(r * 1048576.0);
   int64_t qp = (int64_t)((phi / phimax) * 16777216.0);
   uint64_t h = disco_mix64(seed ^ disco_mix64((uint64_t)qr * 0x100000001B3ull
                                               ^ ((uint64_t)qp << 1)));
   double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
   return 2.0 * u - 1.0;
}

/* prim layout: RHO, PPP, URR, UPP, UZZ, [BRR, BPP, BZZ], passive... */
DISCO_HD void disco_ic_kepler_noise_eval(const disco_ic_kepler_noise *p,
                                         int num_c, int num_q,
                                         double *prim, const double *x){
   double r = x[0];
   double phi = x[1];
   double sig = 1.0;
   if( r >= p->rmin && r <= p->rmax && p->amp != 0.0 )
      sig = 1.0 * (1.0 + p->amp * disco_hash_unit(p->seed, r, phi, p->phimax));
   double omega, press;
   if( p->kind == 1 ){
      /* rigid rotation Omega = 1 balanced by a pressure gradient,
       * dP/dr = rho Omega^2 r with rho = 1: P = 1/Mach^2 + r^2/2 (no gravity) */
      omega = 1.0;
      press = 1.0 / (p->mach * p->mach) + 0.5 * r * r;
   }else{
      double sr = sqrt(r);
      double vphi = 1.0 / sr;
      double cs = vphi / p->mach;
      omega = 1.0 / (r * sr);
      press = sig * cs * cs;
   }
   prim[0] = sig;
   prim[1] = press;
   prim[2] = 0.0;
   prim[3] = omega;
   prim[4] = 0.0;
   int q;
   for( q=5 ; q<num_c ; ++q ) prim[q] = 0.0;
   if( num_q > num_c ){
      double s = phi / p->phimax;
      prim[num_c] = 4.0 * s * (1.0 - s);
      for( q=num_c+1 ; q<num_q ; ++q ) prim[q] = 0.0;
   }
}

#endif
