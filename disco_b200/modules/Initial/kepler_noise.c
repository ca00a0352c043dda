/*
 * Disco Initial module `kepler_noise`: a Keplerian disk with seeded,
 * hash-based density noise.  Drop this file into a Disco tree's Initial/
 * directory and select it with `INITIAL = kepler_noise` in Makefile_opt.in.
 * It follows the Initial-module contract of the reference
 * (setICparams/initial, e.g. Initial/kepler.c:9-37) and evaluates exactly
 * the same function as the device boundary kernels (ic_kepler_noise.h).
 *
 * Compile with -I<disco tree> -I<this repo>/disco_b200/csrc.
 */
#include "paul.h"
#include "ic_kepler_noise.h"

static disco_ic_kepler_noise icp;

void setICparams( struct domain * theDomain ){
   icp.mach   = theDomain->theParList.Disk_Mach;
   icp.amp    = theDomain->theParList.initPar1;
   icp.rmin   = theDomain->theParList.rmin;
   icp.rmax   = theDomain->theParList.rmax;
   icp.phimax = theDomain->theParList.phimax;
   icp.seed   = (uint64_t)(int64_t)theDomain->theParList.initPar0;
   icp.kind   = (int)theDomain->theParList.initPar2;
}

void initial( double * prim , double * x ){
   disco_ic_kepler_noise_eval( &icp , NUM_C , NUM_Q , prim , x );
}
