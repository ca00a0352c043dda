/*
 * Disco Initial module `mhd_shear_noise`: a magnetised Keplerian shearing
 * disk (vertical field of plasma beta Init_Par4, sound speed Init_Par3;
 * optional toroidal field of beta Init_Par5 and radial field of amplitude
 * Init_Par6) with seeded, hash-based velocity noise of amplitude
 * Init_Par1 * cs.  Drop this
 * file into a Disco tree's Initial/ directory and select it with
 * `INITIAL = mhd_shear_noise`; it follows the Initial-module contract
 * (setICparams/initial, e.g. Initial/flock.c) and evaluates the same
 * function as the device set-up and boundary kernels (ic_mhd_shear.h).
 *
 * Compile with -I<disco tree> -I<this repo>/disco_b200/csrc.
 */
#include "paul.h"
#include "ic_mhd_shear.h"

static disco_ic_mhd_shear icp;

void setICparams( struct domain * theDomain ){
   icp.seed   = (uint64_t)(int64_t)theDomain->theParList.initPar0;
   icp.amp    = theDomain->theParList.initPar1;
   icp.cs     = theDomain->theParList.initPar3;
   icp.beta   = theDomain->theParList.initPar4;
   icp.beta_phi = theDomain->theParList.initPar5;
   icp.b_r    = theDomain->theParList.initPar6;
   icp.gam    = theDomain->theParList.Adiabatic_Index;
   icp.rmin   = theDomain->theParList.rmin;
   icp.rmax   = theDomain->theParList.rmax;
   icp.zmin   = theDomain->theParList.zmin;
   icp.zmax   = theDomain->theParList.zmax;
   icp.phimax = theDomain->theParList.phimax;
   icp.kind   = (int)theDomain->theParList.initPar2;
}

void initial( double * prim , double * x ){
   disco_ic_mhd_shear_eval( &icp , NUM_C , NUM_Q , prim , x );
}
