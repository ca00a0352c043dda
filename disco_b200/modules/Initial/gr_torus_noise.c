/*
 * Disco Initial module `gr_torus_noise`: a GRMHD torus with a poloidal loop
 * field, a thin infalling atmosphere and seeded, hash-based pressure noise,
 * for the grmhd2 Hydro module.  Drop this file into a Disco tree's Initial/
 * directory and select it with `INITIAL = gr_torus_noise` in
 * Makefile_opt.in.  It follows the Initial-module contract of the reference
 * (setICparams/initial, e.g. Initial/kepler.c:9-37) and evaluates exactly
 * the same function as the device boundary kernels (ic_gr_torus.h).
 *
 * Compile with -I<disco tree> -I<this repo>/disco_b200/csrc.
 */
#include "paul.h"
#include "ic_gr_torus.h"

static disco_ic_gr_torus icp;

void setICparams( struct domain * theDomain ){
   const struct param_list *L = &theDomain->theParList;
   icp.seed    = (uint64_t)(int64_t)L->initPar0;
   icp.amp     = L->initPar1;
   icp.rc      = L->initPar2;
   icp.wr      = L->initPar3;
   icp.hr      = L->initPar4;
   icp.beta    = L->initPar5;
   icp.rho_atm = L->initPar6;
   icp.p_atm   = L->initPar7;
   icp.s_cut   = L->initPar8;
   icp.M       = L->metricPar2;
   icp.a       = L->metricPar3;
   icp.rmin    = L->rmin;
   icp.rmax    = L->rmax;
   icp.zmin    = L->zmin;
   icp.zmax    = L->zmax;
   icp.phimax  = L->phimax;
}

void initial( double * prim , double * x ){
   disco_ic_gr_torus_eval( &icp , NUM_C , NUM_Q , prim , x );
}
