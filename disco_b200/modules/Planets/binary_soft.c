/*
 * Disco Planets module `binary_soft`: an equal-mass binary on a circular
 * orbit of separation 1 about the origin, each star softened by Init_Par8
 * (the circumbinary configuration's potential).  Drop this file into a
 * Disco tree's Planets/ directory and select it with `PLANETS =
 * binary_soft` in Makefile_opt.in.  It follows the Planets-module contract
 * of the reference (setPlanetParams / planet_motion_analytic /
 * initializePlanets / movePlanets / forcePlanets, e.g. Planets/cm2.c) and
 * sets the same planets as the device's set-up (disco_batch.cu,
 * init_planets): masses 1/2, radii 1/2, phases pi and 0, Omega = a^-3/2.
 * Init_Par8 carries the softening because Init_Par5-7 belong to the disk's
 * Initial module (mhd_shear_noise).
 */
#include "paul.h"

static double eps_soft = 0.0;

void setPlanetParams( struct domain * theDomain ){
   theDomain->Npl = 2;
   eps_soft = theDomain->theParList.initPar8;
}

int planet_motion_analytic( void ){
   return(1);
}

void initializePlanets( struct planet * thePlanets ){
   double a = 1.0;
   double om = 1.0/(a*sqrt(a));
   int p;
   for( p=0 ; p<2 ; ++p ){
      thePlanets[p].M     = 0.5;
      thePlanets[p].vr    = 0.0;
      thePlanets[p].omega = om;
      thePlanets[p].r     = 0.5*a;
      thePlanets[p].eps   = eps_soft;
      thePlanets[p].type  = PLPOINTMASS;
   }
   thePlanets[0].phi = M_PI;
   thePlanets[1].phi = 0.0;
}

void movePlanets( struct planet * thePlanets , double t , double dt ){
   thePlanets[0].phi += thePlanets[0].omega*dt;
   thePlanets[1].phi += thePlanets[1].omega*dt;
}

void forcePlanets( struct planet * thePlanets , double dt ){
}
