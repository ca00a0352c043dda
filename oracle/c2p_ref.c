/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * Thin C entry points around the reference's own GRMHD state conversions,
 * Hydro/grmhd2.c prim2cons (:88-180) and cons2prim (:253-270, Noble 2D
 * Newton :1096-1313), with the Schwarzschild Kerr-Schild cylindrical metric
 * (Hydro/Metric/schw_ks_rpz.c) and the normal-observer frame
 * (Hydro/Frame/normal.c), all compiled unmodified from their sources by
 * oracle/Makefile (target c2p) into oracle/_ref/c2p/libc2p_ref.so.
 * Q = NUM_C 8 + NUM_N 1 = 9 values per state.
 */
#include "paul.h"

void setHydroParams( struct domain * );
void setMetricParams( struct domain * );
void prim2cons( const double *prim, double *cons, const double *x, double dV );
void cons2prim( const double *cons, double *prim, const double *x, double dV );

static struct domain g_dom;

void ref_c2p_setup(double gamma_law, double rho_floor, double p_floor, double M){
   memset(&g_dom, 0, sizeof g_dom);
   g_dom.theParList.Adiabatic_Index = gamma_law;
   g_dom.theParList.Density_Floor = rho_floor;
   g_dom.theParList.Pressure_Floor = p_floor;
   g_dom.theParList.metricPar2 = M;
   setHydroParams(&g_dom);
   setMetricParams(&g_dom);
}

/* n states: prim[9n], x[3n] -> cons[9n] (per unit volume, dV = 1) */
void ref_prim2cons(int n, const double *prim, const double *x, double *cons){
   int i;
   for( i=0 ; i<n ; ++i ) prim2cons(prim + 9*i, cons + 9*i, x + 3*i, 1.0);
}

/* n states: cons[9n], x[3n]; prim[9n] holds the initial guess (the previous
 * prims, as in the reference) and receives the solution */
void ref_cons2prim(int n, const double *cons, const double *x, double *prim){
   int i;
   for( i=0 ; i<n ; ++i ) cons2prim(cons + 9*i, prim + 9*i, x + 3*i, 1.0);
}
