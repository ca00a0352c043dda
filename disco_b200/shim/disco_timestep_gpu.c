/*
 * Drop-in replacement of Disco's timestep() and getmindt() for the serial
 * (USE_MPI=0) build, running the step on a B200 through the disco_b200 C ABI.
 *
 * It is compiled inside a Disco tree (it includes the tree's paul.h and
 * sees the Makefile's -DHYDRO=... -DNUM_C=... definitions) and replaces, at
 * link time:
 *     void   timestep( struct domain * , double )   timestep.c:7-45
 *     double getmindt( struct domain * )            misc.c:39-84
 * main.c's loop (main.c:69-83) is unchanged.  disco_gpu_init(), called once
 * after setupCells (main.c:47-62), uploads the domain (cells, grid,
 * parameters) to the GPU and returns a status, so a host can catch a module
 * selection the device does not run, or a CUDA error, before its loop; a
 * host that does not call it gets the same upload from the first getmindt()
 * or timestep(), which then exits on error.  Afterwards the state stays on
 * the device and struct domain's cells and planets are stale until
 * disco_gpu_sync_to_host() copies them back (call it before output, e.g. at
 * the top of possiblyOutput, domain.c:317; report() is replaced here and
 * needs no copy).  The first call also uploads the domain's planets, so a
 * run restarted by the reference's own restart() (h5in.c) continues from
 * the checkpoint's planets.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "paul.h"
#include "disco_b200.h"

static disco_batch *g_batch = NULL;

static int module_id(const char *name, const char *const *names, int n){
   int i;
   for( i=0 ; i<n ; ++i ) if( strcmp(name, names[i]) == 0 ) return i;
   return -1;
}

static void fill_params(const struct domain *d, disco_params *p){
   const struct param_list *L = &d->theParList;
   memset(p, 0, sizeof *p);
   p->Num_R = L->Num_R; p->Num_Z = L->Num_Z; p->aspect = L->aspect;
   p->rmin = L->rmin; p->rmax = L->rmax; p->zmin = L->zmin; p->zmax = L->zmax;
   p->phimax = L->phimax;
   p->NoBC_Rmin = L->NoBC_Rmin; p->NoBC_Rmax = L->NoBC_Rmax;
   p->NoBC_Zmin = L->NoBC_Zmin; p->NoBC_Zmax = L->NoBC_Zmax;
   p->LogZoning = L->LogZoning; p->R_Periodic = L->R_Periodic; p->Z_Periodic = L->Z_Periodic;
   p->LogRadius = L->LogRadius;
   p->Mesh_Motion = L->Mesh_Motion; p->Riemann_Solver = L->Riemann_Solver;
   p->Timestep = L->Timestep;
   p->CFL = L->CFL; p->PLM = L->PLM; p->maxDT = L->maxDT;
   p->Density_Floor = L->Density_Floor; p->Pressure_Floor = L->Pressure_Floor;
   p->Exact_Mesh_Omega = L->Exact_Mesh_Omega; p->Exact_Mesh_Omega_Par = L->Exact_Mesh_Omega_Par;
   p->Energy_Omega = L->Energy_Omega; p->Energy_Omega_Par = L->Energy_Omega_Par;
   p->RotFrame = L->RotFrame; p->RotOmega = L->RotOmega; p->RotD = L->RotD;
   p->Adiabatic_Index = L->Adiabatic_Index; p->viscosity = L->viscosity;
   p->visc_flag = L->visc_flag; p->alpha_flag = L->alpha_flag;
   p->isothermal_flag = L->isothermal_flag; p->Cs2_Profile = L->Cs2_Profile; p->Cs2_Par = L->Cs2_Par;
   p->Disk_Mach = L->Disk_Mach; p->Mass_Ratio = L->Mass_Ratio; p->grav2D = L->grav2D;
   p->CT = L->CT;
   p->initPar0 = L->initPar0;
   p->initPar[1] = L->initPar1; p->initPar[2] = L->initPar2; p->initPar[3] = L->initPar3;
   p->initPar[4] = L->initPar4; p->initPar[5] = L->initPar5; p->initPar[6] = L->initPar6;
   p->initPar[7] = L->initPar7; p->initPar[8] = L->initPar8;
   p->metricPar[1] = L->metricPar1; p->metricPar[2] = L->metricPar2;
   p->metricPar[3] = L->metricPar3; p->metricPar[4] = L->metricPar4;
   p->t_min = d->t;
   p->include_atmos = L->include_atmos;
   p->noiseType = L->noiseType; p->noiseAbs = L->noiseAbs; p->noiseRel = L->noiseRel;
}

static void fail(const char *what, int s){
   fprintf(stderr, "disco_b200 shim: %s: %s\n", what, disco_strerror(s));
   exit(1);
}

static void report_err(const char *what, int s){
   fprintf(stderr, "disco_b200 shim: %s: %s\n", what, disco_strerror(s));
}

/* Upload the domain after setupCells; returns DISCO_OK or the status of the
 * step that failed (the batch is then released).  The module selection is
 * checked first: a Hydro / Boundary / Planets module the device does not
 * run, and an Analysis module whose diagnostics it does not compute
 * (analysis.c:52-107 would fill theTools.Qrz every step), are refused with
 * DISCO_ERR_UNSUPPORTED rather than run without them.  Calling it again
 * re-uploads the domain. */
int disco_gpu_init( const struct domain * d ){
   static const char *const hydros[] = {"euler", "mhd", "grmhd2"};
   static const char *const bcs[] = {"fixed", "zerograd", "fixed3d", "polar", "outflow3d",
                                     "zerograd_omk", "accrete3d", "polar3d", "horizon",
                                     "horizon3d", "horizon_bin", "fixRrefZ", "tube",
                                     "surfaceGravBox", "fixed_gap", "flowthrough"};
   static const char *const pls[] = {"none", "sun", "cm2", "binary_soft", "circular", "cm"};
   static const char *const ics[] = {"kepler_noise", "mhd_shear_noise", "gr_torus_noise"};
   static const int ic_ids[] = {DISCO_IC_KEPLER_NOISE, DISCO_IC_MHD_SHEAR_NOISE, DISCO_IC_GR_TORUS_NOISE};
   static const char *const metrics[] = {"schw_ks_rpz", "kerr_ks_rpz"};
   static const char *const diags[] = {"diag_disk2d", "diag_euler", "diag_mhdmri"};
   static const int diag_ids[] = {DISCO_DIAG_DISK2D, DISCO_DIAG_EULER, DISCO_DIAG_MHDMRI};
   if( !d ) return DISCO_ERR_ARG;
   if( g_batch ){ disco_batch_destroy(g_batch); g_batch = NULL; }
   disco_modules m;
   memset(&m, 0, sizeof m);
   m.hydro = module_id(HYDRO, hydros, 3);
   m.boundary = module_id(BOUNDARY, bcs, 16);
   m.planets = module_id(PLANETS, pls, 6);
   int ii = module_id(INITIAL, ics, 3);
   m.initial = ii >= 0 ? ic_ids[ii] : -1;
   m.metric = module_id(METRIC, metrics, 2);
   if( m.hydro == DISCO_HYDRO_GRMHD && (m.metric < 0 || strcmp(FRAME, "normal") != 0) )
      return DISCO_ERR_UNSUPPORTED;
   if( m.metric < 0 ) m.metric = DISCO_METRIC_SCHW_KS_RPZ;     /* not read without grmhd2 */
   /* any other Initial module: setupCells evaluated it here on the host, and
    * boundaries that do not call it again (zerograd, outflow3d) run as is */
   if( m.initial < 0 ) m.initial = DISCO_IC_HOST;
   int ia = module_id(ANALYSIS, diags, 3);
   m.analysis = ia >= 0 ? diag_ids[ia] : DISCO_DIAG_NONE;
   m.num_c = NUM_C; m.num_n = NUM_N; m.ct_mode = CT_MODE;
   if( m.hydro < 0 || m.boundary < 0 || m.planets < 0 || m.initial < 0 ) return DISCO_ERR_UNSUPPORTED;
   if( ia < 0 && d->num_tools > 0 ) return DISCO_ERR_UNSUPPORTED;
   disco_params p;
   fill_params(d, &p);
   int Nr = d->Nr, Nz = d->Nz, jk, i, q;
   int Ng[4] = {d->NgRa, d->NgRb, d->NgZa, d->NgZb};
   int s = disco_batch_create(0, &m, DISCO_PREC_FP64, 1, &p, &Nr, &Nz, Ng, d->Np,
                              d->r_jph - 1, d->z_kph - 1, &g_batch);
   if( s ){ g_batch = NULL; return s; }
   int64_t ncell;
   disco_batch_sizes(g_batch, &ncell, NULL, NULL);
   double *prim = malloc(sizeof(double)*NUM_Q*ncell), *cons = malloc(sizeof(double)*NUM_Q*ncell);
   double *piph = malloc(sizeof(double)*ncell), *dphi = malloc(sizeof(double)*ncell);
   double *wiph = malloc(sizeof(double)*ncell);
   int *real = malloc(sizeof(int)*ncell);
   /* the constrained-transport face fluxes, cell->Phi[NUM_FACES] */
   double *phis = NUM_FACES > 0 && d->theParList.CT ? malloc(sizeof(double)*(NUM_FACES > 0 ? NUM_FACES : 1)*ncell) : NULL;
   if( !prim || !cons || !piph || !dphi || !wiph || !real || (NUM_FACES > 0 && d->theParList.CT && !phis) ){
      free(prim); free(cons); free(piph); free(dphi); free(wiph); free(real); free(phis);
      disco_batch_destroy(g_batch); g_batch = NULL;
      return DISCO_ERR_ARG;
   }
   int64_t n = 0;
   for( jk=0 ; jk<Nr*Nz ; ++jk ) for( i=0 ; i<d->Np[jk] ; ++i, ++n ){
      const struct cell *c = &d->theCells[jk][i];
      for( q=0 ; q<NUM_Q ; ++q ){ prim[NUM_Q*n+q] = c->prim[q]; cons[NUM_Q*n+q] = c->cons[q]; }
      piph[n] = c->piph; dphi[n] = c->dphi; wiph[n] = c->wiph; real[n] = c->real;
      if( phis ) for( q=0 ; q<NUM_FACES ; ++q ) phis[NUM_FACES*n+q] = c->Phi[q];
   }
   s = disco_batch_set_cells(g_batch, prim, cons, piph, dphi, wiph, real, phis);
   free(prim); free(cons); free(piph); free(dphi); free(wiph); free(real); free(phis);
   if( s ){ disco_batch_destroy(g_batch); g_batch = NULL; return s; }
   /* the planets as the host domain holds them: a restart reads them from
    * the checkpoint (h5in.c:291-318), not from initializePlanets */
   double *pl = malloc(sizeof(double)*DISCO_PLANET_COLS*(d->Npl > 0 ? d->Npl : 1));
   if( !pl ){ disco_batch_destroy(g_batch); g_batch = NULL; return DISCO_ERR_ARG; }
   int ip;
   for( ip=0 ; ip<d->Npl ; ++ip ){
      const struct planet *P = d->thePlanets + ip;
      double *r = pl + DISCO_PLANET_COLS*ip;
      r[0] = P->M; r[1] = P->vr; r[2] = P->omega; r[3] = P->r; r[4] = P->phi; r[5] = P->eps;
      r[6] = (double)P->type;
   }
   s = disco_batch_set_planets(g_batch, 0, pl, d->Npl);
   free(pl);
   if( s ){ disco_batch_destroy(g_batch); g_batch = NULL; return s; }
   return DISCO_OK;
}

/* the implicit upload of a host that did not call disco_gpu_init() */
static void gpu_init(struct domain *d){
   int s = disco_gpu_init(d);
   if( s ){ report_err("disco_gpu_init", s); exit(1); }
}

/* getmindt replacement (misc.c:39-84): the device min-reduction. */
double getmindt( struct domain * theDomain ){
   if( !g_batch ) gpu_init(theDomain);
   double dt = 0.0;
   int s = disco_batch_mindt(g_batch, &dt);
   if( s ) fail("disco_batch_mindt", s);
   return dt;
}

/* timestep replacement (timestep.c:7-45). */
void timestep( struct domain * theDomain , double dt ){
   if( !g_batch ) gpu_init(theDomain);
   int s = disco_batch_timestep(g_batch, &dt);
   if( s ) fail("disco_batch_timestep", s);
   theDomain->t += dt;
   theDomain->count_steps += 1;
}

/* report replacement (report.c:7-202): the line is computed on the device
 * from the resident state and appended to report.dat in the reference's
 * format, so a report needs no copy of the cells. */
void report( struct domain * theDomain ){
   if( !g_batch ) gpu_init(theDomain);
   double v[17];
   int s = disco_batch_report(g_batch, 0, v);
   if( s ) fail("disco_batch_report", s);
   if( theDomain->rank == 0 ){
      FILE *rFile = fopen("report.dat", "a");
      if( !rFile ) return;
      fprintf(rFile, "%le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le %le\n",
              v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10],
              v[11], v[12], v[13], v[14], v[15], v[16]);
      fclose(rFile);
   }
}

/* Copy the device state back into struct domain's cells (before output). */
void disco_gpu_sync_to_host( struct domain * theDomain ){
   if( !g_batch ) return;
   int64_t ncell;
   disco_batch_sizes(g_batch, &ncell, NULL, NULL);
   double *prim = malloc(sizeof(double)*NUM_Q*ncell), *cons = malloc(sizeof(double)*NUM_Q*ncell);
   double *piph = malloc(sizeof(double)*ncell), *dphi = malloc(sizeof(double)*ncell);
   double *wiph = malloc(sizeof(double)*ncell);
   double *phis = NUM_FACES > 0 && theDomain->theParList.CT ? malloc(sizeof(double)*(NUM_FACES > 0 ? NUM_FACES : 1)*ncell) : NULL;
   int s = disco_batch_get_cells(g_batch, prim, cons, piph, dphi, wiph, phis);
   if( s ) fail("disco_batch_get_cells", s);
   s = disco_batch_last_error(g_batch);
   if( s ) fail("device step", s);
   int jk, i, q;
   int64_t n = 0;
   for( jk=0 ; jk<theDomain->Nr*theDomain->Nz ; ++jk ) for( i=0 ; i<theDomain->Np[jk] ; ++i, ++n ){
      struct cell *c = &theDomain->theCells[jk][i];
      for( q=0 ; q<NUM_Q ; ++q ){ c->prim[q] = prim[NUM_Q*n+q]; c->cons[q] = cons[NUM_Q*n+q]; }
      c->piph = piph[n]; c->dphi = dphi[n]; c->wiph = wiph[n];
      if( phis ) for( q=0 ; q<NUM_FACES ; ++q ) c->Phi[q] = phis[NUM_FACES*n+q];
   }
   free(prim); free(cons); free(piph); free(dphi); free(wiph); free(phis);
   /* the planets, moved on the device (planet data of a checkpoint) */
   double *pl = malloc(sizeof(double)*DISCO_PLANET_COLS*(theDomain->Npl > 0 ? theDomain->Npl : 1));
   int npl = 0;
   if( disco_batch_get_planets(g_batch, 0, pl, theDomain->Npl, &npl) == DISCO_OK && npl == theDomain->Npl ){
      int p;
      for( p=0 ; p<npl ; ++p ){
         struct planet *P = theDomain->thePlanets + p;
         const double *r = pl + DISCO_PLANET_COLS*p;
         P->M = r[0]; P->vr = r[1]; P->omega = r[2]; P->r = r[3]; P->phi = r[4]; P->eps = r[5];
      }
   }
   free(pl);
   /* time-averaged diagnostics accumulated on the device (analysis.c:52-107) */
   int nq = 0;
   double tavg = 0.0;
   if( theDomain->num_tools > 0 &&
       disco_batch_get_diagnostics(g_batch, 0, theDomain->theTools.Qrz, &nq, &tavg) == DISCO_OK )
      theDomain->theTools.t_avg = tavg;
}

/* The rest of the drop-in's surface: the face lists of the resident state
 * (for a bit-exact comparison with the reference's buildfaces: fIndex has
 * N_ftracks+1 entries, iL / iR cell indices in annulus order, LR the
 * LRtype; any pointer may be NULL, *nfaces receives the count), the
 * device error word since the last call, and releasing the device state. */
int disco_gpu_get_faces( struct domain * theDomain , int dim , int *nfaces ,
                         int *fIndex , int *iL , int *iR , int *LR ){
   if( !g_batch ) gpu_init(theDomain);
   return disco_batch_get_faces(g_batch, 0, dim, nfaces, fIndex, iL, iR, LR, NULL);
}

int disco_gpu_last_error( void ){
   return g_batch ? disco_batch_last_error(g_batch) : DISCO_OK;
}

void disco_gpu_free( void ){
   if( g_batch ) disco_batch_destroy(g_batch);
   g_batch = NULL;
}
