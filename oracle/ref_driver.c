/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * Fixed-step driver linked against the reference Disco objects compiled
 * unmodified from their own sources (see oracle/Makefile).  The reference
 * has no step-count limit (its loop runs to T_End, main.c:69-83), so parity
 * "after N steps" needs this driver.  It repeats main.c's setup sequence
 * (main.c:31-62) and then runs  getmindt + timestep  N times
 * (main.c:72-81), without check_dt / possiblyOutput (no I/O in the loop).
 *
 * usage:  disco_ref RUNDIR NSTEPS [DUMPDIR]      dump state after N steps
 *         disco_ref RUNDIR NSTEPS --time          print wall-time JSON only
 * environment: DISCO_REF_REPORT (report.dat line), DISCO_REF_ASCII=<filestart>
 * (ascii output of the final state), DISCO_REF_CHECKPOINT=<dir> (checkpoint
 * datasets as raw files), DISCO_REF_RESTART=<dir> (with Restart 1 in in.par:
 * start from such a checkpoint)
 *
 * RUNDIR must hold in.par (read_par_file reads "in.par" from the CWD,
 * readpar.c:62).  Dumps are raw little-endian arrays, one file each,
 * cells in annulus order jk = j + Nr*k, i = 0..Np[jk]-1.
 */
#include "paul.h"
#include "profiler.h"
#include <sys/stat.h>
#include <sys/time.h>
#include <unistd.h>

int mpiSetup( struct domain * , int , char *[] );
void setupGrid( struct domain * );
void setupDomain( struct domain * );
void setupCells( struct domain * );
void timestep( struct domain * , double );
void boundary_trans( struct domain * , int );
void exchangeData( struct domain * , int );
double getmindt( struct domain * );
void report( struct domain * );
int read_par_file( struct domain * );
void setup_faces( struct domain * , int );
void freeDomain( struct domain * );
/* Present only when this driver is linked with the GPU drop-in
 * (disco_b200/shim): copies the device state back into the cells. */
void disco_gpu_sync_to_host( struct domain * ) __attribute__((weak));
int disco_gpu_init( const struct domain * ) __attribute__((weak));
int disco_gpu_get_faces( struct domain * , int , int * , int * , int * , int * , int * ) __attribute__((weak));
int disco_gpu_last_error( void ) __attribute__((weak));
void disco_gpu_free( void ) __attribute__((weak));
/* oracle/ref_checkpoint.c: h5out.c's datasets as raw files */
void disco_ref_checkpoint( struct domain * , const char * );
/* the output module (Output/ascii.c in the oracle build) */
void output( struct domain * , char * );

static double wall(void){
   struct timeval tv; gettimeofday(&tv, NULL);
   return tv.tv_sec + 1e-6*tv.tv_usec;
}

static void dump(const char *dir, const char *name, const void *p, size_t nbytes){
   char fn[4200];
   snprintf(fn, sizeof fn, "%s/%s", dir, name);
   FILE *f = fopen(fn, "wb");
   if(!f){ fprintf(stderr, "cannot write %s\n", fn); exit(2); }
   fwrite(p, 1, nbytes, f);
   fclose(f);
}

static void dump_faces(struct domain *d, int dim, const char *dir, int *cell_off){
   int Nr = d->Nr, Nz = d->Nz;
   setup_faces(d, dim);
   int NN = dim==1 ? d->N_ftracks_r : d->N_ftracks_z;
   int *fI = dim==1 ? d->fIndex_r : d->fIndex_z;
   struct face *F = dim==1 ? d->theFaces_1 : d->theFaces_2;
   int Nf = fI[NN];
   int *idx = malloc(sizeof(int)*3*(size_t)(Nf>0?Nf:1));
   double *geo = malloc(sizeof(double)*8*(size_t)(Nf>0?Nf:1));
   int n, JK;
   int Nrmax = dim==1 ? Nr-1 : Nr;
   for( JK=0 ; JK<NN ; ++JK )
   for( n=fI[JK] ; n<fI[JK+1] ; ++n ){
      /* pointer -> global cell index; track JK joins annuli jk and jkp
       * (faces_alt.c:102-109) */
      int j = JK % Nrmax, k = JK / Nrmax;
      int jk = j + Nr*k;
      int jkp = dim==1 ? jk+1 : j + Nr*(k+1);
      int gL = cell_off[jk]  + (int)(F[n].L - d->theCells[jk]);
      int gR = cell_off[jkp] + (int)(F[n].R - d->theCells[jkp]);
      (void)Nz;
      idx[3*n+0] = gL; idx[3*n+1] = gR; idx[3*n+2] = F[n].LRtype;
      geo[8*n+0] = F[n].dxL;  geo[8*n+1] = F[n].dxR;
      geo[8*n+2] = F[n].cm[0]; geo[8*n+3] = F[n].cm[1]; geo[8*n+4] = F[n].cm[2];
      geo[8*n+5] = F[n].dphi; geo[8*n+6] = F[n].dl; geo[8*n+7] = F[n].dA;
   }
   char nm[64];
   snprintf(nm, sizeof nm, "fIndex_%d.i32", dim);
   dump(dir, nm, fI, sizeof(int)*(NN+1));
   snprintf(nm, sizeof nm, "faces_%d.i32", dim);
   dump(dir, nm, idx, sizeof(int)*3*(size_t)Nf);
   snprintf(nm, sizeof nm, "faces_%d.f64", dim);
   dump(dir, nm, geo, sizeof(double)*8*(size_t)Nf);
   free(idx); free(geo);
   if( dim==1 ){ free(d->theFaces_1); d->theFaces_1 = NULL; }
   else        { free(d->theFaces_2); d->theFaces_2 = NULL; }
}

int main(int argc, char *argv[]){
   if( argc < 3 ){
      fprintf(stderr, "usage: %s RUNDIR NSTEPS [DUMPDIR|--time]\n", argv[0]);
      return 1;
   }
   const char *rundir = argv[1];
   int nsteps = atoi(argv[2]);
   const char *dumpdir = argc > 3 ? argv[3] : NULL;
   int timing = dumpdir && strcmp(dumpdir, "--time") == 0;
   char absdump[4096] = "";
   if( dumpdir && !timing ){
      mkdir(dumpdir, 0755);
      if( !realpath(dumpdir, absdump) ){ perror("realpath"); return 2; }
   }
   if( chdir(rundir) != 0 ){ perror("chdir"); return 2; }

   /* main.c:31-62 */
   struct domain theDomain = {0};
   struct profiler prof;
   theDomain.prof = &prof;
   start_clock( &theDomain );
   read_par_file( &theDomain );
   if( mpiSetup(&theDomain, argc, argv) == 1 ) return 0;
   setupGrid( &theDomain );
   setupDomain( &theDomain );
   setupCells( &theDomain );
   if( theDomain.Nr > 1 ){
      exchangeData( &theDomain , 0 );
      if( !theDomain.theParList.R_Periodic ) boundary_trans( &theDomain , 1 );
   }
   if( theDomain.Nz > 1 ){
      exchangeData( &theDomain , 1 );
      if( !theDomain.theParList.Z_Periodic ) boundary_trans( &theDomain , 2 );
   }

   /* the drop-in's explicit upload, after main.c's set-up and boundaries */
   if( disco_gpu_init ){
      int st = disco_gpu_init( &theDomain );
      if( st != 0 ){ fprintf(stderr, "disco_gpu_init: status %d\n", st); return 4; }
   }

   int Nr = theDomain.Nr, Nz = theDomain.Nz;
   int *cell_off = malloc(sizeof(int)*(Nr*Nz+1));
   int jk;
   cell_off[0] = 0;
   for( jk=0 ; jk<Nr*Nz ; ++jk ) cell_off[jk+1] = cell_off[jk] + theDomain.Np[jk];
   int Ncell = cell_off[Nr*Nz];
   int Nreal = count_cells(&theDomain);

   double *dts = malloc(sizeof(double)*(nsteps>0?nsteps:1));
   double t0 = wall();
   int s;
   for( s=0 ; s<nsteps ; ++s ){
      double dt = getmindt( &theDomain );
      dts[s] = dt;
      timestep( &theDomain , dt );
   }
   double t1 = wall();
   double secs = t1 - t0;

   if( timing ){
      printf("{\"seconds\": %.6f, \"steps\": %d, \"real_cells\": %d, "
             "\"zone_updates_per_s\": %.6e}\n",
             secs, nsteps, Nreal, secs > 0 ? (double)Nreal*nsteps/secs : 0.0);
      return 0;
   }
   /* DISCO_REF_REPORT set: one report() of the final state into report.dat
    * of RUNDIR (the current directory), as possiblyOutput would write it */
   if( getenv("DISCO_REF_REPORT") ) report( &theDomain );
   /* DISCO_REF_ASCII=<filestart>: the output module's file of the final
    * state; DISCO_REF_CHECKPOINT=<dir>: its checkpoint (after the dump,
    * since output() averages and then zeroes the diagnostics) */
   const char *ascii = getenv("DISCO_REF_ASCII");
   const char *ckpt = getenv("DISCO_REF_CHECKPOINT");
   if( (ascii || ckpt || dumpdir) && disco_gpu_sync_to_host ) disco_gpu_sync_to_host( &theDomain );
   if( ascii ){
      char fs[4096];
      snprintf(fs, sizeof fs, "%s", ascii);
      output( &theDomain , fs );
   }
   if( !dumpdir ){
      if( ckpt ) disco_ref_checkpoint( &theDomain , ckpt );
      return 0;
   }

   int Q = NUM_Q;
   double *prim = malloc(sizeof(double)*Q*(size_t)Ncell);
   double *cons = malloc(sizeof(double)*Q*(size_t)Ncell);
   double *piph = malloc(sizeof(double)*(size_t)Ncell);
   double *dphi = malloc(sizeof(double)*(size_t)Ncell);
   double *wiph = malloc(sizeof(double)*(size_t)Ncell);
   double *phis = malloc(sizeof(double)*(size_t)Ncell*(NUM_FACES>0?NUM_FACES:1));
   double *grr = malloc(sizeof(double)*Q*(size_t)Ncell);
   double *grp = malloc(sizeof(double)*Q*(size_t)Ncell);
   int *real = malloc(sizeof(int)*(size_t)Ncell);
   int i, q, n = 0;
   for( jk=0 ; jk<Nr*Nz ; ++jk ){
      for( i=0 ; i<theDomain.Np[jk] ; ++i, ++n ){
         struct cell *c = &theDomain.theCells[jk][i];
         for( q=0 ; q<Q ; ++q ){ prim[Q*n+q] = c->prim[q]; cons[Q*n+q] = c->cons[q];
                                 grr[Q*n+q] = c->gradr[q]; grp[Q*n+q] = c->gradp[q]; }
         piph[n] = c->piph; dphi[n] = c->dphi; wiph[n] = c->wiph; real[n] = c->real;
         for( q=0 ; q<NUM_FACES ; ++q ) phis[NUM_FACES*n+q] = c->Phi[q];
      }
   }
   FILE *m;
   char fn[4200];
   snprintf(fn, sizeof fn, "%s/meta.txt", absdump);
   m = fopen(fn, "w");
   fprintf(m, "Nr %d\nNz %d\nNgRa %d\nNgRb %d\nNgZa %d\nNgZb %d\nQ %d\nNcell %d\n"
              "Nreal %d\nnsteps %d\nt %.17g\nnum_faces %d\nnum_tools %d\nt_avg %.17g\nNpl %d\n",
           Nr, Nz, theDomain.NgRa, theDomain.NgRb, theDomain.NgZa, theDomain.NgZb,
           Q, Ncell, Nreal, nsteps, theDomain.t, NUM_FACES, theDomain.num_tools,
           theDomain.theTools.t_avg, theDomain.Npl);
   fclose(m);
   dump(absdump, "Np.i32", theDomain.Np, sizeof(int)*Nr*Nz);
   dump(absdump, "r_jph.f64", theDomain.r_jph-1, sizeof(double)*(Nr+1));
   dump(absdump, "z_kph.f64", theDomain.z_kph-1, sizeof(double)*(Nz+1));
   dump(absdump, "prim.f64", prim, sizeof(double)*Q*(size_t)Ncell);
   dump(absdump, "cons.f64", cons, sizeof(double)*Q*(size_t)Ncell);
   dump(absdump, "piph.f64", piph, sizeof(double)*(size_t)Ncell);
   dump(absdump, "dphi.f64", dphi, sizeof(double)*(size_t)Ncell);
   dump(absdump, "wiph.f64", wiph, sizeof(double)*(size_t)Ncell);
   dump(absdump, "real.i32", real, sizeof(int)*(size_t)Ncell);
   /* the last substep's slopes (plm_phi, plm_trans), for diagnosing */
   dump(absdump, "gradr.f64", grr, sizeof(double)*Q*(size_t)Ncell);
   dump(absdump, "gradp.f64", grp, sizeof(double)*Q*(size_t)Ncell);
   if( NUM_FACES > 0 ) dump(absdump, "Phi.f64", phis, sizeof(double)*NUM_FACES*(size_t)Ncell);
   dump(absdump, "dt.f64", dts, sizeof(double)*(size_t)nsteps);
   dump(absdump, "Qrz.f64", theDomain.theTools.Qrz,
        sizeof(double)*(size_t)Nr*Nz*theDomain.num_tools);
   if( Nr > 1 ) dump_faces(&theDomain, 1, absdump, cell_off);
   if( Nz > 1 ) dump_faces(&theDomain, 2, absdump, cell_off);
   /* planets: M vr omega r phi eps type (h5out.c:444-455) */
   double *pl = malloc(sizeof(double)*7*(size_t)theDomain.Npl);
   int p;
   for( p=0 ; p<theDomain.Npl ; ++p ){
      struct planet *P = theDomain.thePlanets + p;
      double *r = pl + 7*p;
      r[0] = P->M; r[1] = P->vr; r[2] = P->omega; r[3] = P->r; r[4] = P->phi; r[5] = P->eps;
      r[6] = (double)P->type;
   }
   dump(absdump, "planets.f64", pl, sizeof(double)*7*(size_t)theDomain.Npl);
   /* the dt the next step would take */
   double dt_next = getmindt(&theDomain);
   dump(absdump, "dt_next.f64", &dt_next, sizeof(double));
   if( ckpt ) disco_ref_checkpoint( &theDomain , ckpt );
   /* through the drop-in: its own face lists equal the host's, rebuilt from
    * the synced cells above, and the device state is released */
   if( disco_gpu_get_faces && Nr > 1 ){
      int nf = 0;
      disco_gpu_get_faces( &theDomain , 1 , &nf , NULL , NULL , NULL , NULL );
      int *gL = malloc(sizeof(int)*(nf>0?nf:1)), *gR = malloc(sizeof(int)*(nf>0?nf:1));
      disco_gpu_get_faces( &theDomain , 1 , &nf , NULL , gL , gR , NULL );
      dump(absdump, "gpu_faces_1.i32", gL, sizeof(int)*(size_t)nf);
      dump(absdump, "gpu_facesR_1.i32", gR, sizeof(int)*(size_t)nf);
      free(gL); free(gR);
   }
   if( disco_gpu_last_error && disco_gpu_last_error() != 0 ){ fprintf(stderr, "device error\n"); return 3; }
   if( disco_gpu_free ) disco_gpu_free();
   return 0;
}
