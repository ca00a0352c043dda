/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * The reference's checkpoint and restart modules need HDF5 (Output/h5out.c,
 * Restart/h5in.c), which this machine does not have.  This file stands in
 * for them in the oracle build, over a directory of raw little-endian files
 * with the same datasets:
 *
 *   dims.txt       Nr_Tot Nz_Tot Nc Nq Npl NpDat Ntools
 *   T.f64 [1]  r_jph.f64 [Nr_Tot+1]  z_kph.f64 [Nz_Tot+1]
 *   Index.i32 Np.i32 Id_phi0.i32 [Nz_Tot][Nr_Tot]
 *   Cells.f64 [Nc][Nq]  Planets.f64 [Npl][NpDat]  Diagnostics.f64 [Nz][Nr][Ntools]
 *
 * disco_ref_checkpoint() restates output() of h5out.c:349-598 for one rank
 * (dim_rank 0, dim_size 1): avg_diagnostics, the datasets, zero_diagnostics.
 * restart() replaces the Restart module (the reference's setupCells calls
 * it when in.par has Restart 1, domain.c:141-142) and restates h5in.c:100-354
 * for one rank over the directory named by DISCO_REF_RESTART, for a grid
 * equal to the one setupGrid/setupDomain already built from the same in.par
 * (it checks that, and aborts otherwise, instead of re-allocating the grid):
 * t from T, each annulus's cells from Cells at Index (Doub2Cell), the
 * planets' seven columns, diagnostics zeroed.
 */
#include "paul.h"
#include <sys/stat.h>

void avg_diagnostics( struct domain * );
void zero_diagnostics( struct domain * );

static void put(const char *dir, const char *name, const void *p, size_t nbytes){
   char fn[4200];
   snprintf(fn, sizeof fn, "%s/%s", dir, name);
   FILE *f = fopen(fn, "wb");
   if( !f ){ fprintf(stderr, "ref_checkpoint: cannot write %s\n", fn); exit(2); }
   if( nbytes ) fwrite(p, 1, nbytes, f);
   fclose(f);
}

static void get(const char *dir, const char *name, void *p, size_t nbytes){
   char fn[4200];
   snprintf(fn, sizeof fn, "%s/%s", dir, name);
   FILE *f = fopen(fn, "rb");
   if( !f || (nbytes && fread(p, 1, nbytes, f) != nbytes) ){
      fprintf(stderr, "ref_checkpoint: cannot read %s\n", fn);
      exit(2);
   }
   fclose(f);
}

void disco_ref_checkpoint( struct domain * theDomain , const char * dir ){
   int Nr = theDomain->Nr, Nz = theDomain->Nz;
   int *Np = theDomain->Np;
   int Npl = theDomain->Npl;
   int Ntools = theDomain->num_tools;
   const int NpDat = 7;
   int Nq = NUM_Q + NUM_FACES + 1;
   mkdir(dir, 0755);
   avg_diagnostics( theDomain );

   int jk, i, q, Nc = 0;
   for( jk=0 ; jk<Nr*Nz ; ++jk ) Nc += Np[jk];
   double *Cells = malloc(sizeof(double)*(size_t)Nc*Nq);
   int *Index = malloc(sizeof(int)*Nr*Nz), *Id = malloc(sizeof(int)*Nr*Nz);
   int index = 0;
   for( jk=0 ; jk<Nr*Nz ; ++jk ){            /* k outer, j inner: jk order */
      Index[jk] = index;
      double phi0 = M_PI;
      int best = 0;
      for( i=0 ; i<Np[jk] ; ++i ){
         struct cell *c = &theDomain->theCells[jk][i];
         double *row = Cells + (size_t)index*Nq;
         for( q=0 ; q<NUM_Q ; ++q ) row[q] = c->prim[q];
         for( q=0 ; q<NUM_FACES ; ++q ) row[NUM_Q+q] = c->Phi[q];
         row[NUM_Q+NUM_FACES] = c->piph;
         double phi = c->piph - .5*c->dphi;
         if( cos(phi0) < cos(phi) ){ phi0 = phi; best = index; }
         ++index;
      }
      Id[jk] = best;
   }
   double *Pl = malloc(sizeof(double)*(size_t)Npl*NpDat);
   int p;
   for( p=0 ; p<Npl ; ++p ){
      struct planet *pl = theDomain->thePlanets + p;
      double *r = Pl + (size_t)p*NpDat;
      r[0] = pl->M; r[1] = pl->vr; r[2] = pl->omega; r[3] = pl->r; r[4] = pl->phi;
      r[5] = pl->eps; r[6] = (double)pl->type;
   }
   char fn[4200];
   snprintf(fn, sizeof fn, "%s/dims.txt", dir);
   FILE *f = fopen(fn, "w");
   fprintf(f, "%d %d %d %d %d %d %d\n", Nr, Nz, Nc, Nq, Npl, NpDat, Ntools);
   fclose(f);
   put(dir, "T.f64", &theDomain->t, sizeof(double));
   put(dir, "r_jph.f64", theDomain->r_jph - 1, sizeof(double)*(Nr+1));
   put(dir, "z_kph.f64", theDomain->z_kph - 1, sizeof(double)*(Nz+1));
   put(dir, "Index.i32", Index, sizeof(int)*Nr*Nz);
   put(dir, "Np.i32", Np, sizeof(int)*Nr*Nz);
   put(dir, "Id_phi0.i32", Id, sizeof(int)*Nr*Nz);
   put(dir, "Cells.f64", Cells, sizeof(double)*(size_t)Nc*Nq);
   put(dir, "Planets.f64", Pl, sizeof(double)*(size_t)Npl*NpDat);
   put(dir, "Diagnostics.f64", theDomain->theTools.Qrz, sizeof(double)*(size_t)Nr*Nz*Ntools);
   zero_diagnostics( theDomain );
   free(Cells); free(Index); free(Id); free(Pl);
}

void restart( struct domain * theDomain ){
   const char *dir = getenv("DISCO_REF_RESTART");
   if( !dir ){ fprintf(stderr, "ref_checkpoint: Restart 1 needs DISCO_REF_RESTART\n"); exit(2); }
   int Nr = theDomain->Nr, Nz = theDomain->Nz;
   int NrT, NzT, Nc, Nq, Npl, NpDat, Ntools;
   char fn[4200];
   snprintf(fn, sizeof fn, "%s/dims.txt", dir);
   FILE *f = fopen(fn, "r");
   if( !f || fscanf(f, "%d %d %d %d %d %d %d", &NrT, &NzT, &Nc, &Nq, &Npl, &NpDat, &Ntools) != 7 ){
      fprintf(stderr, "ref_checkpoint: bad %s\n", fn);
      exit(2);
   }
   fclose(f);
   if( NrT != Nr || NzT != Nz || Npl != theDomain->Npl ){
      fprintf(stderr, "ref_checkpoint: checkpoint grid differs from in.par's\n");
      exit(2);
   }
   if( Nq != NUM_Q+NUM_FACES+1 ){ printf("Ummm, I got an hdf5 read error. Check NUM_Q.\n"); exit(1); }
   int jk, i, q;
   int *Np = malloc(sizeof(int)*Nr*Nz), *Index = malloc(sizeof(int)*Nr*Nz);
   double *rj = malloc(sizeof(double)*(Nr+1)), *zk = malloc(sizeof(double)*(Nz+1));
   get(dir, "T.f64", &theDomain->t, sizeof(double));
   get(dir, "Np.i32", Np, sizeof(int)*Nr*Nz);
   get(dir, "Index.i32", Index, sizeof(int)*Nr*Nz);
   get(dir, "r_jph.f64", rj, sizeof(double)*(Nr+1));
   get(dir, "z_kph.f64", zk, sizeof(double)*(Nz+1));
   if( memcmp(Np, theDomain->Np, sizeof(int)*Nr*Nz) ||
       memcmp(rj, theDomain->r_jph - 1, sizeof(double)*(Nr+1)) ||
       memcmp(zk, theDomain->z_kph - 1, sizeof(double)*(Nz+1)) ){
      fprintf(stderr, "ref_checkpoint: checkpoint grid differs from in.par's\n");
      exit(2);
   }
   double *Cells = malloc(sizeof(double)*(size_t)Nc*Nq);
   get(dir, "Cells.f64", Cells, sizeof(double)*(size_t)Nc*Nq);
   for( jk=0 ; jk<Nr*Nz ; ++jk ){
      for( i=0 ; i<Np[jk] ; ++i ){
         struct cell *c = &theDomain->theCells[jk][i];
         const double *row = Cells + ((size_t)Index[jk] + i)*Nq;
         for( q=0 ; q<NUM_Q ; ++q ) c->prim[q] = row[q];
         for( q=0 ; q<NUM_FACES ; ++q ) c->Phi[q] = row[NUM_Q+q];
         c->piph = row[NUM_Q+NUM_FACES];
      }
   }
   double *Pl = malloc(sizeof(double)*(size_t)Npl*NpDat);
   get(dir, "Planets.f64", Pl, sizeof(double)*(size_t)Npl*NpDat);
   int p;
   for( p=0 ; p<Npl ; ++p ){
      struct planet *pl = theDomain->thePlanets + p;
      const double *r = Pl + (size_t)p*NpDat;
      pl->M = r[0]; pl->vr = r[1]; pl->omega = r[2]; pl->r = r[3]; pl->phi = r[4]; pl->eps = r[5];
      pl->type = NpDat > 6 ? (int)r[6] : PLPOINTMASS;
   }
   zero_diagnostics( theDomain );
   free(Np); free(Index); free(rj); free(zk); free(Cells); free(Pl);
}
