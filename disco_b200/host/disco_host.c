/*
 * Host-side start-up of the B200 Disco timestep: in.par / Makefile_opt.in
 * parsing and grid set-up.  Restates readpar.c, gridsetup.c and the
 * phi-offset part of domain.c for the serial path (one rank, dim_rank = 0).
 */
#include "disco_host.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { VAR_INT, VAR_DOUB };

/* readvar (readpar.c:6-42): the first line whose first token equals the key;
 * value starts after the key and any of "\t :=>_"; parsed with %lf and
 * truncated to int for integer keys. */
static int readvar(const char *path, const char *key, int type, void *ptr){
   FILE *f = fopen(path, "r");
   if( !f ) return 1;
   char s[512], nm[512] = "", s1[512] = "";
   int found = 0;
   while( !found && fgets(s, sizeof s, f) != NULL ){
      nm[0] = '\0';
      if( sscanf(s, "%511s ", nm) < 1 ) continue;
      if( strcmp(nm, key) == 0 ){ strcpy(s1, s); found = 1; }
   }
   fclose(f);
   if( !found ) return 1;
   char *s2 = s1 + strlen(nm);
   s2 += strspn(s2, "\t :=>_");
   double v = 0.0;
   if( sscanf(s2, "%lf", &v) < 1 ) v = 0.0;
   if( type == VAR_INT ) *(int *)ptr = (int)v;
   else *(double *)ptr = v;
   return 0;
}

int disco_read_par(const char *path, disco_params *p, int *nmissing){
   if( !path || !p ) return DISCO_ERR_ARG;
   FILE *f = fopen(path, "r");
   if( !f ) return DISCO_ERR_ARG;
   fclose(f);
   memset(p, 0, sizeof *p);
   int err = 0, tT = 0, pT = 0, zT = 0, tmp = 0;
   double dummy = 0.0;
#define RI(k,v) err += readvar(path, k, VAR_INT,  &(v))
#define RD(k,v) err += readvar(path, k, VAR_DOUB, &(v))
   RI("Num_R", p->Num_R);            RI("Num_Z", p->Num_Z);
   RD("aspect", p->aspect);
   RI("Num_Reports", tmp);           RI("Num_Snapshots", tmp);
   RI("Num_Checkpoints", tmp);
   RD("T_Start", p->t_min);          RD("T_End", dummy);
   RD("R_Min", p->rmin);             RD("R_Max", p->rmax);
   RD("Z_Min", p->zmin);             RD("Z_Max", p->zmax);
   RD("Phi_Max", p->phimax);
   RI("Use_Logtime", tmp);
   RI("Log_Zoning", p->LogZoning);
   RI("R_Periodic", p->R_Periodic);  RI("Z_Periodic", p->Z_Periodic);
   RI("NoBC_Rmin", p->NoBC_Rmin);    RI("NoBC_Rmax", p->NoBC_Rmax);
   RI("NoBC_Zmin", p->NoBC_Zmin);    RI("NoBC_Zmax", p->NoBC_Zmax);
   RD("Log_Radius", p->LogRadius);
   RD("Max_Aspect_Short", dummy);    RD("Max_Aspect_Long", dummy);
   RI("Timestep", p->Timestep);
   RD("CFL", p->CFL);                RD("Max_DT", p->maxDT);
   RD("PLM", p->PLM);
   RD("Adiabatic_Index", p->Adiabatic_Index);
   RI("Isothermal", p->isothermal_flag);
   RI("Cs2_Profile", p->Cs2_Profile); RD("Cs2_Par", p->Cs2_Par);
   RD("Density_Floor", p->Density_Floor);
   RD("Pressure_Floor", p->Pressure_Floor);
   RI("Mesh_Motion", p->Mesh_Motion);
   RI("Exact_Mesh_Omega", p->Exact_Mesh_Omega);
   RD("Exact_Mesh_Omega_Par", p->Exact_Mesh_Omega_Par);
   RI("Energy_Omega", p->Energy_Omega);
   RD("Energy_Omega_Par", p->Energy_Omega_Par);
   RI("RotFrame", p->RotFrame);      RD("RotOmega", p->RotOmega);
   RD("RotD", p->RotD);
   RI("Riemann_Solver", p->Riemann_Solver);
   RI("Initial_Regrid", tmp);        RI("Restart", tmp);
   RI("Use_Viscosity", p->visc_flag); RD("Viscosity", p->viscosity);
   RI("Use_As_Alpha", p->alpha_flag);
   RI("Include_Atmos", p->include_atmos);
   RI("T_Times_2pi", tT);            RI("P_Times_2pi", pT);
   RI("Z_Times_pi", zT);
   RD("Mach_Number", p->Disk_Mach);  RD("Mass_Ratio", p->Mass_Ratio);
   RD("Eccentricity", dummy);        RD("Drift_Rate", dummy);
   RD("Drift_Exp", dummy);
   RI("Grav2D", p->grav2D);
   RI("Constrained_Transport", p->CT);
   RI("Metric_Par0", tmp);
   RD("Metric_Par1", p->metricPar[1]); RD("Metric_Par2", p->metricPar[2]);
   RD("Metric_Par3", p->metricPar[3]); RD("Metric_Par4", p->metricPar[4]);
   RI("Init_Par0", p->initPar0);
   RD("Init_Par1", p->initPar[1]);   RD("Init_Par2", p->initPar[2]);
   RD("Init_Par3", p->initPar[3]);   RD("Init_Par4", p->initPar[4]);
   RD("Init_Par5", p->initPar[5]);   RD("Init_Par6", p->initPar[6]);
   RD("Init_Par7", p->initPar[7]);   RD("Init_Par8", p->initPar[8]);
   RI("Noise_Type", p->noiseType);
   RD("Noise_Abs", p->noiseAbs);     RD("Noise_Rel", p->noiseRel);
#undef RI
#undef RD
   /* readpar.c:162-172 */
   if( tT ) p->t_min *= 2.*M_PI;
   if( pT ) p->phimax *= 2.*M_PI;
   if( zT ){ p->zmin *= M_PI; p->zmax *= M_PI; }
   if( nmissing ) *nmissing = err;
   return DISCO_OK;
}

static int opt_value(const char *path, const char *key, char *out, size_t n){
   FILE *f = fopen(path, "r");
   if( !f ) return 1;
   char s[512];
   int found = 0;
   while( !found && fgets(s, sizeof s, f) ){
      char *h = strchr(s, '#'); if( h ) *h = '\0';
      char k[128] = "", v[256] = "";
      char *eq = strchr(s, '=');
      if( !eq ) continue;
      *eq = '\0';
      if( sscanf(s, "%127s", k) != 1 ) continue;
      if( strcmp(k, key) ) continue;
      if( sscanf(eq+1, "%255s", v) != 1 ) continue;
      strncpy(out, v, n-1); out[n-1] = '\0';
      found = 1;
   }
   fclose(f);
   return found ? 0 : 1;
}

int disco_read_opt(const char *path, disco_modules *m){
   if( !path || !m ) return DISCO_ERR_ARG;
   char v[256];
   memset(m, 0, sizeof *m);
   if( opt_value(path, "HYDRO", v, sizeof v) ) return DISCO_ERR_ARG;
   if( !strcmp(v, "euler") ) m->hydro = DISCO_HYDRO_EULER;
   else if( !strcmp(v, "mhd") ) m->hydro = DISCO_HYDRO_MHD;
   else if( !strcmp(v, "grmhd2") ) m->hydro = DISCO_HYDRO_GRMHD;
   else return DISCO_ERR_UNSUPPORTED;
   m->metric = DISCO_METRIC_SCHW_KS_RPZ;
   if( m->hydro == DISCO_HYDRO_GRMHD ){
      if( opt_value(path, "METRIC", v, sizeof v) ) return DISCO_ERR_ARG;
      if( !strcmp(v, "schw_ks_rpz") ) m->metric = DISCO_METRIC_SCHW_KS_RPZ;
      else if( !strcmp(v, "kerr_ks_rpz") ) m->metric = DISCO_METRIC_KERR_KS_RPZ;
      else return DISCO_ERR_UNSUPPORTED;
      if( opt_value(path, "FRAME", v, sizeof v) || strcmp(v, "normal") ) return DISCO_ERR_UNSUPPORTED;
   }
   if( opt_value(path, "BOUNDARY", v, sizeof v) ) return DISCO_ERR_ARG;
   if( !strcmp(v, "fixed") ) m->boundary = DISCO_BC_FIXED;
   else if( !strcmp(v, "zerograd") ) m->boundary = DISCO_BC_ZEROGRAD;
   else if( !strcmp(v, "fixed3d") ) m->boundary = DISCO_BC_FIXED3D;
   else if( !strcmp(v, "polar") ) m->boundary = DISCO_BC_POLAR;
   else if( !strcmp(v, "outflow3d") ) m->boundary = DISCO_BC_OUTFLOW3D;
   else if( !strcmp(v, "zerograd_omk") ) m->boundary = DISCO_BC_ZEROGRAD_OMK;
   else if( !strcmp(v, "accrete3d") ) m->boundary = DISCO_BC_ACCRETE3D;
   else if( !strcmp(v, "polar3d") ) m->boundary = DISCO_BC_POLAR3D;
   else if( !strcmp(v, "horizon") ) m->boundary = DISCO_BC_HORIZON;
   else if( !strcmp(v, "horizon3d") ) m->boundary = DISCO_BC_HORIZON3D;
   else if( !strcmp(v, "horizon_bin") ) m->boundary = DISCO_BC_HORIZON_BIN;
   else if( !strcmp(v, "fixRrefZ") ) m->boundary = DISCO_BC_FIXRREFZ;
   else if( !strcmp(v, "tube") ) m->boundary = DISCO_BC_TUBE;
   else if( !strcmp(v, "surfaceGravBox") ) m->boundary = DISCO_BC_SURFACEGRAVBOX;
   else if( !strcmp(v, "fixed_gap") ) m->boundary = DISCO_BC_FIXED_GAP;
   else if( !strcmp(v, "flowthrough") ) m->boundary = DISCO_BC_FLOWTHROUGH;
   else return DISCO_ERR_UNSUPPORTED;
   if( opt_value(path, "PLANETS", v, sizeof v) ) return DISCO_ERR_ARG;
   if( !strcmp(v, "none") ) m->planets = DISCO_PLANETS_NONE;
   else if( !strcmp(v, "sun") ) m->planets = DISCO_PLANETS_SUN;
   else if( !strcmp(v, "cm2") ) m->planets = DISCO_PLANETS_CM2;
   else if( !strcmp(v, "binary_soft") ) m->planets = DISCO_PLANETS_BINARY_SOFT;
   else if( !strcmp(v, "circular") ) m->planets = DISCO_PLANETS_CIRCULAR;
   else if( !strcmp(v, "cm") ) m->planets = DISCO_PLANETS_CM;
   else return DISCO_ERR_UNSUPPORTED;
   if( opt_value(path, "INITIAL", v, sizeof v) ) return DISCO_ERR_ARG;
   if( !strcmp(v, "kepler_noise") ) m->initial = DISCO_IC_KEPLER_NOISE;
   else if( !strcmp(v, "mhd_shear_noise") ) m->initial = DISCO_IC_MHD_SHEAR_NOISE;
   else if( !strcmp(v, "gr_torus_noise") ) m->initial = DISCO_IC_GR_TORUS_NOISE;
   else m->initial = DISCO_IC_HOST;      /* another module: its state comes from the host */
   if( opt_value(path, "ANALYSIS", v, sizeof v) ) m->analysis = DISCO_DIAG_NONE;
   else if( !strcmp(v, "diag_disk2d") ) m->analysis = DISCO_DIAG_DISK2D;
   else if( !strcmp(v, "diag_euler") ) m->analysis = DISCO_DIAG_EULER;
   else if( !strcmp(v, "diag_mhdmri") ) m->analysis = DISCO_DIAG_MHDMRI;
   else m->analysis = DISCO_DIAG_NONE;
   if( opt_value(path, "GEOMETRY", v, sizeof v) || strcmp(v, "cylindrical") )
      return DISCO_ERR_UNSUPPORTED;
   if( opt_value(path, "NUM_C", v, sizeof v) ) return DISCO_ERR_ARG;
   m->num_c = atoi(v);
   if( opt_value(path, "NUM_N", v, sizeof v) ) return DISCO_ERR_ARG;
   m->num_n = atoi(v);
   if( opt_value(path, "CT_MODE", v, sizeof v) ) return DISCO_ERR_ARG;
   m->ct_mode = atoi(v);
   return DISCO_OK;
}

/* gridsetup.c:15-142 with dim_rank = {0,0}, dim_size = {1,1}. */
int disco_setup_grid(const disco_params *p, int *pNr, int *pNz, int *Ng,
                     int *Np, double *r_jph, double *z_kph){
   if( !p || !pNr || !pNz || !Ng ) return DISCO_ERR_ARG;
   const int NG = 2;                                    /* NUM_G, paul.h:30 */
   int Num_R = p->Num_R, Num_Z = p->Num_Z;
   if( Num_R < 1 || Num_Z < 1 || p->phimax <= 0.0 ) return DISCO_ERR_ARG;
   int N0r = 0, N1r = Num_R;
   int NgRa = NG, NgRb = NG;
   if( p->NoBC_Rmin ) NgRa = 0;
   if( p->NoBC_Rmax ) NgRb = 0;
   N0r -= NgRa; N1r += NgRb;
   int Nr = N1r - N0r;
   int N0z = 0, N1z = Num_Z;
   int NgZa = NG, NgZb = NG;
   if( Num_Z == 1 || p->NoBC_Zmin ) NgZa = 0;
   if( Num_Z == 1 || p->NoBC_Zmax ) NgZb = 0;
   N0z -= NgZa; N1z += NgZb;
   int Nz = N1z - N0z;
   *pNr = Nr; *pNz = Nz;
   Ng[0] = NgRa; Ng[1] = NgRb; Ng[2] = NgZa; Ng[3] = NgZb;
   if( !Np || !r_jph || !z_kph ) return DISCO_OK;

   double Rmin = p->rmin, Rmax = p->rmax, R0 = p->LogRadius;
   int j, k;
   for( j=-1 ; j<Nr ; ++j ){
      double x = (N0r + j + 1) / (double) Num_R;
      double v;
      if( p->LogZoning == 0 ) v = Rmin + x*(Rmax-Rmin);
      else if( p->LogZoning == 1 ) v = Rmin*pow(Rmax/Rmin, x);
      else v = R0*(pow(Rmax/R0, x)-1) + Rmin + (R0-Rmin)*x;
      r_jph[j+1] = v;
   }
   double dz = (p->zmax - p->zmin)/(double)Num_Z;
   double z0 = p->zmin + (double)N0z*dz;
   for( k=-1 ; k<Nz ; ++k ) z_kph[k+1] = z0 + ((double)k+1.)*dz;

   double Pmax = p->phimax;
   for( k=0 ; k<Nz ; ++k ) for( j=0 ; j<Nr ; ++j ){
      double rp = r_jph[j+1], rm = r_jph[j];
      double dr = rp - rm;                               /* get_dL(..,1) */
      double hp = rp;                                    /* get_scale_factor(xp,0) */
      double dp = p->aspect*dr/hp;
      int n = (int)(Pmax/dp);
      if( n < 4 ) n = 4;
      Np[j + Nr*k] = n;
   }
   return DISCO_OK;
}

/* The draws of addNoise (noise.c:15-50) for each real cell, in setupCells'
 * order (domain.c:183-205: k, then j, then i), continuing glibc's rand()
 * stream where setupDomain left it: 4 per cell for types 1 and 3, 2 for
 * type 2, each 2*rand()/RAND_MAX - 1. */
static void noise_draws(const disco_params *p, int Nr, int Nz, const int *Ng, const int *Np,
                        const int *coff, double *noise){
   int per = p->noiseType == 2 ? 2 : (p->noiseType == 1 || p->noiseType == 3) ? 4 : 0;
   int j, k, i, m;
   for( k=Ng[2] ; k<Nz-Ng[3] ; ++k ) for( j=Ng[0] ; j<Nr-Ng[1] ; ++j ){
      int jk = j + Nr*k;
      for( i=0 ; i<Np[jk] ; ++i ) for( m=0 ; m<per ; ++m )
         noise[4*(coff[jk]+i) + m] = 2 * ((double)rand() / (double)(RAND_MAX)) - 1;
   }
}

static int setup_phi(const disco_params *p, int Nr, int Nz, const int *Ng,
                     const int *Np, double *piph, double *dphi, int *real, double *noise);

/* domain.c:172-233 (serial), then calc_dp (misc.c:271-288). */
int disco_setup_phi(const disco_params *p, int Nr, int Nz, const int *Ng,
                    const int *Np, double *piph, double *dphi, int *real){
   return setup_phi(p, Nr, Nz, Ng, Np, piph, dphi, real, NULL);
}

int disco_setup_noise(const disco_params *p, int Nr, int Nz, const int *Ng,
                      const int *Np, double *noise){
   if( !p || !Ng || !Np || !noise ) return DISCO_ERR_ARG;
   size_t n = 0;
   int jk;
   for( jk=0 ; jk<Nr*Nz ; ++jk ) n += (size_t)Np[jk];
   double *piph = malloc(sizeof(double)*(n ? n : 1)), *dphi = malloc(sizeof(double)*(n ? n : 1));
   if( !piph || !dphi ){ free(piph); free(dphi); return DISCO_ERR_ARG; }
   memset(noise, 0, sizeof(double)*4*n);
   int s = setup_phi(p, Nr, Nz, Ng, Np, piph, dphi, NULL, noise);
   free(piph); free(dphi);
   return s;
}

static int setup_phi(const disco_params *p, int Nr, int Nz, const int *Ng,
                     const int *Np, double *piph, double *dphi, int *real, double *noise){
   if( !p || !Ng || !Np || !piph || !dphi ) return DISCO_ERR_ARG;
   double Pmax = p->phimax;
   const int NG = 2;
   /* global index ranges of gridsetup.c:57-74: ghost layers count as global
    * annuli unless NoBC, even in z when Num_Z == 1 (then NgZa = 0 locally) */
   int N0r = -Ng[0], N0z = -Ng[2];
   int N0r_glob = p->NoBC_Rmin ? 0 : -NG;
   int N0z_glob = p->NoBC_Zmin ? 0 : -NG;
   int Nr_glob = p->Num_R + (p->NoBC_Rmin ? 0 : NG) + (p->NoBC_Rmax ? 0 : NG);
   srand(314159);
   rand();
   int j, k, i, c = 0;
   int *coff = malloc(sizeof(int)*(Nr*Nz+1));
   coff[0] = 0;
   for( j=0 ; j<Nr*Nz ; ++j ) coff[j+1] = coff[j] + Np[j];
   for( k=N0z_glob ; k<N0z ; ++k ) for( j=0 ; j<Nr_glob ; ++j ) rand();   /* domain.c:202-204 */
   for( k=0 ; k<Nz ; ++k ){
      for( j=N0r_glob ; j<N0r ; ++j ) rand();                              /* :209-210 */
      for( j=0 ; j<Nr ; ++j ){
         int jk = k*Nr + j;
         double p0 = Pmax*(double)rand()/(double)RAND_MAX;
         double dp = Pmax/(double)Np[jk];
         for( i=0 ; i<Np[jk] ; ++i ){
            double phi = p0 + dp*(double)i;
            if( phi > Pmax ) phi -= Pmax;
            piph[coff[jk]+i] = phi;
         }
      }
      for( j=N0r+Nr ; j<N0r_glob+Nr_glob ; ++j ) rand();                  /* :227-231 */
   }
   if( noise ) noise_draws(p, Nr, Nz, Ng, Np, coff, noise);
   for( j=0 ; j<Nr*Nz ; ++j ){
      for( i=0 ; i<Np[j] ; ++i ){
         int im = i==0 ? Np[j]-1 : i-1;
         double dpp = piph[coff[j]+i] - piph[coff[j]+im];
         int n = 0;
         while( dpp < 0.0 && n++ < 64 ) dpp += Pmax;
         while( dpp > Pmax && n++ < 64 ) dpp -= Pmax;
         dphi[coff[j]+i] = dpp;
      }
   }
   if( real ){
      for( k=0 ; k<Nz ; ++k ) for( j=0 ; j<Nr ; ++j ){
         int jk = j + Nr*k;
         int isreal = (j >= Ng[0] && j < Nr-Ng[1] && k >= Ng[2] && k < Nz-Ng[3]);
         for( i=0 ; i<Np[jk] ; ++i ) real[coff[jk]+i] = isreal;
      }
   }
   (void)c;
   free(coff);
   return DISCO_OK;
}

/* sizes of the ABI structs, for binding checks (ctypes / cgo mirrors) */
int disco_sizeof(int which){
   switch( which ){
      case 0: return (int)sizeof(disco_params);
      case 1: return (int)sizeof(disco_modules);
   }
   return -1;
}
