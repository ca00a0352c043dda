/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * CPU restatement of the reference Disco serial RK timestep (USE_MPI=0),
 * plain C, FP64, one thread, written in the reference's own scatter order so
 * that on the same libm it reproduces the reference bit for bit.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it,
 * as the checker.  Pinned against the reference binary built by
 * oracle/Makefile (tests/test_oracle_pin.py).
 *
 * Scope: cylindrical geometry; Hydro euler (Hydro/euler.c); planets sun /
 * none / cm2 / softened binary; boundaries fixed / zerograd; Initial
 * kepler_noise; diagnostics diag_disk2d; HLL and HLLC; mesh motion 0/1/3/4;
 * RK2 and forward Euler.  Array layout: cells in annulus order (jk = j+Nr*k,
 * i = 0..Np[jk]-1), Q doubles per cell (cell-major), as struct cell holds
 * them (paul.h:183-203).
 */
#include "oracle.h"
#include "ic_kepler_noise.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum{RHO,PPP,URR,UPP,UZZ,BRR,BPP,BZZ};
enum{DDD,TAU,SRR,LLL,SZZ};
#define MAXQ 16
#define WRAP_CAP 64

typedef struct {
   double r, phi, M, omega, vr;
   double RK_r, RK_phi, RK_M, RK_omega, RK_vr;
   double eps;
   int type;
} orc_planet;

typedef struct {
   int L, R;          /* global cell index */
   double dxL, dxR, cm[3], dphi, dl, dA;
   int LRtype;
} orc_face;

struct orc_domain {
   disco_params p;
   disco_modules m;
   int Nr, Nz, NgRa, NgRb, NgZa, NgZb, Q, NC;
   int *Np, *coff, Ncell;
   double *rj, *zk;          /* shifted by one: rj[-1] valid */
   double *prim, *cons, *RKcons, *gradp, *gradr, *gradz;
   double *piph, *dphi, *wiph;
   int *real;
   int Npl;
   orc_planet pl[4];
   int Ntr[3];               /* number of face tracks per dim (1,2) */
   int *fI[3];
   orc_face *F[3];
   double t;
   int count_steps;
   int nq;
   double *Qrz, t_avg;
   disco_ic_kepler_noise ic;
};

/* ---------------------------------------------------------------- geometry
 * Geometry/cylindrical.c:10-63 */
static double PMAX;

static double get_dp(double phip, double phim){           /* cylindrical.c:10 */
   double dp = phip - phim;
   int n = 0;
   while( dp < 0.0 && n++ < WRAP_CAP ) dp += PMAX;
   while( dp > PMAX && n++ < WRAP_CAP ) dp -= PMAX;
   return dp;
}
static double get_signed_dp(double phip, double phim){    /* cylindrical.c:17 */
   double dp = phip - phim;
   int n = 0;
   while( dp < -.5*PMAX && n++ < WRAP_CAP ) dp += PMAX;
   while( dp >  .5*PMAX && n++ < WRAP_CAP ) dp -= PMAX;
   return dp;
}
static double get_centroid(double xp, double xm, int dim){ /* cylindrical.c:24 */
   if( dim == 1 ) return 2.0*(xp*xp + xp*xm + xm*xm) / (3.0*(xp+xm));
   return 0.5*(xp+xm);
}
static double get_dL(const double *xp, const double *xm, int dim){ /* :32 */
   double r = .5*(xp[0]+xm[0]);
   double dphi = get_dp(xp[1], xm[1]);
   if( dim == 0 ) return r*dphi;
   else if( dim == 1 ) return xp[0]-xm[0];
   return xp[2]-xm[2];
}
static double get_dA(const double *xp, const double *xm, int dim){ /* :43 */
   double r  = .5*(xp[0]+xm[0]);
   double dr = xp[0]-xm[0];
   double dphi = get_dp(xp[1], xm[1]);
   double dz = xp[2]-xm[2];
   if( dim == 0 ) return dr*dz;
   else if( dim == 1 ) return r*dphi*dz;
   return r*dr*dphi;
}
static double get_dV(const double *xp, const double *xm){  /* :56 */
   double r  = .5*(xp[0]+xm[0]);
   double dr = xp[0]-xm[0];
   double dphi = get_dp(xp[1], xm[1]);
   double dz = xp[2]-xm[2];
   return r*dr*dphi*dz;
}

/* ---------------------------------------------------------------- omega.c */
static double get_om(const disco_params *p, const double *x){   /* omega.c:62 */
   double r = x[0], O0 = p->RotOmega;
   switch( p->Energy_Omega ){
      case 1: return 1.0-O0;
      case 2: return 1.0/pow(r,1.5)-O0;
      case 3: { double n = 8.0; return 1./pow( pow( r , 1.5*n ) + 1. , 1./n )-O0; }
      case 4: return 10.*exp(-.5*r*r)-O0;
      default: return 0.0-O0;
   }
}
static double get_om1(const disco_params *p, const double *x){  /* omega.c:87 */
   double r = x[0];
   switch( p->Energy_Omega ){
      case 1: return 0.0;
      case 2: return -1.5/pow(r,2.5);
      case 3: { double n = 8.0;
                return -1.5 * pow(r,-1+1.5*n) / pow( pow(r,1.5*n) + 1. , 1.0+1./n ); }
      case 4: return 10.*r*exp(-.5*r*r);
      default: return 0.0;
   }
}
static double get_om2(const disco_params *p, const double *x){ (void)p; (void)x; return 0.0; }
static double get_cs2(const disco_params *p, const double *x){  /* omega.c:116 */
   double r = x[0], Mach = p->Disk_Mach;
   switch( p->Cs2_Profile ){
      case 1: return 1./(Mach*Mach);
      case 2: { double nu = .5; return .5/Mach/Mach/pow(r,2.*nu); }
      case 3: { double M = p->metricPar[2];
                return M*p->initPar[4]*p->initPar[4] / (2*p->initPar[2]*p->initPar[2]*p->initPar[2]); }
      case 4: { double v2 = p->metricPar[2]/r; return v2/(Mach*Mach); }
      default: return 1.0;
   }
}
static double mesh_om(const disco_params *p, const double *x){  /* omega.c:43 */
   double r = x[0];
   if( p->Exact_Mesh_Omega == 1 ) return 1.0;
   if( p->Exact_Mesh_Omega == 2 ) return pow(r,-1.5);
   if( p->Exact_Mesh_Omega == 3 ){ double n = 8.0; return 1./pow( pow( r , 1.5*n ) + 1. , 1./n ); }
   return 0.0;
}

/* ---------------------------------------------------------------- euler.c */
static void prim2cons(const orc_domain *d, const double *prim, double *cons,
                      const double *x, double dV){            /* euler.c:36 */
   const disco_params *p = &d->p;
   double gam = p->Adiabatic_Index;
   double r = x[0];
   double rho = prim[RHO], Pp = prim[PPP], vr = prim[URR];
   double vp = prim[UPP]*r, vz = prim[UZZ];
   double om = get_om(p, x);
   double vp_off = vp - om*r;
   double v2 = vr*vr + vp_off*vp_off + vz*vz;
   double rhoe = Pp/(gam - 1.);
   cons[DDD] = rho*dV;
   cons[TAU] = (.5*rho*v2 + rhoe )*dV;
   cons[SRR] = rho*vr*dV;
   cons[LLL] = r*rho*vp*dV;
   cons[SZZ] = rho*vz*dV;
   int q;
   for( q=d->NC ; q<d->Q ; ++q ) cons[q] = prim[q]*cons[DDD];
}
static void getUstar(const orc_domain *d, const double *prim, double *Ustar,
                     const double *x, double Sk, double Ss, const double *n){ /* euler.c:64 */
   const disco_params *p = &d->p;
   double gam = p->Adiabatic_Index;
   double r = x[0];
   double rho = prim[RHO], vr = prim[URR], vp = prim[UPP]*r, vz = prim[UZZ];
   double Pp = prim[PPP];
   double om = get_om(p, x);
   double vp_off = vp - om*r;
   double v2 = vr*vr+vp_off*vp_off+vz*vz;
   double vn = vr*n[0] + vp*n[1] + vz*n[2];
   double vn_off = vn - om*r*n[1];
   double Ss_off = Ss + vn_off - vn;
   double rhoe = Pp/(gam - 1.);
   double rhostar = rho*(Sk - vn)/(Sk - Ss);
   double Pstar = Pp*(Ss - vn)/(Sk - Ss);
   double Us = rhoe*(Sk - vn)/(Sk - Ss);
   Ustar[DDD] = rhostar;
   Ustar[SRR] =   rhostar*( vr + (Ss-vn)*n[0] );
   Ustar[LLL] = r*rhostar*( vp + (Ss-vn)*n[1] );
   Ustar[SZZ] =   rhostar*( vz + (Ss-vn)*n[2] );
   Ustar[TAU] = .5*rhostar*v2 + Us + rhostar*Ss_off*(Ss - vn) + Pstar;
   int q;
   for( q=d->NC ; q<d->Q ; ++q ) Ustar[q] = prim[q]*Ustar[DDD];
}
static void cons2prim(const orc_domain *d, const double *cons, double *prim,
                      const double *x, double dV){            /* euler.c:102 */
   const disco_params *p = &d->p;
   double gam = p->Adiabatic_Index;
   double r = x[0];
   double rho = cons[DDD]/dV;
   if( rho < p->Density_Floor ) rho = p->Density_Floor;
   double Sr = cons[SRR]/dV;
   double Sp = cons[LLL]/dV/r;
   double Sz = cons[SZZ]/dV;
   double E  = cons[TAU]/dV;
   double om = get_om(p, x);
   double vr = Sr/rho;
   double vp = Sp/rho;
   double vp_off = vp - om*r;
   double vz = Sz/rho;
   double KE = .5*( Sr*vr + rho*vp_off*vp_off + Sz*vz );
   double rhoe = E-KE;
   double Pp = (gam - 1.)*rhoe;
   if( Pp < p->Pressure_Floor*rho ) Pp = p->Pressure_Floor*rho;
   if( p->isothermal_flag ){
      double cs2 = get_cs2(p, x);
      Pp = cs2*rho/gam;
   }
   prim[RHO] = rho;
   prim[PPP] = Pp;
   prim[URR] = vr;
   prim[UPP] = vp/r;
   prim[UZZ] = vz;
   int q;
   for( q=d->NC ; q<d->Q ; ++q ) prim[q] = cons[q]/cons[DDD];
}
static void flux(const orc_domain *d, const double *prim, double *F,
                 const double *x, const double *n){           /* euler.c:141 */
   const disco_params *p = &d->p;
   double gam = p->Adiabatic_Index;
   double r = x[0];
   double rho = prim[RHO], Pp = prim[PPP], vr = prim[URR];
   double vp = prim[UPP]*r, vz = prim[UZZ];
   double om = get_om(p, x);
   double vn = vr*n[0] + vp*n[1] + vz*n[2];
   double wn = om*r*n[1];
   double vp_off = vp - om*r;
   double rhoe = Pp/(gam - 1.);
   double v2 = vr*vr + vp_off*vp_off + vz*vz;
   F[DDD] = rho*vn;
   F[SRR] = rho*vr*vn + Pp*n[0];
   F[LLL] = r*(rho*vp*vn + Pp*n[1]);
   F[SZZ] = rho*vz*vn + Pp*n[2];
   F[TAU] = ( .5*rho*v2 + rhoe + Pp )*vn - Pp*wn;
   int q;
   for( q=d->NC ; q<d->Q ; ++q ) F[q] = prim[q]*F[DDD];
}
static void source(const orc_domain *d, const double *prim, double *cons,
                   const double *xp, const double *xm, double dVdt){ /* euler.c:171 */
   const disco_params *p = &d->p;
   double rp = xp[0], rm = xm[0];
   double rho = prim[RHO], Pp = prim[PPP];
   double r = get_centroid(rp, rm, 1);
   double z = get_centroid(xp[2], xm[2], 2);
   double r_1 = .5*(rp+rm);
   double vr = prim[URR], omega = prim[UPP], vz = prim[UZZ];
   double x[3] = {r, 0.5*(xm[1]+xp[1]), z};
   double centrifugal = rho*omega*omega*r;
   if( p->NoBC_Rmin == 1 ){                     /* polar_sources, euler.c:196 */
      double dphi = get_dp(xp[1], xm[1]);
      centrifugal *= sin(0.5*dphi) / (0.5*dphi);
   }
   double press_bal = Pp/r_1;
   cons[SRR] += dVdt*( centrifugal + press_bal );
   double om = get_om(p, x);
   double om_r = get_om1(p, x);
   double om_z = get_om2(p, x);
   cons[TAU] += dVdt*rho*( r*vr*om*om - r*r*(omega-om)*(vr*om_r + vz*om_z));
}
static void vel(const orc_domain *d, const double *prim1, const double *prim2,
                double *Sl, double *Sr, double *Ss, const double *n, const double *x){
   /* euler.c:305 */
   double gam = d->p.Adiabatic_Index;
   double r = x[0];
   double P1 = prim1[PPP], rho1 = prim1[RHO];
   double vn1 = prim1[URR]*n[0] + prim1[UPP]*n[1]*r + prim1[UZZ]*n[2];
   double cs1 = sqrt(gam*P1/rho1);
   double P2 = prim2[PPP], rho2 = prim2[RHO];
   double vn2 = prim2[URR]*n[0] + prim2[UPP]*n[1]*r + prim2[UZZ]*n[2];
   double cs2 = sqrt(gam*P2/rho2);
   *Ss = ( P2 - P1 + rho1*vn1*(-cs1) - rho2*vn2*cs2 )/( rho1*(-cs1) - rho2*cs2 );
   *Sr =  cs1 + vn1;
   *Sl = -cs1 + vn1;
   if( *Sr <  cs2 + vn2 ) *Sr =  cs2 + vn2;
   if( *Sl > -cs2 + vn2 ) *Sl = -cs2 + vn2;
}
static double mindt_cell(const orc_domain *d, const double *prim, double w,
                         const double *xp, const double *xm){  /* euler.c:332 */
   double gam = d->p.Adiabatic_Index;
   double r = get_centroid(xp[0], xm[0], 1);
   double Pp = prim[PPP], rho = prim[RHO];
   double vp = (prim[UPP]-w)*r;
   double vr = prim[URR], vz = prim[UZZ];
   double cs = sqrt(gam*Pp/rho);
   double maxvr = cs + fabs(vr);
   double maxvp = cs + fabs(vp);
   double maxvz = cs + fabs(vz);
   double dtr = get_dL(xp,xm,1)/maxvr;
   double dtp = get_dL(xp,xm,0)/maxvp;
   double dtz = get_dL(xp,xm,2)/maxvz;
   double dt = dtr;
   if( dt > dtp ) dt = dtp;
   if( dt > dtz ) dt = dtz;
   return dt;
}

/* ---------------------------------------------------------------- planets
 * planet.c:36-196, Planets/{sun,none,cm2}.c */
enum{PLPOINTMASS, PLPW, PLSURFACEGRAV};
/* planet.c:4: a mutable global, so the compiler cannot fold pow(r,n) into r*r
 * (glibc pow is not always correctly rounded, so the two can differ by an ulp) */
double orc_PHI_ORDER = 2.0;
static double fgrav(double M, double r, double eps, int type){  /* planet.c:56 */
   if( type == PLPOINTMASS ){
      double n = orc_PHI_ORDER;
      return( M*pow(r,n-1.)/pow( pow(r,n) + pow(eps,n) ,1.+1./n) );
   }
   return 0.0;
}
static void planetaryForce(const orc_domain *d, const orc_planet *pl, double r,
                           double phi, double z, double *fr, double *fp, double *fz){
   /* planet.c:99-150, mode 0 */
   double rp = pl->r, pp = pl->phi;
   if( d->p.grav2D == 1 ) z = 0.0;
   else if( d->p.grav2D == 2 ){ rp = r; pp = phi; z = 1.0; }
   double cosp = cos(phi), sinp = sin(phi);
   double dx = r*cosp-rp*cos(pp);
   double dy = r*sinp-rp*sin(pp);
   double script_r = sqrt(dx*dx+dy*dy+z*z);
   double script_r_perp = sqrt(dx*dx+dy*dy);
   double f1 = -fgrav( pl->M , script_r , pl->eps , pl->type );
   double cosa = dx/script_r_perp;
   double sina = dy/script_r_perp;
   double cosap = cosa*cosp+sina*sinp;
   double sinap = sina*cosp-cosa*sinp;
   if( script_r_perp <= 0.0 ){ cosap = 0.0; sinap = 0.0; }
   double sint = script_r_perp/script_r;
   double cost = z/script_r;
   *fr = cosap*f1*sint;
   *fp = sinap*f1*sint;
   *fz = f1*cost;
}
static void planet_src(const orc_domain *d, const orc_planet *pl, const double *prim,
                       double *cons, const double *xp, const double *xm, double dVdt){
   /* planet.c:152-196 (cylindrical: rpz maps are identities) */
   double rho = prim[RHO], vr = prim[URR], vz = prim[UZZ], omega = prim[UPP];
   double dphi = get_dp(xp[1],xm[1]);
   double phi = xm[1] + 0.5*dphi;
   double x[3] = {get_centroid(xp[0],xm[0],1), phi, get_centroid(xp[2],xm[2],2)};
   double F[3];
   planetaryForce(d, pl, x[0], x[1], x[2], &F[0], &F[1], &F[2]);
   double hr = 1.0, hp = x[0], hz = 1.0;
   if( d->p.NoBC_Rmin == 1 ){
      double adj = sin(0.5*dphi) / (0.5*dphi);
      F[0] *= adj; F[1] *= adj;
   }
   cons[SRR] += rho*hr*F[0]*dVdt;
   cons[LLL] += rho*hp*F[1]*dVdt;
   cons[SZZ] += rho*hz*F[2]*dVdt;
   cons[TAU] += rho*( hr*F[0]*vr + hz*F[2]*vz + hp*F[1]*omega )*dVdt;
}
static void init_planets(orc_domain *d){
   memset(d->pl, 0, sizeof d->pl);
   switch( d->m.planets ){
      case DISCO_PLANETS_SUN:                       /* Planets/sun.c:9-17 */
         d->Npl = 1; d->pl[0].M = 1.0; d->pl[0].type = PLPOINTMASS; break;
      case DISCO_PLANETS_CM2: {                     /* Planets/cm2.c:14-38 */
         d->Npl = 2;
         double a = 1.0, q = d->p.Mass_Ratio, mu = q/(1.+q), om = pow(a,-1.5);
         d->pl[0].M = 1.-mu; d->pl[0].omega = om; d->pl[0].r = a*mu; d->pl[0].phi = M_PI;
         d->pl[1].M = mu;    d->pl[1].omega = om; d->pl[1].r = a*(1.-mu);
         break; }
      case DISCO_PLANETS_BINARY_SOFT: {             /* new: equal-mass softened binary */
         d->Npl = 2;
         double a = d->p.initPar[5] > 0 ? d->p.initPar[5] : 1.0;
         double eps = d->p.initPar[6];
         double om = 1.0/(a*sqrt(a));
         d->pl[0].M = 0.5; d->pl[0].omega = om; d->pl[0].r = 0.5*a; d->pl[0].phi = M_PI; d->pl[0].eps = eps;
         d->pl[1].M = 0.5; d->pl[1].omega = om; d->pl[1].r = 0.5*a; d->pl[1].phi = 0.0;  d->pl[1].eps = eps;
         break; }
      default:                                       /* Planets/none.c:9-17 */
         d->Npl = 1; d->pl[0].M = 0.0; d->pl[0].eps = 1.0; d->pl[0].type = PLPOINTMASS; break;
   }
}
static int planets_move(const orc_domain *d){ return d->m.planets == DISCO_PLANETS_CM2 ||
                                                     d->m.planets == DISCO_PLANETS_BINARY_SOFT; }

/* ---------------------------------------------------------------- initial */
static void initial(const orc_domain *d, double *prim, const double *x){
   disco_ic_kepler_noise_eval(&d->ic, d->NC, d->Q, prim, x);
}

/* ---------------------------------------------------------------- helpers */
#define CELL(d,jk,i) ((d)->coff[jk] + (i))
#define PR(d,c)  ((d)->prim + (size_t)(c)*(d)->Q)
#define CO(d,c)  ((d)->cons + (size_t)(c)*(d)->Q)

orc_domain *orc_create(const disco_params *p, const disco_modules *m,
                       int Nr, int Nz, const int *Ng, const int *Np,
                       const double *r_jph, const double *z_kph){
   orc_domain *d = calloc(1, sizeof *d);
   d->p = *p; d->m = *m;
   d->Nr = Nr; d->Nz = Nz;
   d->NgRa = Ng[0]; d->NgRb = Ng[1]; d->NgZa = Ng[2]; d->NgZb = Ng[3];
   d->NC = m->num_c; d->Q = m->num_c + m->num_n;
   d->Np = malloc(sizeof(int)*Nr*Nz);
   memcpy(d->Np, Np, sizeof(int)*Nr*Nz);
   d->coff = malloc(sizeof(int)*(Nr*Nz+1));
   d->coff[0] = 0;
   int jk;
   for( jk=0 ; jk<Nr*Nz ; ++jk ) d->coff[jk+1] = d->coff[jk] + Np[jk];
   d->Ncell = d->coff[Nr*Nz];
   d->rj = malloc(sizeof(double)*(Nr+1)); memcpy(d->rj, r_jph, sizeof(double)*(Nr+1)); d->rj++;
   d->zk = malloc(sizeof(double)*(Nz+1)); memcpy(d->zk, z_kph, sizeof(double)*(Nz+1)); d->zk++;
   size_t nq = (size_t)d->Ncell*d->Q;
   d->prim = calloc(nq, sizeof(double)); d->cons = calloc(nq, sizeof(double));
   d->RKcons = calloc(nq, sizeof(double)); d->gradp = calloc(nq, sizeof(double));
   d->gradr = calloc(nq, sizeof(double)); d->gradz = calloc(nq, sizeof(double));
   d->piph = calloc(d->Ncell, sizeof(double)); d->dphi = calloc(d->Ncell, sizeof(double));
   d->wiph = calloc(d->Ncell, sizeof(double)); d->real = calloc(d->Ncell, sizeof(int));
   d->Ntr[1] = (Nr-1)*Nz;                                 /* faces_alt.c:5-8 */
   d->Ntr[2] = (Nz-1)*Nr;
   d->fI[1] = calloc(d->Ntr[1]+1, sizeof(int));
   d->fI[2] = calloc(d->Ntr[2]+1, sizeof(int));
   d->t = p->t_min;
   init_planets(d);
   d->nq = m->analysis == DISCO_DIAG_DISK2D ? 5 : 0;
   d->Qrz = calloc((size_t)Nr*Nz*(d->nq>0?d->nq:1), sizeof(double));
   d->ic.mach = p->Disk_Mach; d->ic.amp = p->initPar[1];
   d->ic.rmin = p->rmin; d->ic.rmax = p->rmax; d->ic.phimax = p->phimax;
   d->ic.seed = (uint64_t)(int64_t)p->initPar0;
   d->ic.kind = (int)p->initPar[2];
   return d;
}

void orc_destroy(orc_domain *d){
   if( !d ) return;
   free(d->Np); free(d->coff); free(d->rj-1); free(d->zk-1);
   free(d->prim); free(d->cons); free(d->RKcons); free(d->gradp); free(d->gradr); free(d->gradz);
   free(d->piph); free(d->dphi); free(d->wiph); free(d->real);
   free(d->fI[1]); free(d->fI[2]); free(d->F[1]); free(d->F[2]); free(d->Qrz);
   free(d);
}
int orc_ncell(const orc_domain *d){ return d->Ncell; }
double orc_time(const orc_domain *d){ return d->t; }

void orc_set_cells(orc_domain *d, const double *prim, const double *cons,
                   const double *piph, const double *dphi, const double *wiph,
                   const int *real){
   size_t nq = (size_t)d->Ncell*d->Q;
   if( prim ) memcpy(d->prim, prim, nq*sizeof(double));
   if( cons ) memcpy(d->cons, cons, nq*sizeof(double));
   if( piph ) memcpy(d->piph, piph, d->Ncell*sizeof(double));
   if( dphi ) memcpy(d->dphi, dphi, d->Ncell*sizeof(double));
   if( wiph ) memcpy(d->wiph, wiph, d->Ncell*sizeof(double));
   if( real ) memcpy(d->real, real, d->Ncell*sizeof(int));
}
void orc_get_cells(const orc_domain *d, double *prim, double *cons,
                   double *piph, double *dphi, double *wiph){
   size_t nq = (size_t)d->Ncell*d->Q;
   if( prim ) memcpy(prim, d->prim, nq*sizeof(double));
   if( cons ) memcpy(cons, d->cons, nq*sizeof(double));
   if( piph ) memcpy(piph, d->piph, d->Ncell*sizeof(double));
   if( dphi ) memcpy(dphi, d->dphi, d->Ncell*sizeof(double));
   if( wiph ) memcpy(wiph, d->wiph, d->Ncell*sizeof(double));
}
void orc_get_grad(const orc_domain *d, int which, double *out){
   const double *g = which==0 ? d->gradp : which==1 ? d->gradr : d->gradz;
   memcpy(out, g, (size_t)d->Ncell*d->Q*sizeof(double));
}

/* ---------------------------------------------------------------- misc.c */
static void clean_pi(orc_domain *d){                          /* misc.c:8-36 */
   int c, n;
   for( c=0 ; c<d->Ncell ; ++c ){
      double phi = d->piph[c];
      n = 0;
      while( phi > PMAX && n++ < WRAP_CAP ) phi -= PMAX;
      while( phi < 0.0  && n++ < WRAP_CAP ) phi += PMAX;
      d->piph[c] = phi;
   }
   int p;
   for( p=0 ; p<d->Npl ; ++p ){
      orc_planet *pl = d->pl + p;
      double phi = pl->phi;
      n = 0;
      while( phi > PMAX && n++ < WRAP_CAP ){ phi -= PMAX; pl->RK_phi -= PMAX; }
      while( phi < 0.0  && n++ < WRAP_CAP ){ phi += PMAX; pl->RK_phi += PMAX; }
      pl->phi = phi;
   }
}

double orc_mindt(orc_domain *d){                                 /* misc.c:39-84 */
   PMAX = d->p.phimax;
   double dt = d->p.maxDT / d->p.CFL;
   if( dt <= 0.0 ) dt = 1.0e100;
   int i, j, k;
   for( k=d->NgZa ; k<d->Nz-d->NgZb ; ++k )
   for( j=d->NgRa ; j<d->Nr-d->NgRb ; ++j ){
      int jk = j + d->Nr*k;
      for( i=0 ; i<d->Np[jk] ; ++i ){
         int c = CELL(d,jk,i);
         if( !d->real[c] ) continue;
         double phip = d->piph[c];
         double phim = phip - d->dphi[c];
         double xp[3] = {d->rj[j], phip, d->zk[k]};
         double xm[3] = {d->rj[j-1], phim, d->zk[k-1]};
         int im = i-1; if( i==0 ) im = d->Np[jk]-1;
         double wm = d->wiph[CELL(d,jk,im)];
         double wp = d->wiph[c];
         double w = .5*(wm+wp);
         double dt_temp = mindt_cell(d, PR(d,c), w, xp, xm);
         if( dt > dt_temp ) dt = dt_temp;
      }
   }
   dt *= d->p.CFL;
   return dt;
}

static void set_wcell(orc_domain *d){                            /* misc.c:101-168 */
   int mm = d->p.Mesh_Motion;
   int i, j, k;
   for( k=0 ; k<d->Nz ; ++k ){
      double z = get_centroid(d->zk[k], d->zk[k-1], 2);
      for( j=0 ; j<d->Nr ; ++j ){
         int jk = j + d->Nr*k;
         double r = get_centroid(d->rj[j], d->rj[j-1], 1);
         for( i=0 ; i<d->Np[jk] ; ++i ){
            int cL = CELL(d,jk,i);
            double w = 0.0;
            if( mm ){
               double phip = d->piph[cL];
               double phim = phip - d->dphi[cL];
               double x[3] = {r, 0.5*(phim+phip), z}; (void)x;
               double wL = PR(d,cL)[UPP];                /* get_omega, euler.c:32 */
               int ip = (i+1)%d->Np[jk];
               int cR = CELL(d,jk,ip);
               double wR = PR(d,cR)[UPP];
               w = .5*(wL + wR);
            }
            d->wiph[cL] = w;
         }
      }
   }
   if( mm == 3 ){
      for( k=0 ; k<d->Nz ; ++k ) for( j=0 ; j<d->Nr ; ++j ){
         int jk = j + d->Nr*k;
         double w = 0.0;
         for( i=0 ; i<d->Np[jk] ; ++i ) w += d->wiph[CELL(d,jk,i)];
         w /= (double)d->Np[jk];
         for( i=0 ; i<d->Np[jk] ; ++i ) d->wiph[CELL(d,jk,i)] = w;
      }
   }
   if( mm == 4 ){
      for( k=0 ; k<d->Nz ; ++k ){
         double z = get_centroid(d->zk[k], d->zk[k-1], 2);
         for( j=0 ; j<d->Nr ; ++j ){
            int jk = j + d->Nr*k;
            double r = get_centroid(d->rj[j], d->rj[j-1], 1);
            for( i=0 ; i<d->Np[jk] ; ++i ){
               int c = CELL(d,jk,i);
               double phip = d->piph[c], phim = phip - d->dphi[c];
               double x[3] = {r, 0.5*(phim+phip), z};
               d->wiph[c] = mesh_om(&d->p, x);
            }
         }
      }
   }
}

static void adjust_RK_cons(orc_domain *d, double RK){           /* misc.c:226-244 */
   size_t n, nq = (size_t)d->Ncell*d->Q;
   for( n=0 ; n<nq ; ++n ) d->cons[n] = (1.-RK)*d->cons[n] + RK*d->RKcons[n];
}
static void move_cells(orc_domain *d, double dt){               /* misc.c:256-268 */
   int c;
   for( c=0 ; c<d->Ncell ; ++c ) d->piph[c] += d->wiph[c]*dt;
}
static void calc_dp(orc_domain *d){                             /* misc.c:271-288 */
   int jk, i;
   for( jk=0 ; jk<d->Nr*d->Nz ; ++jk )
   for( i=0 ; i<d->Np[jk] ; ++i ){
      int im = i-1; if( i==0 ) im = d->Np[jk]-1;
      d->dphi[CELL(d,jk,i)] = get_dp(d->piph[CELL(d,jk,i)], d->piph[CELL(d,jk,im)]);
   }
}
static void calc_prim(orc_domain *d){                           /* misc.c:290-325 */
   int i, j, k;
   for( k=d->NgZa ; k<d->Nz-d->NgZb ; ++k ){
      double zm = d->zk[k-1], zp = d->zk[k];
      double z = get_centroid(zp, zm, 2);
      for( j=d->NgRa ; j<d->Nr-d->NgRb ; ++j ){
         int jk = j + d->Nr*k;
         double rm = d->rj[j-1], rp = d->rj[j];
         double r = get_centroid(rp, rm, 1);
         for( i=0 ; i<d->Np[jk] ; ++i ){
            int c = CELL(d,jk,i);
            double phip = d->piph[c], phim = phip - d->dphi[c];
            double xp[3] = {rp, phip, zp}, xm[3] = {rm, phim, zm};
            double dV = get_dV(xp, xm);
            double x[3] = {r, 0.5*(phim+phip), z};
            cons2prim(d, CO(d,c), PR(d,c), x, dV);
         }
      }
   }
}

/* ---------------------------------------------------------------- plm.c */
static double minmod(double a, double b, double c){             /* plm.c:6 */
   double m = a;
   if( a*b < 0.0 ) m = 0.0;
   if( fabs(b) < fabs(m) ) m = b;
   if( b*c < 0.0 ) m = 0.0;
   if( fabs(c) < fabs(m) ) m = c;
   return m;
}
static void plm_phi(orc_domain *d){                             /* plm.c:15-51 */
   double PLM = d->p.PLM;
   int jk, i, q, Q = d->Q;
   for( jk=0 ; jk<d->Nr*d->Nz ; ++jk ){
      int Np = d->Np[jk];
      for( i=0 ; i<Np ; ++i ){
         int im = i-1; if( im == -1 ) im = Np-1;
         int ip = (i+1)%Np;
         int c = CELL(d,jk,i), cl = CELL(d,jk,im), cr = CELL(d,jk,ip);
         double dpL = d->dphi[cl], dpC = d->dphi[c], dpR = d->dphi[cr];
         for( q=0 ; q<Q ; ++q ){
            double pL = PR(d,cl)[q], pC = PR(d,c)[q], pR = PR(d,cr)[q];
            double sL = pC - pL;  sL /= .5*( dpC + dpL );
            double sR = pR - pC;  sR /= .5*( dpR + dpC );
            double sC = pR - pL;  sC /= .5*( dpL + dpR ) + dpC;
            d->gradp[(size_t)c*Q+q] = minmod( PLM*sL , sC , PLM*sR );
         }
      }
   }
}

/* ---------------------------------------------------------------- faces_alt.c */
static void add_face(orc_domain *d, orc_face *F, int cL, int cR, double dxL, double dxR,
                     const double *xp, const double *xm, int dim, int LRtype){
   /* faces_alt.c:10-34 */
   double dp = get_dp(xp[1], xm[1]);
   double phic = get_dp(xp[1], .5*dp);
   double r = dim==1 ? 0.5*(xp[0]+xm[0]) : get_centroid(xp[0], xm[0], 1);
   double z = dim==2 ? 0.5*(xp[2]+xm[2]) : get_centroid(xp[2], xm[2], 2);
   F->cm[0] = r; F->cm[1] = phic; F->cm[2] = z;
   F->L = cL; F->R = cR; F->dxL = dxL; F->dxR = dxR;
   F->dphi = dp;
   F->dA = get_dA(xp, xm, dim);
   F->dl = get_dL(xp, xm, 3-dim);
   F->LRtype = LRtype;
   (void)d;
}

static void build_faces(orc_domain *d, int dim){                /* faces_alt.c:36-179 */
   int Nr = d->Nr, Nz = d->Nz;
   int i, j, k, jk;
   int *I0 = malloc(sizeof(int)*Nr*Nz);
   for( jk=0 ; jk<Nr*Nz ; ++jk ){                                 /* :59-79 */
      int found = 0, quad_prev = 0;
      for( i=0 ; i<d->Np[jk] && !found ; ++i ){
         double convert = 2.*M_PI/PMAX;
         double piph = d->piph[CELL(d,jk,i)];
         double sn = sin(piph*convert), cs = cos(piph*convert);
         if( sn>0. && cs>0. && quad_prev ){ quad_prev = 0; found = 1; I0[jk] = i; }
         else if( sn<0. && cs>0. ) quad_prev = 1;
      }
      if( !found ) I0[jk] = 0;
   }
   int Nrmax = dim==2 ? Nr : Nr-1;
   int Nzmax = dim==1 ? Nz : Nz-1;
   int *ntj = d->fI[dim];
   int n = 0;
   for( k=0 ; k<Nzmax ; ++k ) for( j=0 ; j<Nrmax ; ++j ){          /* :87-100 */
      int JK = j + Nrmax*k, jk0 = j + Nr*k;
      int jkp = dim==2 ? j + Nr*(k+1) : j+1 + Nr*k;
      ntj[JK] = n;
      n += d->Np[jk0] + d->Np[jkp];
   }
   ntj[Nrmax*Nzmax] = n;
   free(d->F[dim]);
   d->F[dim] = malloc(sizeof(orc_face)*(size_t)(n>0?n:1));
   orc_face *F = d->F[dim];
   n = 0;
   for( k=0 ; k<Nzmax ; ++k ) for( j=0 ; j<Nrmax ; ++j ){          /* :102-177 */
      int jp = j+1, kp = k+1;
      int jk0 = j + Nr*k;
      int jkp = dim==2 ? j + Nr*kp : jp + Nr*k;
      double dxL, dxR;
      if( dim==1 ){
         double rm = get_centroid(d->rj[j], d->rj[j-1], 1);
         double rp = get_centroid(d->rj[jp], d->rj[j], 1);
         dxL = d->rj[j] - rm; dxR = rp - d->rj[j];
      }else{
         double zm = get_centroid(d->zk[k], d->zk[k-1], 2);
         double zp = get_centroid(d->zk[kp], d->zk[k], 2);
         dxL = d->zk[k] - zm; dxR = zp - d->zk[k];
      }
      double xp[3] = {d->rj[j], 0.0, d->zk[k]};
      double xm[3] = {d->rj[j], 0.0, d->zk[k-1]};
      if( dim==2 ){ xm[0] = d->rj[j-1]; xm[2] = d->zk[k]; }
      int ia = I0[jk0], ib = I0[jkp];
      int f, NA = d->Np[jk0], NB = d->Np[jkp];
      for( f=0 ; f<NA+NB ; ++f ){
         int cL = CELL(d,jk0,ia), cR = CELL(d,jkp,ib);
         double dphi = d->piph[cL] - d->piph[cR];
         int w = 0;
         while( dphi > .5*PMAX && w++ < WRAP_CAP ) dphi -= PMAX;
         while( dphi <-.5*PMAX && w++ < WRAP_CAP ) dphi += PMAX;
         int LR = dphi > 0. ? 1 : 0;
         dphi = d->piph[cL]-d->dphi[cL] - d->piph[cR]+d->dphi[cR];
         w = 0;
         while( dphi > .5*PMAX && w++ < WRAP_CAP ) dphi -= PMAX;
         while( dphi <-.5*PMAX && w++ < WRAP_CAP ) dphi += PMAX;
         int LR_back = dphi < 0. ? 1 : 0;
         xp[1] = LR==0 ? d->piph[cL] : d->piph[cR];
         xm[1] = LR_back==0 ? d->piph[cL]-d->dphi[cL] : d->piph[cR]-d->dphi[cR];
         add_face(d, F+n, cL, cR, dxL, dxR, xp, xm, dim, LR);
         ++n;
         if( LR == 0 ){ ++ia; if( ia == NA ) ia = 0; }
         else         { ++ib; if( ib == NB ) ib = 0; }
      }
   }
   free(I0);
}

static void plm_trans(orc_domain *d, int dim){                  /* plm.c:56-195 */
   double PLM = d->p.PLM;
   int Q = d->Q, q, n;
   double *grad = dim==1 ? d->gradr : d->gradz;
   memset(grad, 0, sizeof(double)*(size_t)d->Ncell*Q);
   if( PLM == 0.0 ) return;
   int Nf = d->fI[dim][d->Ntr[dim]];
   orc_face *F = d->F[dim];
   for( n=0 ; n<Nf ; ++n ){
      orc_face *f = F+n;
      double phi = f->cm[1];
      int cL = f->L, cR = f->R;
      double phiL = d->piph[cL] - .5*d->dphi[cL];
      double phiR = d->piph[cR] - .5*d->dphi[cR];
      double dpL = get_signed_dp(phi, phiL);
      double dpR = get_signed_dp(phiR, phi);
      double dA = f->dA;
      for( q=0 ; q<Q ; ++q ){
         double WL = PR(d,cL)[q] + dpL*d->gradp[(size_t)cL*Q+q];
         double WR = PR(d,cR)[q] - dpR*d->gradp[(size_t)cR*Q+q];
         double S = (WR-WL)/(f->dxR+f->dxL);
         grad[(size_t)cL*Q+q] += S*dA;
         grad[(size_t)cR*Q+q] += S*dA;
      }
   }
   int i, j, k;
   for( j=0 ; j<d->Nr ; ++j ) for( k=0 ; k<d->Nz ; ++k ){
      int jk = j + d->Nr*k;
      for( i=0 ; i<d->Np[jk] ; ++i ){
         int c = CELL(d,jk,i);
         double phip = d->piph[c], phim = phip - d->dphi[c];
         double xp[3] = {d->rj[j], phip, d->zk[k]};
         double xm[3] = {d->rj[j-1], phim, d->zk[k-1]};
         if( dim==1 ) xm[0] = d->rj[j]; else xm[2] = d->zk[k];
         double dAp = get_dA(xp, xm, dim);
         if( dim==1 ){ xp[0] = d->rj[j-1]; xm[0] = d->rj[j-1]; }
         else        { xp[2] = d->zk[k-1]; xm[2] = d->zk[k-1]; }
         double dAm = get_dA(xp, xm, dim);
         double dAtot = dAp + dAm;
         if( (dim==1 && j==0) || (dim==2 && k==0) ) dAtot = dAp;
         if( (dim==1 && j==d->Nr-1) || (dim==2 && k==d->Nz-1) ) dAtot = dAm;
         for( q=0 ; q<Q ; ++q ) grad[(size_t)c*Q+q] /= dAtot;
      }
   }
   for( n=0 ; n<Nf ; ++n ){
      orc_face *f = F+n;
      double phi = f->cm[1];
      int cL = f->L, cR = f->R;
      double phiL = d->piph[cL] - .5*d->dphi[cL];
      double phiR = d->piph[cR] - .5*d->dphi[cR];
      double dpL = get_signed_dp(phi, phiL);
      double dpR = get_signed_dp(phiR, phi);
      for( q=0 ; q<Q ; ++q ){
         double WL = PR(d,cL)[q] + dpL*d->gradp[(size_t)cL*Q+q];
         double WR = PR(d,cR)[q] - dpR*d->gradp[(size_t)cR*Q+q];
         double S = (WR-WL)/(f->dxR+f->dxL);
         double *gL = grad + (size_t)cL*Q+q, *gR = grad + (size_t)cR*Q+q;
         double SL = *gL, SR = *gR;
         if( S*SL < 0.0 ) *gL = 0.0;
         else if( fabs(PLM*S) < fabs(SL) ) *gL = PLM*S;
         if( S*SR < 0.0 ) *gR = 0.0;
         else if( fabs(PLM*S) < fabs(SR) ) *gR = PLM*S;
      }
   }
   /* plm_geom_boundary only when NgRa==0 / NgZa==0 (NoBC): not in scope */
}

/* ---------------------------------------------------------------- riemann.c */
static void solve_riemann(orc_domain *d, const double *primL, const double *primR,
                          double *consL, double *consR, const double *x,
                          const double *n, double w, double dAdt){ /* riemann.c:216-318 */
   int q, Q = d->Q;
   double Flux[MAXQ], Ustr[MAXQ];
   for( q=0 ; q<Q ; ++q ){ Flux[q] = 0.0; Ustr[q] = 0.0; }
   double Sl, Sr, Ss;
   vel(d, primL, primR, &Sl, &Sr, &Ss, n, x);
   if( w < Sl ){
      flux(d, primL, Flux, x, n);
      prim2cons(d, primL, Ustr, x, 1.0);
   }else if( w > Sr ){
      flux(d, primR, Flux, x, n);
      prim2cons(d, primR, Ustr, x, 1.0);
   }else if( d->p.Riemann_Solver == 0 ){
      double Fl[MAXQ], Fr[MAXQ], Ul[MAXQ], Ur[MAXQ];
      double aL = Sr, aR = -Sl;
      prim2cons(d, primL, Ul, x, 1.0);
      prim2cons(d, primR, Ur, x, 1.0);
      flux(d, primL, Fl, x, n);
      flux(d, primR, Fr, x, n);
      for( q=0 ; q<Q ; ++q ){
         Flux[q] = ( aL*Fl[q] + aR*Fr[q] + aL*aR*( Ul[q] - Ur[q] ) )/( aL + aR );
         Ustr[q] = ( aR*Ul[q] + aL*Ur[q] + Fl[q] - Fr[q] )/( aL + aR );
      }
   }else{
      double Uk[MAXQ], Fk[MAXQ];
      if( w < Ss ){
         prim2cons(d, primL, Uk, x, 1.0);
         getUstar(d, primL, Ustr, x, Sl, Ss, n);
         flux(d, primL, Fk, x, n);
         for( q=0 ; q<Q ; ++q ) Flux[q] = Fk[q] + Sl*( Ustr[q] - Uk[q] );
      }else{
         prim2cons(d, primR, Uk, x, 1.0);
         getUstar(d, primR, Ustr, x, Sr, Ss, n);
         flux(d, primR, Fk, x, n);
         for( q=0 ; q<Q ; ++q ) Flux[q] = Fk[q] + Sr*( Ustr[q] - Uk[q] );
      }
   }
   for( q=0 ; q<Q ; ++q ){
      consL[q] -= (Flux[q] - w*Ustr[q])*dAdt;
      consR[q] += (Flux[q] - w*Ustr[q])*dAdt;
   }
}

static void phi_flux(orc_domain *d, double dt){                 /* misc.c:368-426 */
   int Q = d->Q, q, i, j, k;
   for( k=d->NgZa ; k<d->Nz-d->NgZb ; ++k ){
      double zp = d->zk[k], zm = d->zk[k-1];
      double z = get_centroid(zp, zm, 2);
      for( j=d->NgRa ; j<d->Nr-d->NgRb ; ++j ){
         double rp = d->rj[j], rm = d->rj[j-1];
         double r = get_centroid(rp, rm, 1);
         int jk = j + d->Nr*k;
         int Np = d->Np[jk];
         for( i=0 ; i<Np ; ++i ){
            int ip = i<Np-1 ? i+1 : 0;
            int cL = CELL(d,jk,i), cR = CELL(d,jk,ip);
            double phi = d->piph[cL];
            double xp[3] = {rp, phi, zp}, xm[3] = {rm, phi, zm};
            double dA = get_dA(xp, xm, 0);
            double x[3] = {r, phi, z};
            /* riemann_phi, riemann.c:39-112 */
            double primL[MAXQ], primR[MAXQ];
            for( q=0 ; q<Q ; ++q ){
               primL[q] = PR(d,cL)[q] + .5*d->gradp[(size_t)cL*Q+q]*d->dphi[cL];
               primR[q] = PR(d,cR)[q] - .5*d->gradp[(size_t)cR*Q+q]*d->dphi[cR];
            }
            double n[3] = {0.0, 1.0, 0.0};
            double hn = x[0];
            solve_riemann(d, primL, primR, CO(d,cL), CO(d,cR), x, n, hn*d->wiph[cL], dA*dt);
         }
      }
   }
}

static void trans_flux(orc_domain *d, double dt, int dim){      /* misc.c:431-509 */
   int Nr = d->Nr, Nz = d->Nz, Q = d->Q, q;
   int jmin, jmax, kmin, kmax, Nfr;
   if( dim==1 ){
      Nfr = Nr-1;
      jmin = d->NgRa==0 ? 0 : d->NgRa-1;
      jmax = d->NgRb==0 ? Nr-1 : Nr-d->NgRb;
      kmin = d->NgZa; kmax = Nz-d->NgZb;
   }else{
      Nfr = Nr;
      jmin = d->NgRa; jmax = Nr-d->NgRb;
      kmin = d->NgZa==0 ? 0 : d->NgZa-1;
      kmax = d->NgZb==0 ? Nz-1 : Nz-d->NgZb;
   }
   int j, k, f;
   for( k=kmin ; k<kmax ; ++k ) for( j=jmin ; j<jmax ; ++j ){
      int JK = j + Nfr*k;
      for( f=d->fI[dim][JK] ; f<d->fI[dim][JK+1] ; ++f ){
         /* riemann_trans, riemann.c:114-213 */
         orc_face *F = d->F[dim] + f;
         int cL = F->L, cR = F->R;
         double dAdt = F->dA*dt;
         double dxL = F->dxL, dxR = F->dxR, phi = F->cm[1];
         double phiL = d->piph[cL] - .5*d->dphi[cL];
         double phiR = d->piph[cR] - .5*d->dphi[cR];
         double dpL = get_signed_dp(phi, phiL);
         double dpR = get_signed_dp(phiR, phi);
         const double *gL = (dim==1 ? d->gradr : d->gradz) + (size_t)cL*Q;
         const double *gR = (dim==1 ? d->gradr : d->gradz) + (size_t)cR*Q;
         double primL[MAXQ], primR[MAXQ];
         for( q=0 ; q<Q ; ++q ){
            primL[q] = PR(d,cL)[q] + gL[q]*dxL + d->gradp[(size_t)cL*Q+q]*dpL;
            primR[q] = PR(d,cR)[q] - gR[q]*dxR - d->gradp[(size_t)cR*Q+q]*dpR;
         }
         double n[3] = {0.0, 0.0, 0.0};
         if( dim==1 ) n[0] = 1.0; else n[2] = 1.0;
         solve_riemann(d, primL, primR, CO(d,cL), CO(d,cR), F->cm, n, 0.0, dAdt);
      }
   }
}

static void add_source(orc_domain *d, double dt){               /* misc.c:538-580 */
   int i, j, k, p;
   for( k=d->NgZa ; k<d->Nz-d->NgZb ; ++k )
   for( j=d->NgRa ; j<d->Nr-d->NgRb ; ++j ){
      int jk = j + d->Nr*k;
      for( i=0 ; i<d->Np[jk] ; ++i ){
         int c = CELL(d,jk,i);
         double phip = d->piph[c], phim = d->piph[c] - d->dphi[c];
         double xp[3] = {d->rj[j], phip, d->zk[k]};
         double xm[3] = {d->rj[j-1], phim, d->zk[k-1]};
         double dV = get_dV(xp, xm);
         source(d, PR(d,c), CO(d,c), xp, xm, dV*dt);
         for( p=0 ; p<d->Npl ; ++p ) planet_src(d, d->pl+p, PR(d,c), CO(d,c), xp, xm, dV*dt);
         /* visc_source (off), omega_src (RotFrame 0: no-op, rotframe.c:32),
          * sink_src (Nozzle_Type 0: no-op, sink.c:35) */
      }
   }
}

/* ---------------------------------------------------------------- boundaries */
static void boundary_fixed(orc_domain *d, int dim){             /* Boundary/fixed.c:11-60 */
   if( dim != 1 ) return;
   int j, k, i;
   for( j=d->Nr-1 ; j>d->Nr-1-d->NgRb ; --j ) for( k=0 ; k<d->Nz ; ++k ){
      int jk = j + d->Nr*k;
      for( i=0 ; i<d->Np[jk] ; ++i ){
         int c = CELL(d,jk,i);
         double phi = d->piph[c] - .5*d->dphi[c];
         double x[3] = { .5*(d->rj[j]+d->rj[j-1]), phi, .5*(d->zk[k]+d->zk[k-1]) };
         initial(d, PR(d,c), x);
      }
   }
   for( j=0 ; j<d->NgRa ; ++j ) for( k=0 ; k<d->Nz ; ++k ){
      int jk = j + d->Nr*k;
      for( i=0 ; i<d->Np[jk] ; ++i ){
         int c = CELL(d,jk,i);
         double phi = d->piph[c] - .5*d->dphi[c];
         double x[3] = { .5*(d->rj[j]+d->rj[j-1]), phi, .5*(d->zk[k]+d->zk[k-1]) };
         initial(d, PR(d,c), x);
      }
   }
}

static void boundary_trans(orc_domain *d, int dim){
   if( d->m.boundary == DISCO_BC_FIXED ) boundary_fixed(d, dim);
}

/* ---------------------------------------------------------------- analysis.c */
static void add_diagnostics(orc_domain *d, double dt){          /* analysis.c:52-107 */
   int Nq = d->nq;
   if( Nq == 0 ){ d->t_avg += dt; return; }
   int NN = d->Nr*d->Nz;
   double *tsum = calloc((size_t)NN*Nq, sizeof(double));
   double *tvol = calloc((size_t)NN, sizeof(double));
   int i, j, k, q;
   for( k=0 ; k<d->Nz ; ++k ) for( j=0 ; j<d->Nr ; ++j ){
      int jk = k*d->Nr + j;
      for( i=0 ; i<d->Np[jk] ; ++i ){
         int c = CELL(d,jk,i);
         double phip = d->piph[c], phim = phip - d->dphi[c];
         double xp[3] = {d->rj[j], phip, d->zk[k]}, xm[3] = {d->rj[j-1], phim, d->zk[k-1]};
         double xc[3];
         for( q=0 ; q<3 ; ++q ) xc[q] = .5*(xp[q]+xm[q]);
         double dV = get_dV(xp, xm);
         /* get_diagnostics, Diagnostics/diag_disk2d.c:17-38 */
         const double *prim = PR(d,c);
         double r = xc[0], phi = xc[1];
         double rho = prim[RHO], vr = prim[URR], omega = prim[UPP];
         double Qd[5];
         Qd[0] = rho;
         Qd[1] = 2.*M_PI*r*rho*vr;
         double Fr, Fp = 0.0, Fz;
         if( d->Npl > 1 ) planetaryForce(d, d->pl+1, r, phi, 0.0, &Fr, &Fp, &Fz);
         Qd[2] = 2.*M_PI*r*rho*(r*Fp);
         Qd[3] = 2.*M_PI*r*rho*( r*r*omega*vr );
         Qd[4] = omega;
         for( q=0 ; q<Nq ; ++q ) tsum[jk*Nq+q] += Qd[q]*dV;
         tvol[jk] += dV;
      }
   }
   for( k=0 ; k<d->Nz ; ++k ) for( j=0 ; j<d->Nr ; ++j ){
      int jk = k*d->Nr + j;
      for( q=0 ; q<Nq ; ++q ) d->Qrz[jk*Nq+q] += tsum[jk*Nq+q]*dt / tvol[jk];
   }
   d->t_avg += dt;
   free(tsum); free(tvol);
}

void orc_get_diagnostics(const orc_domain *d, double *Qrz, double *t_avg){
   if( Qrz ) memcpy(Qrz, d->Qrz, sizeof(double)*(size_t)d->Nr*d->Nz*d->nq);
   if( t_avg ) *t_avg = d->t_avg;
}

/* ---------------------------------------------------------------- onestep.c */
static void onestep(orc_domain *d, double RK, double dt, int first_step, int last_step){
   (void)last_step;                                               /* onestep.c:84-229 */
   if( first_step ) set_wcell(d);
   adjust_RK_cons(d, RK);
   plm_phi(d);
   if( d->Nr > 1 ){ build_faces(d, 1); plm_trans(d, 1); }
   if( d->Nz > 1 ){ build_faces(d, 2); plm_trans(d, 2); }
   phi_flux(d, dt);
   if( d->Nr > 1 ) trans_flux(d, dt, 1);
   if( d->Nz > 1 ) trans_flux(d, dt, 2);
   add_source(d, dt);
   if( first_step ) move_cells(d, dt);
   if( !1 || first_step ){                   /* planet_motion_analytic() == 1 */
      int p;
      for( p=0 ; p<d->Npl ; ++p ){           /* planet_RK_adjust, planet.c:206 */
         orc_planet *pl = d->pl+p;
         pl->r     = (1.-RK)*pl->r     + RK*pl->RK_r;
         pl->phi   = (1.-RK)*pl->phi   + RK*pl->RK_phi;
         pl->M     = (1.-RK)*pl->M     + RK*pl->RK_M;
         pl->omega = (1.-RK)*pl->omega + RK*pl->RK_omega;
         pl->vr    = (1.-RK)*pl->vr    + RK*pl->RK_vr;
      }
      if( planets_move(d) )                  /* Planets/cm2.c:40-43 */
         for( p=0 ; p<d->Npl ; ++p ) d->pl[p].phi += d->pl[p].omega*dt;
   }
   clean_pi(d);
   calc_dp(d);
   calc_prim(d);
   if( !d->p.R_Periodic ) boundary_trans(d, 1);
   if( d->Nz > 1 && !d->p.Z_Periodic ) boundary_trans(d, 2);
}

void orc_timestep(orc_domain *d, double dt){                     /* timestep.c:7-45 */
   PMAX = d->p.phimax;
   memcpy(d->RKcons, d->cons, sizeof(double)*(size_t)d->Ncell*d->Q);
   int p;
   for( p=0 ; p<d->Npl ; ++p ){                                     /* planet.c:198 */
      orc_planet *pl = d->pl+p;
      pl->RK_r = pl->r; pl->RK_phi = pl->phi; pl->RK_M = pl->M;
      pl->RK_omega = pl->omega; pl->RK_vr = pl->vr;
   }
   if( d->p.Timestep == 1 ){
      onestep(d, 0.0, dt, 1, 1);
      d->t += dt;
   }else{
      onestep(d, 0.0, dt, 1, 0);
      d->t += dt;
      onestep(d, 0.5, 0.5*dt, 0, 1);
   }
   add_diagnostics(d, dt);
   d->count_steps += 1;
}

int orc_get_faces(orc_domain *d, int dim, int *fIndex, int *iL, int *iR,
                  int *LRtype, double *geom){
   PMAX = d->p.phimax;
   if( dim==1 && d->Nr < 2 ) return 0;
   if( dim==2 && d->Nz < 2 ) return 0;
   build_faces(d, dim);
   int NN = d->Ntr[dim];
   int Nf = d->fI[dim][NN];
   if( fIndex ) memcpy(fIndex, d->fI[dim], sizeof(int)*(NN+1));
   int n;
   for( n=0 ; n<Nf ; ++n ){
      orc_face *F = d->F[dim] + n;
      if( iL ) iL[n] = F->L;
      if( iR ) iR[n] = F->R;
      if( LRtype ) LRtype[n] = F->LRtype;
      if( geom ){
         double *g = geom + 8*(size_t)n;
         g[0] = F->dxL; g[1] = F->dxR; g[2] = F->cm[0]; g[3] = F->cm[1];
         g[4] = F->cm[2]; g[5] = F->dphi; g[6] = F->dl; g[7] = F->dA;
      }
   }
   return Nf;
}

int orc_stage(orc_domain *d, const char *s, double RK, double dt){
   PMAX = d->p.phimax;
   if( !strcmp(s, "wcell") ) set_wcell(d);
   else if( !strcmp(s, "snapshot") ) memcpy(d->RKcons, d->cons, sizeof(double)*(size_t)d->Ncell*d->Q);
   else if( !strcmp(s, "adjust_rk") ) adjust_RK_cons(d, RK);
   else if( !strcmp(s, "plm_phi") ) plm_phi(d);
   else if( !strcmp(s, "faces_r") ) build_faces(d, 1);
   else if( !strcmp(s, "plm_r") ) plm_trans(d, 1);
   else if( !strcmp(s, "flux_phi") ) phi_flux(d, dt);
   else if( !strcmp(s, "flux_r") ) trans_flux(d, dt, 1);
   else if( !strcmp(s, "source") ) add_source(d, dt);
   else if( !strcmp(s, "move") ) move_cells(d, dt);
   else if( !strcmp(s, "clean_dp") ){ clean_pi(d); calc_dp(d); }
   else if( !strcmp(s, "c2p") ) calc_prim(d);
   else if( !strcmp(s, "boundary") ) boundary_trans(d, 1);
   else return -1;
   return 0;
}
