/*
 * Device-side physics of the B200 Disco timestep.
 *
 * Per-state algebra of the selected modules, written with the same
 * floating-point operation order as the reference so that, compiled with
 * --fmad=false, everything except libm calls (pow/sin/cos/exp) rounds
 * exactly as the serial CPU build does:
 *   geometry  Geometry/cylindrical.c:10-63
 *   omega     omega.c:43-141
 *   euler     Hydro/euler.c:36-380
 *   planets   planet.c:36-196, Planets/{sun,none,cm2}.c
 * Phi-wrap loops are bounded (the reference's are not, misc.c:22-23,
 * cylindrical.c:12-13) and raise DISCO_ERR_PHI_WRAP in the batch error word.
 */
#pragma once
#include <stdint.h>
#include "ic_kepler_noise.h"

namespace disco {

#define DISCO_PI 3.14159265358979323846
#define WRAP_CAP 64
#define MAXPL 2

enum { RHO = 0, PPP = 1, URR = 2, UPP = 3, UZZ = 4, BRR = 5, BPP = 6, BZZ = 7 };
enum { DDD = 0, TAU = 1, SRR = 2, LLL = 3, SZZ = 4 };
enum { ERRF_WRAP = 1, ERRF_NONFINITE = 2 };

struct Planet {
   double r, phi, M, omega, vr;
   double RK_r, RK_phi, RK_M, RK_omega, RK_vr;
   double eps;
   int type;
   int pad;
};

/* Per-disk constants (read-only inside a step). */
struct DiskParams {
   double gam, PLM, CFL, maxDT, Pmax;
   double rho_floor, p_floor;
   double RotOmega, Mach, Cs2_M, Cs2_H0, Cs2_r1;
   int mesh_motion, riemann, en_om, mesh_om, isothermal, cs2_profile;
   int grav2D, polar, timestep, planets_move, rotframe;
   int Nr, Nz, NgRa, NgRb, NgZa, NgZb;
   int ann0;          /* first global annulus of the disk */
   int rj0, zk0;      /* offset of r_jph[-1] / z_kph[-1] in the global arrays */
   int cell0;         /* first global cell */
   int trr0, ntrr;    /* first global r-track, count */
   int face_r0;       /* first global r-face */
   int npl;
   disco_ic_kepler_noise ic;
};

/* Per-disk mutable state (device resident across steps). */
struct DiskState {
   double t;
   double dt;                    /* dt of the step in flight */
   unsigned long long dtmin;     /* bits of the running min (positive doubles) */
   double dt_next;               /* getmindt of the current state */
   double t_avg;
   int count_steps;
   int pad;
   Planet pl[MAXPL];
};

/* ------------------------------------------------------------ geometry */
__device__ __forceinline__ double get_dp(double phip, double phim, double Pmax, int *err){
   double dp = phip - phim;
   int n = 0;
   while( dp < 0.0 ){ dp += Pmax; if( ++n > WRAP_CAP ){ *err |= ERRF_WRAP; break; } }
   while( dp > Pmax ){ dp -= Pmax; if( ++n > WRAP_CAP ){ *err |= ERRF_WRAP; break; } }
   return dp;
}
__device__ __forceinline__ double get_signed_dp(double phip, double phim, double Pmax, int *err){
   double dp = phip - phim;
   int n = 0;
   while( dp < -.5*Pmax ){ dp += Pmax; if( ++n > WRAP_CAP ){ *err |= ERRF_WRAP; break; } }
   while( dp >  .5*Pmax ){ dp -= Pmax; if( ++n > WRAP_CAP ){ *err |= ERRF_WRAP; break; } }
   return dp;
}
/* cylindrical.c:24-30; the sum is spelled with round-to-nearest intrinsics so
 * that no translation unit (the mixed form is built with FMA contraction)
 * turns it into an FMA: the mesh must be the same in every form. */
__device__ __forceinline__ double centroid_r(double xp, double xm){
   double s = __dadd_rn(__dadd_rn(__dmul_rn(xp, xp), __dmul_rn(xp, xm)), __dmul_rn(xm, xm));
   return 2.0*s / (3.0*(xp+xm));
}
__device__ __forceinline__ double centroid_z(double xp, double xm){ return 0.5*(xp+xm); }
/* get_dV(xp,xm) given dphi = get_dp(xp1,xm1) already evaluated */
__device__ __forceinline__ double dV_of(double rp, double rm, double dphi, double zp, double zm){
   double r = .5*(rp+rm);
   double dr = rp-rm;
   double dz = zp-zm;
   return r*dr*dphi*dz;
}

/* ------------------------------------------------------------ omega.c */
__device__ __forceinline__ double get_om(const DiskParams &P, double r){
   double O0 = P.RotOmega;
   switch( P.en_om ){
      case 1: return 1.0-O0;
      case 2: return 1.0/pow(r,1.5)-O0;
      case 3: { double n = 8.0; return 1./pow( pow( r , 1.5*n ) + 1. , 1./n )-O0; }
      case 4: return 10.*exp(-.5*r*r)-O0;
      default: return 0.0-O0;
   }
}
__device__ __forceinline__ double get_om1(const DiskParams &P, double r){
   switch( P.en_om ){
      case 1: return 0.0;
      case 2: return -1.5/pow(r,2.5);
      case 3: { double n = 8.0;
                return -1.5 * pow(r,-1+1.5*n) / pow( pow(r,1.5*n) + 1. , 1.0+1./n ); }
      case 4: return 10.*r*exp(-.5*r*r);
      default: return 0.0;
   }
}
__device__ __forceinline__ double get_cs2(const DiskParams &P, double r){
   double Mach = P.Mach;
   switch( P.cs2_profile ){
      case 1: return 1./(Mach*Mach);
      case 2: { double nu = .5; return .5/Mach/Mach/pow(r,2.*nu); }
      case 3: return P.Cs2_M*P.Cs2_H0*P.Cs2_H0 / (2*P.Cs2_r1*P.Cs2_r1*P.Cs2_r1);
      case 4: { double v2 = P.Cs2_M/r; return v2/(Mach*Mach); }
      default: return 1.0;
   }
}
__device__ __forceinline__ double mesh_om(const DiskParams &P, double r){
   if( P.mesh_om == 1 ) return 1.0;
   if( P.mesh_om == 2 ) return pow(r,-1.5);
   if( P.mesh_om == 3 ){ double n = 8.0; return 1./pow( pow( r , 1.5*n ) + 1. , 1./n ); }
   return 0.0;
}

/* ------------------------------------------------------------ euler.c
 * Templated on the bulk real type R: R = double is the reference's FP64
 * arithmetic (constants written R(...) so the double instantiation rounds
 * exactly as before); R = float is the mixed form's FP32 flux arithmetic.
 * r is the radius used by the state algebra and om = get_om(x) there. */
template<int Q, int NC, class R>
__device__ __forceinline__ void prim2cons(const DiskParams &P, const R *prim, R *cons,
                                          R r, R om, R dV){
   const R gam = (R)P.gam;
   R rho = prim[RHO], Pp = prim[PPP], vr = prim[URR];
   R vp = prim[UPP]*r, vz = prim[UZZ];
   R vp_off = vp - om*r;
   R v2 = vr*vr + vp_off*vp_off + vz*vz;
   R rhoe = Pp/(gam - R(1.));
   cons[DDD] = rho*dV;
   cons[TAU] = (R(.5)*rho*v2 + rhoe )*dV;
   cons[SRR] = rho*vr*dV;
   cons[LLL] = r*rho*vp*dV;
   cons[SZZ] = rho*vz*dV;
#pragma unroll
   for( int q=NC ; q<Q ; ++q ) cons[q] = prim[q]*cons[DDD];
}

/* cons2prim (euler.c:102-139), always FP64 */
template<int Q, int NC>
__device__ __forceinline__ void cons2prim(const DiskParams &P, const double *cons, double *prim,
                                          double r, double om, double dV){
   double rho = cons[DDD]/dV;
   if( rho < P.rho_floor ) rho = P.rho_floor;
   double Sr = cons[SRR]/dV;
   double Sp = cons[LLL]/dV/r;
   double Sz = cons[SZZ]/dV;
   double E  = cons[TAU]/dV;
   double vr = Sr/rho;
   double vp = Sp/rho;
   double vp_off = vp - om*r;
   double vz = Sz/rho;
   double KE = .5*( Sr*vr + rho*vp_off*vp_off + Sz*vz );
   double rhoe = E-KE;
   double Pp = (P.gam - 1.)*rhoe;
   if( Pp < P.p_floor*rho ) Pp = P.p_floor*rho;
   if( P.isothermal ){
      double cs2 = get_cs2(P, r);
      Pp = cs2*rho/P.gam;
   }
   prim[RHO] = rho;
   prim[PPP] = Pp;
   prim[URR] = vr;
   prim[UPP] = vp/r;
   prim[UZZ] = vz;
#pragma unroll
   for( int q=NC ; q<Q ; ++q ) prim[q] = cons[q]/cons[DDD];
}

/* flux(), euler.c:141, for a normal n = e_dim (dim 0: phi, 1: r, 2: z) */
template<int Q, int NC, int DIM, class R>
__device__ __forceinline__ void flux(const DiskParams &P, const R *prim, R *F, R r, R om){
   const R n0 = DIM==1 ? R(1.0) : R(0.0), n1 = DIM==0 ? R(1.0) : R(0.0), n2 = DIM==2 ? R(1.0) : R(0.0);
   const R gam = (R)P.gam;
   R rho = prim[RHO], Pp = prim[PPP], vr = prim[URR];
   R vp = prim[UPP]*r, vz = prim[UZZ];
   R vn = vr*n0 + vp*n1 + vz*n2;
   R wn = om*r*n1;
   R vp_off = vp - om*r;
   R rhoe = Pp/(gam - R(1.));
   R v2 = vr*vr + vp_off*vp_off + vz*vz;
   F[DDD] = rho*vn;
   F[SRR] = rho*vr*vn + Pp*n0;
   F[LLL] = r*(rho*vp*vn + Pp*n1);
   F[SZZ] = rho*vz*vn + Pp*n2;
   F[TAU] = ( R(.5)*rho*v2 + rhoe + Pp )*vn - Pp*wn;
#pragma unroll
   for( int q=NC ; q<Q ; ++q ) F[q] = prim[q]*F[DDD];
}

/* getUstar(), euler.c:64 */
template<int Q, int NC, int DIM, class R>
__device__ __forceinline__ void getUstar(const DiskParams &P, const R *prim, R *Ustar,
                                         R r, R om, R Sk, R Ss){
   const R n0 = DIM==1 ? R(1.0) : R(0.0), n1 = DIM==0 ? R(1.0) : R(0.0), n2 = DIM==2 ? R(1.0) : R(0.0);
   const R gam = (R)P.gam;
   R rho = prim[RHO], vr = prim[URR], vp = prim[UPP]*r, vz = prim[UZZ];
   R Pp = prim[PPP];
   R vp_off = vp - om*r;
   R v2 = vr*vr+vp_off*vp_off+vz*vz;
   R vn = vr*n0 + vp*n1 + vz*n2;
   R vn_off = vn - om*r*n1;
   R Ss_off = Ss + vn_off - vn;
   R rhoe = Pp/(gam - R(1.));
   R rhostar = rho*(Sk - vn)/(Sk - Ss);
   R Pstar = Pp*(Ss - vn)/(Sk - Ss);
   R Us = rhoe*(Sk - vn)/(Sk - Ss);
   Ustar[DDD] = rhostar;
   Ustar[SRR] =   rhostar*( vr + (Ss-vn)*n0 );
   Ustar[LLL] = r*rhostar*( vp + (Ss-vn)*n1 );
   Ustar[SZZ] =   rhostar*( vz + (Ss-vn)*n2 );
   Ustar[TAU] = R(.5)*rhostar*v2 + Us + rhostar*Ss_off*(Ss - vn) + Pstar;
#pragma unroll
   for( int q=NC ; q<Q ; ++q ) Ustar[q] = prim[q]*Ustar[DDD];
}

/* vel(), euler.c:305 */
template<int DIM, class R>
__device__ __forceinline__ void vel(const DiskParams &P, const R *p1, const R *p2,
                                    R r, R *Sl, R *Sr, R *Ss){
   const R n0 = DIM==1 ? R(1.0) : R(0.0), n1 = DIM==0 ? R(1.0) : R(0.0), n2 = DIM==2 ? R(1.0) : R(0.0);
   const R gam = (R)P.gam;
   R P1 = p1[PPP], rho1 = p1[RHO];
   R vn1 = p1[URR]*n0 + p1[UPP]*n1*r + p1[UZZ]*n2;
   R cs1 = sqrt(gam*P1/rho1);
   R P2 = p2[PPP], rho2 = p2[RHO];
   R vn2 = p2[URR]*n0 + p2[UPP]*n1*r + p2[UZZ]*n2;
   R cs2 = sqrt(gam*P2/rho2);
   *Ss = ( P2 - P1 + rho1*vn1*(-cs1) - rho2*vn2*cs2 )/( rho1*(-cs1) - rho2*cs2 );
   *Sr =  cs1 + vn1;
   *Sl = -cs1 + vn1;
   if( *Sr <  cs2 + vn2 ) *Sr =  cs2 + vn2;
   if( *Sl > -cs2 + vn2 ) *Sl = -cs2 + vn2;
}

/* solve_riemann(), riemann.c:216-318, HLL / HLLC.  Returns
 * G_q = (Flux_q - w*Ustr_q)*dAdt, the amount subtracted from cons_L and
 * added to cons_R (riemann.c:312-315). */
template<int Q, int NC, int DIM, class R>
__device__ __forceinline__ void solve_riemann(const DiskParams &P, const R *primL,
                                              const R *primR, R r, R om,
                                              R w, R dAdt, R *G){
   R Flux[Q], Ustr[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){ Flux[q] = R(0.0); Ustr[q] = R(0.0); }
   R Sl, Sr, Ss;
   vel<DIM,R>(P, primL, primR, r, &Sl, &Sr, &Ss);
   if( w < Sl ){
      flux<Q,NC,DIM,R>(P, primL, Flux, r, om);
      prim2cons<Q,NC,R>(P, primL, Ustr, r, om, R(1.0));
   }else if( w > Sr ){
      flux<Q,NC,DIM,R>(P, primR, Flux, r, om);
      prim2cons<Q,NC,R>(P, primR, Ustr, r, om, R(1.0));
   }else if( P.riemann == 0 ){
      R Fl[Q], Fr[Q], Ul[Q], Ur[Q];
      R aL = Sr, aR = -Sl;
      prim2cons<Q,NC,R>(P, primL, Ul, r, om, R(1.0));
      prim2cons<Q,NC,R>(P, primR, Ur, r, om, R(1.0));
      flux<Q,NC,DIM,R>(P, primL, Fl, r, om);
      flux<Q,NC,DIM,R>(P, primR, Fr, r, om);
#pragma unroll
      for( int q=0 ; q<Q ; ++q ){
         Flux[q] = ( aL*Fl[q] + aR*Fr[q] + aL*aR*( Ul[q] - Ur[q] ) )/( aL + aR );
         Ustr[q] = ( aR*Ul[q] + aL*Ur[q] + Fl[q] - Fr[q] )/( aL + aR );
      }
   }else{
      R Uk[Q], Fk[Q];
      const R *pk = (w < Ss) ? primL : primR;
      R Sk = (w < Ss) ? Sl : Sr;
      prim2cons<Q,NC,R>(P, pk, Uk, r, om, R(1.0));
      getUstar<Q,NC,DIM,R>(P, pk, Ustr, r, om, Sk, Ss);
      flux<Q,NC,DIM,R>(P, pk, Fk, r, om);
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) Flux[q] = Fk[q] + Sk*( Ustr[q] - Uk[q] );
   }
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) G[q] = (Flux[q] - w*Ustr[q])*dAdt;
}

/* ------------------------------------------------------------ planets */
__device__ __forceinline__ double fgrav(double M, double r, double eps, int type){
   if( type == 0 ){                                   /* PLPOINTMASS, planet.c:58 */
      double n = 2.0;
      return( M*pow(r,n-1.)/pow( pow(r,n) + pow(eps,n) ,1.+1./n) );
   }
   return 0.0;
}
/* planetaryForce(), planet.c:99-150, mode 0 */
__device__ __forceinline__ void planetary_force(int grav2D, const Planet &pl, double r,
                                                double phi, double z, double *fr,
                                                double *fp, double *fz){
   double rp = pl.r, pp = pl.phi;
   if( grav2D == 1 ) z = 0.0;
   else if( grav2D == 2 ){ rp = r; pp = phi; z = 1.0; }
   double cosp = cos(phi), sinp = sin(phi);
   double dx = r*cosp-rp*cos(pp);
   double dy = r*sinp-rp*sin(pp);
   double script_r = sqrt(dx*dx+dy*dy+z*z);
   double script_r_perp = sqrt(dx*dx+dy*dy);
   double f1 = -fgrav( pl.M , script_r , pl.eps , pl.type );
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

/* ------------------------------------------------------------ initial */
template<int Q, int NC>
__device__ __forceinline__ void initial(const DiskParams &P, double *prim, const double *x){
   disco_ic_kepler_noise_eval(&P.ic, NC, Q, prim, x);
}

/* positive doubles order like their bit patterns */
__device__ __forceinline__ unsigned long long dbits(double x){
   return (unsigned long long)__double_as_longlong(x);
}

} // namespace disco
