/*
 * Device-side physics of the B200 Disco timestep.
 *
 * Per-state algebra of the selected modules, written with the same
 * floating-point operation order as the reference so that, compiled with
 * --fmad=false, everything except libm calls (pow/sin/cos/exp) rounds
 * exactly as the serial CPU build does:
 *   geometry  Geometry/cylindrical.c:10-63
 *   omega     omega.c:43-141
 *   euler     Hydro/euler.c:36-380              (NC == 5)
 *   mhd       Hydro/mhd.c:35-486, hlld.c:20-401 (NC == 8; no CT: B evolves
 *             as a conserved variable through the fluxes, as CT_MODE 0 does)
 *   planets   planet.c:36-196, Planets/{sun,none,cm2}.c
 * Phi-wrap loops are bounded (the reference's are not, misc.c:22-23,
 * cylindrical.c:12-13) and raise DISCO_ERR_PHI_WRAP in the batch error word.
 */
#pragma once
#include <stdint.h>
#include "ic_kepler_noise.h"
#include "ic_mhd_shear.h"
#include "ic_gr_torus.h"

namespace disco {

#define DISCO_PI 3.14159265358979323846
#define WRAP_CAP 64
#define MAXPL 2

enum { RHO = 0, PPP = 1, URR = 2, UPP = 3, UZZ = 4, BRR = 5, BPP = 6, BZZ = 7 };
enum { DDD = 0, TAU = 1, SRR = 2, LLL = 3, SZZ = 4 };
enum { ERRF_WRAP = 1, ERRF_NONFINITE = 2, ERRF_INTERNAL = 4,
       ERRF_TIMEOUT = 8 /* a bounded device wait ran out (persistent step) */ };

struct Planet {
   double r, phi, M, omega, vr;
   double RK_r, RK_phi, RK_M, RK_omega, RK_vr;
   double eps;
   double cphi, sphi;    /* cos(phi), sin(phi), set on the device whenever phi changes */
   int type;
   int pad;
};

/* Per-cell-block diagnostic partials: up to 18 quantities of the Analysis
 * module (diag_disk2d 5, diag_euler 8, diag_mhdmri 18) and the volume in
 * the last slot. */
#define DIAG_SLOTS 19
#define DIAG_VOL 18

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
   int trz0, ntrz;    /* first global z-track, count (Nr*(Nz-1)) */
   int ln0;           /* first global (r, z) edge line, (Nr-1)*(Nz-1) of them (3D CT) */
   int atmos;         /* Include_Atmos: adjust_gas at set-up */
   int visc, visc_alpha;  /* Use_Viscosity, Use_As_Alpha (euler.c:217-295) */
   int pl_eps_decay, pad_pl;  /* Planets/cm.c: eps = pl_smooth + exp(-t/30) when moved */
   double pl_smooth;
   double visc_nu;        /* Viscosity: nu, or alpha */
   int noise_type;    /* Noise_Type 0..3 (addNoise) */
   int pad_noise;
   double noise_abs, noise_rel;
   int npl;
   int ic_module;     /* 0 kepler_noise, 1 mhd_shear_noise, 2 gr_torus_noise */
   int pad_ic;
   disco_ic_kepler_noise ic;
   disco_ic_mhd_shear ic_mhd;
   disco_ic_gr_torus ic_gr;
   /* grmhd2 (HYDRO = grmhd2): the metric module (0 schw_ks_rpz, 1 the
    * Kerr-Schild kerr_ks_rpz) and its Metric_Par2 (M) / Metric_Par3 (a) */
   int gr, gr_metric;
   double gr_M, gr_a;
   int bc_horizon;    /* 8 (Boundary/horizon.c) or 9 (horizon3d) when cells are excised, else 0 */
   int side_fixed;    /* bc 11: the fixed sides (bit 0 inner r, 1 outer r, 2 lower z, 3 upper z) */
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
   if constexpr ( NC == 8 ){                         /* mhd.c:35-68 */
      R Br = prim[BRR], Bp = prim[BPP], Bz = prim[BZZ];
      R B2 = Br*Br + Bp*Bp + Bz*Bz;
      cons[TAU] = (R(.5)*rho*v2 + rhoe + R(.5)*B2 )*dV;
      cons[BRR] = Br*dV * (R(1.0)/r);                /* bfield_scale_factor(r,0) */
      cons[BPP] = Bp*dV/r;
      cons[BZZ] = Bz*dV;
   }else{
      cons[TAU] = (R(.5)*rho*v2 + rhoe )*dV;
   }
   cons[SRR] = rho*vr*dV;
   cons[LLL] = r*rho*vp*dV;
   cons[SZZ] = rho*vz*dV;
#pragma unroll
   for( int q=NC ; q<Q ; ++q ) cons[q] = prim[q]*cons[DDD];
}

/* cons2prim (euler.c:102-139; mhd.c:138-185), always FP64 */
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
   double Br = 0.0, Bp = 0.0, Bz = 0.0, B2 = 0.0;
   if constexpr ( NC == 8 ){
      Br = cons[BRR]/(dV * (1.0/r));
      Bp = cons[BPP]/dV*r;
      Bz = cons[BZZ]/dV;
      B2 = Br*Br+Bp*Bp+Bz*Bz;
   }
   double KE = .5*( Sr*vr + rho*vp_off*vp_off + Sz*vz );
   double rhoe;
   if constexpr ( NC == 8 ) rhoe = E-KE-.5*B2;
   else rhoe = E-KE;
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
   if constexpr ( NC == 8 ){ prim[BRR] = Br; prim[BPP] = Bp; prim[BZZ] = Bz; }
#pragma unroll
   for( int q=NC ; q<Q ; ++q ) prim[q] = cons[q]/cons[DDD];
}

/* flux(), euler.c:141 / mhd.c:187-223, for a normal n = e_dim (dim 0: phi,
 * 1: r, 2: z) */
template<int Q, int NC, int DIM, class R>
__device__ __forceinline__ void flux(const DiskParams &P, const R *prim, R *F, R r, R om){
   const R n0 = DIM==1 ? R(1.0) : R(0.0), n1 = DIM==0 ? R(1.0) : R(0.0), n2 = DIM==2 ? R(1.0) : R(0.0);
   const R gam = (R)P.gam;
   R rho = prim[RHO], Pp = prim[PPP], vr = prim[URR];
   R vp = prim[UPP]*r, vz = prim[UZZ];
   R vn = vr*n0 + vp*n1 + vz*n2;
   R rhoe = Pp/(gam - R(1.));
   if constexpr ( NC == 8 ){
      R Br = prim[BRR], Bp = prim[BPP], Bz = prim[BZZ];
      R Bn = Br*n0 + Bp*n1 + Bz*n2;
      R vB = vr*Br + vp*Bp + vz*Bz;
      R v2 = vr*vr + vp*vp + vz*vz;
      R B2 = Br*Br + Bp*Bp + Bz*Bz;
      F[DDD] = rho*vn;
      F[SRR] =     rho*vr*vn + (Pp+R(.5)*B2)*n0 - Br*Bn;
      F[LLL] = r*( rho*vp*vn + (Pp+R(.5)*B2)*n1 - Bp*Bn );
      F[SZZ] =     rho*vz*vn + (Pp+R(.5)*B2)*n2 - Bz*Bn;
      F[TAU] = ( R(.5)*rho*v2 + rhoe + Pp + B2 )*vn - vB*Bn;
      F[BRR] = (Br*vn - vr*Bn) * (R(1.0)/r);
      F[BPP] = (Bp*vn - vp*Bn)/r;
      F[BZZ] = Bz*vn - vz*Bn;
   }else{
      R wn = om*r*n1;
      R vp_off = vp - om*r;
      R v2 = vr*vr + vp_off*vp_off + vz*vz;
      F[DDD] = rho*vn;
      F[SRR] = rho*vr*vn + Pp*n0;
      F[LLL] = r*(rho*vp*vn + Pp*n1);
      F[SZZ] = rho*vz*vn + Pp*n2;
      F[TAU] = ( R(.5)*rho*v2 + rhoe + Pp )*vn - Pp*wn;
   }
#pragma unroll
   for( int q=NC ; q<Q ; ++q ) F[q] = prim[q]*F[DDD];
}

/* getUstar(), euler.c:64 / mhd.c:70-136 (Bpack from the MHD vel) */
template<int Q, int NC, int DIM, class R>
__device__ __forceinline__ void getUstar(const DiskParams &P, const R *prim, R *Ustar,
                                         R r, R om, R Sk, R Ss, const R *Bpack){
   const R n0 = DIM==1 ? R(1.0) : R(0.0), n1 = DIM==0 ? R(1.0) : R(0.0), n2 = DIM==2 ? R(1.0) : R(0.0);
   const R gam = (R)P.gam;
   if constexpr ( NC == 8 ){
      R Bsn = Bpack[0], Bsr = Bpack[1], Bsp = Bpack[2], Bsz = Bpack[3], vBs = Bpack[4];
      R rho = prim[RHO], vr = prim[URR], vp = prim[UPP]*r, vz = prim[UZZ], Pp = prim[PPP];
      R Br = prim[BRR], Bp = prim[BPP], Bz = prim[BZZ];
      R v2 = vr*vr+vp*vp+vz*vz;
      R B2 = Br*Br+Bp*Bp+Bz*Bz;
      R vn = vr*n0 + vp*n1 + vz*n2;
      R Bn = Br*n0 + Bp*n1 + Bz*n2;
      R vB = vr*Br   + vp*Bp   + vz*Bz;
      R rhoe = Pp/(gam-R(1.));
      R D  = rho;
      R mr = rho*vr, mp = rho*vp, mz = rho*vz;
      R E  = R(.5)*rho*v2 + rhoe + R(.5)*B2;
      R Bs2 = Bsr*Bsr+Bsp*Bsp+Bsz*Bsz;
      R Ps  = rho*( Sk - vn )*( Ss - vn ) + (Pp+R(.5)*B2-Bn*Bn) - R(.5)*Bs2 + Bsn*Bsn;
      R Dstar = ( Sk - vn )*D/( Sk - Ss );
      R Msr   = ( ( Sk - vn )*mr + ( Br*Bn - Bsr*Bsn ) ) / ( Sk - Ss );
      R Msp   = ( ( Sk - vn )*mp + ( Bp*Bn - Bsp*Bsn ) ) / ( Sk - Ss );
      R Msz   = ( ( Sk - vn )*mz + ( Bz*Bn - Bsz*Bsn ) ) / ( Sk - Ss );
      R Estar = ( ( Sk - vn )*E + (Ps+R(.5)*Bs2)*Ss - (Pp+R(.5)*B2)*vn - vBs*Bsn + vB*Bn ) / ( Sk - Ss );
      R Msn = Dstar*Ss;
      R mn  = Msr*n0 + Msp*n1 + Msz*n2;
      Msr += n0*( Msn - mn );
      Msp += n1*( Msn - mn );
      Msz += n2*( Msn - mn );
      Ustar[DDD] = Dstar;
      Ustar[SRR] = Msr;
      Ustar[LLL] = r*Msp;
      Ustar[SZZ] = Msz;
      Ustar[TAU] = Estar;
      Ustar[BRR] = Bsr * (R(1.0)/r);
      Ustar[BPP] = Bsp/r;
      Ustar[BZZ] = Bsz;
   }else{
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
   }
#pragma unroll
   for( int q=NC ; q<Q ; ++q ) Ustar[q] = prim[q]*Ustar[DDD];
}

/* vel(), euler.c:305 / mhd.c:318-450 (fast magnetosonic bounds and the HLL
 * average of B and momentum in Bpack) */
template<int NC, int DIM, class R>
__device__ __forceinline__ void vel(const DiskParams &P, const R *p1, const R *p2,
                                    R r, R *Sl, R *Sr, R *Ss, R *Bpack){
   const R n0 = DIM==1 ? R(1.0) : R(0.0), n1 = DIM==0 ? R(1.0) : R(0.0), n2 = DIM==2 ? R(1.0) : R(0.0);
   const R gam = (R)P.gam;
   if constexpr ( NC == 8 ){
      R L_Mins, L_Plus, L_Star;
      R P1 = p1[PPP], rho1 = p1[RHO];
      R vr1 = p1[URR], vp1 = r*p1[UPP], vz1 = p1[UZZ];
      R vn1 = vr1*n0 + vp1*n1 + vz1*n2;
      R cs1 = sqrt( gam*(P1/rho1) );
      R Br1 = p1[BRR], Bp1 = p1[BPP], Bz1 = p1[BZZ];
      R Bn1 = Br1*n0 + Bp1*n1 + Bz1*n2;
      R B21 = (Br1*Br1 + Bp1*Bp1 + Bz1*Bz1);
      R b21 = B21/rho1;
      R FrL = vn1*Br1 - Bn1*vr1, FpL = vn1*Bp1 - Bn1*vp1, FzL = vn1*Bz1 - Bn1*vz1;
      R mrL = rho1*vr1, mpL = rho1*vp1, mzL = rho1*vz1;
      R FmrL = rho1*vr1*vn1 + (P1+R(.5)*B21)*n0 - Br1*Bn1;
      R FmpL = rho1*vp1*vn1 + (P1+R(.5)*B21)*n1 - Bp1*Bn1;
      R FmzL = rho1*vz1*vn1 + (P1+R(.5)*B21)*n2 - Bz1*Bn1;
      R cf21 = R(.5)*( cs1*cs1 + b21 + sqrt(fabs( (cs1*cs1+b21)*(cs1*cs1+b21) - R(4.0)*cs1*cs1*Bn1*Bn1/rho1 )) );
      L_Mins = vn1 - sqrt( cf21 );
      L_Plus = vn1 + sqrt( cf21 );
      R P2 = p2[PPP], rho2 = p2[RHO];
      R vr2 = p2[URR], vp2 = r*p2[UPP], vz2 = p2[UZZ];
      R vn2 = vr2*n0 + vp2*n1 + vz2*n2;
      R cs2 = sqrt( gam*(P2/rho2) );
      R Br2 = p2[BRR], Bp2 = p2[BPP], Bz2 = p2[BZZ];
      R Bn2 = Br2*n0 + Bp2*n1 + Bz2*n2;
      R B22 = (Br2*Br2 + Bp2*Bp2 + Bz2*Bz2);
      R b22 = B22/rho2;
      R FrR = vn2*Br2 - Bn2*vr2, FpR = vn2*Bp2 - Bn2*vp2, FzR = vn2*Bz2 - Bn2*vz2;
      R mrR = rho2*vr2, mpR = rho2*vp2, mzR = rho2*vz2;
      R FmrR = rho2*vr2*vn2 + (P2+R(.5)*B22)*n0 - Br2*Bn2;
      R FmpR = rho2*vp2*vn2 + (P2+R(.5)*B22)*n1 - Bp2*Bn2;
      R FmzR = rho2*vz2*vn2 + (P2+R(.5)*B22)*n2 - Bz2*Bn2;
      R cf22 = R(.5)*( cs2*cs2 + b22 + sqrt(fabs( (cs2*cs2+b22)*(cs2*cs2+b22) - R(4.0)*cs2*cs2*Bn2*Bn2/rho2 )) );
      if( L_Mins > vn2 - sqrt( cf22 ) ) L_Mins = vn2 - sqrt( cf22 );
      if( L_Plus < vn2 + sqrt( cf22 ) ) L_Plus = vn2 + sqrt( cf22 );
      R aL = L_Plus;
      R aR = -L_Mins;
      R Br = ( aR*Br1 + aL*Br2 + FrL - FrR )/( aL + aR );
      R Bp = ( aR*Bp1 + aL*Bp2 + FpL - FpR )/( aL + aR );
      R Bz = ( aR*Bz1 + aL*Bz2 + FzL - FzR )/( aL + aR );
      R Bn = Br*n0 + Bp*n1 + Bz*n2;
      R mr = ( aR*mrL + aL*mrR + FmrL - FmrR )/( aL + aR );
      R mp = ( aR*mpL + aL*mpR + FmpL - FmpR )/( aL + aR );
      R mz = ( aR*mzL + aL*mzR + FmzL - FmzR )/( aL + aR );
      R mnL = mrL*n0+mpL*n1+mzL*n2;
      R mnR = mrR*n0+mpR*n1+mzR*n2;
      R rho = ( aR*rho1 + aL*rho2 + mnL - mnR )/( aL + aR );
      L_Star = ( rho2*vn2*(L_Plus-vn2) - rho1*vn1*(L_Mins-vn1) + (P1+R(.5)*B21-Bn1*Bn1)
                 - (P2+R(.5)*B22-Bn2*Bn2) )/( rho2*(L_Plus-vn2) - rho1*(L_Mins-vn1) );
      R vr = mr/rho, vp = mp/rho, vz = mz/rho;
      R vdotB = vr*Br + vp*Bp + vz*Bz;
      Bpack[0] = Bn; Bpack[1] = Br; Bpack[2] = Bp; Bpack[3] = Bz; Bpack[4] = vdotB;
      *Sl = L_Mins;
      *Sr = L_Plus;
      *Ss = L_Star;
   }else{
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
}

/* ------------------------------------------------------------ HLLD
 * hlld.c:20-401 in the frame of the face: velocities scaled to physical
 * units (u_phi *= r), fluxes and star states scaled back; pow(x, 2.) is
 * written x*x (gcc -O3 emits exactly that multiply for it). */
#define HLLD_TOL 1e-10

template<class R>
__device__ __forceinline__ void hlld_velocities(const DiskParams &P, const R *pL, const R *pR,
                                                R n0, R n1, R n2, R *vel, R *Pt_star){
   const R gam = (R)P.gam;
   R rho_L = pL[RHO], P_L = pL[PPP];
   R u_L  = pL[URR]*n0 + pL[UPP]*n1 + pL[UZZ]*n2;
   R Bn_L = pL[BRR]*n0 + pL[BPP]*n1 + pL[BZZ]*n2;
   R B2_L = pL[BRR]*pL[BRR] + pL[BPP]*pL[BPP] + pL[BZZ]*pL[BZZ];
   R Pt_L = P_L + R(.5)*B2_L;
   R rho_R = pR[RHO], P_R = pR[PPP];
   R u_R  = pR[URR]*n0 + pR[UPP]*n1 + pR[UZZ]*n2;
   R Bn_R = pR[BRR]*n0 + pR[BPP]*n1 + pR[BZZ]*n2;
   R B2_R = pR[BRR]*pR[BRR] + pR[BPP]*pR[BPP] + pR[BZZ]*pR[BZZ];
   R Pt_R = P_R + R(.5)*B2_R;
   R Bn = R(.5)*(Bn_L+Bn_R);
   R aL = gam*P_L + B2_L, aR = gam*P_R + B2_R;
   R cf2_L = R(.5)*(gam*P_L + B2_L + sqrt( fabs( aL*aL - R(4.)*gam*P_L*Bn_L*Bn_L ) ) )/rho_L;
   R cf2_R = R(.5)*(gam*P_R + B2_R + sqrt( fabs( aR*aR - R(4.)*gam*P_R*Bn_R*Bn_R ) ) )/rho_R;
   R cf2 = cf2_L > cf2_R ? cf2_L : cf2_R;
   R umin, umax;
   if( u_L < u_R ){ umin = u_L; umax = u_R; }else{ umin = u_R; umax = u_L; }
   R S_R = umax + sqrt(fabs(cf2));
   R S_L = umin - sqrt(fabs(cf2));
   R S_M = ( ( S_R - u_R )*rho_R*u_R - ( S_L - u_L )*rho_L*u_L - Pt_R + Pt_L )
           /( ( S_R - u_R )*rho_R - (S_L-u_L)*rho_L );
   R rhostar_L = rho_L*( S_L - u_L )/( S_L - S_M );
   R rhostar_R = rho_R*( S_R - u_R )/( S_R - S_M );
   R Ss_L = S_M - fabs(Bn)/sqrt(rhostar_L);
   R Ss_R = S_M + fabs(Bn)/sqrt(rhostar_R);
   vel[0] = S_L; vel[1] = Ss_L; vel[2] = S_M; vel[3] = Ss_R; vel[4] = S_R;
   R num   = ( S_R - u_R )*rho_R*Pt_L - ( S_L - u_L )*rho_L*Pt_R
             + rho_L*rho_R*( S_R - u_R )*( S_L - u_L )*( u_R - u_L );
   R denom = ( S_R - u_R )*rho_R - ( S_L - u_L )*rho_L;
   *Pt_star = num/denom;
}

template<class R>
__device__ __forceinline__ void hlld_prim_to_cons(const DiskParams &P, const R *prim, R *cons){
   const R gam = (R)P.gam;
   R rho = prim[RHO], Pp = prim[PPP], vx = prim[URR], vy = prim[UPP], vz = prim[UZZ];
   R Bx = prim[BRR], By = prim[BPP], Bz = prim[BZZ];
   R v2 = vx*vx + vy*vy + vz*vz;
   R rhoe = Pp/(gam-R(1.));
   R B2 = Bx*Bx + By*By + Bz*Bz;
   cons[DDD] = rho;
   cons[SRR] = rho*vx;
   cons[LLL] = rho*vy;
   cons[SZZ] = rho*vz;
   cons[TAU] = ( R(.5)*rho*v2 + rhoe + R(.5)*B2 );
   cons[BRR] = Bx; cons[BPP] = By; cons[BZZ] = Bz;
}

template<class R>
__device__ __forceinline__ void hlld_flux(const DiskParams &P, const R *prim, R *flux,
                                         R n0, R n1, R n2){
   const R gam = (R)P.gam;
   R rho = prim[RHO], Pp = prim[PPP], vx = prim[URR], vy = prim[UPP], vz = prim[UZZ];
   R Bx = prim[BRR], By = prim[BPP], Bz = prim[BZZ];
   R v2 = vx*vx+vy*vy+vz*vz;
   R vB = vx*Bx + vy*By + vz*Bz;
   R B2 = Bx*Bx + By*By + Bz*Bz;
   R vn = vx*n0 + vy*n1 + vz*n2;
   R Bn = Bx*n0 + By*n1 + Bz*n2;
   R rhoe = Pp/(gam-R(1.));
   flux[DDD] = rho*vn;
   flux[SRR] = rho*vx*vn + ( Pp + R(.5)*B2 )*n0 - Bx*Bn;
   flux[LLL] = rho*vy*vn + ( Pp + R(.5)*B2 )*n1 - By*Bn;
   flux[SZZ] = rho*vz*vn + ( Pp + R(.5)*B2 )*n2 - Bz*Bn;
   flux[TAU] = (R(.5)*rho*v2 + rhoe + Pp + B2 )*vn - vB*Bn;
   flux[BRR] = Bx*vn - vx*Bn;
   flux[BPP] = By*vn - vy*Bn;
   flux[BZZ] = Bz*vn - vz*Bn;
}

template<class R>
__device__ __forceinline__ void hlld_single_star(const DiskParams &P, const R *prim, R *Ustar,
                                                R S_K, R S_M, R Pt_star, R n0, R n1, R n2){
   const R gam = (R)P.gam;
   R rho = prim[RHO], vx = prim[URR], vy = prim[UPP], vz = prim[UZZ], Pp = prim[PPP];
   R Bx = prim[BRR], By = prim[BPP], Bz = prim[BZZ];
   R u_K   = vx*n0 + vy*n1 + vz*n2;
   R Bn    = Bx*n0 + By*n1 + Bz*n2;
   R vdotB = vx*Bx + vy*By + vz*Bz;
   R v2    = vx*vx + vy*vy + vz*vz;
   R B2    = Bx*Bx + By*By + Bz*Bz;
   R Pt = Pp + R(.5)*B2;
   R e = R(.5)*rho*v2 + Pp/(gam-R(1.)) + R(.5)*B2;
   R rhostar = rho*( S_K - u_K )/( S_K - S_M );
   R denom = rho*(S_K-u_K)*(S_K-S_M) - Bn*Bn ;
   if( fabs(denom) < R(HLLD_TOL) ) denom = R(HLLD_TOL);
   R vx_star = vx - Bn*Bx*( S_M - u_K )/denom;
   R vy_star = vy - Bn*By*( S_M - u_K )/denom;
   R vz_star = vz - Bn*Bz*( S_M - u_K )/denom;
   R sk2 = (S_K-u_K)*(S_K-u_K);
   R Bx_star = Bx*( rho*sk2 - Bn*Bn )/denom;
   R By_star = By*( rho*sk2 - Bn*Bn )/denom;
   R Bz_star = Bz*( rho*sk2 - Bn*Bn )/denom;
   R vn_star = vx_star*n0 + vy_star*n1 + vz_star*n2;
   R Bn_star = Bx_star*n0 + By_star*n1 + Bz_star*n2;
   vx_star += ( S_M - vn_star )*n0;
   vy_star += ( S_M - vn_star )*n1;
   vz_star += ( S_M - vn_star )*n2;
   Bx_star += ( Bn  - Bn_star )*n0;
   By_star += ( Bn  - Bn_star )*n1;
   Bz_star += ( Bn  - Bn_star )*n2;
   R vBstar = vx_star*Bx_star + vy_star*By_star + vz_star*Bz_star;
   R e_star = ( (S_K-u_K)*e - Pt*u_K + Pt_star*S_M + Bn*( vdotB - vBstar ) )/( S_K - S_M );
   Ustar[DDD] = rhostar;
   Ustar[SRR] = rhostar*vx_star;
   Ustar[LLL] = rhostar*vy_star;
   Ustar[SZZ] = rhostar*vz_star;
   Ustar[TAU] = e_star;
   Ustar[BRR] = Bx_star; Ustar[BPP] = By_star; Ustar[BZZ] = Bz_star;
}

template<class R>
__device__ __forceinline__ void hlld_double_star(const R *UsL, const R *UsR, R *Uss, const R *vel,
                                                R n0, R n1, R n2, int LR){
   R rho_L = UsL[DDD], rho_R = UsR[DDD];
   R rhostar_K = LR == 0 ? rho_L : rho_R;
   R rrh_L = sqrt( rho_L ), rrh_R = sqrt( rho_R ), rrh_K = sqrt( rhostar_K );
   R Sx_L = UsL[SRR], Sy_L = UsL[LLL], Sz_L = UsL[SZZ];
   R Bx_L = UsL[BRR], By_L = UsL[BPP], Bz_L = UsL[BZZ];
   R vx_L = Sx_L/rho_L, vy_L = Sy_L/rho_L, vz_L = Sz_L/rho_L;
   R Sx_R = UsR[SRR], Sy_R = UsR[LLL], Sz_R = UsR[SZZ];
   R Bx_R = UsR[BRR], By_R = UsR[BPP], Bz_R = UsR[BZZ];
   R vx_R = Sx_R/rho_R, vy_R = Sy_R/rho_R, vz_R = Sz_R/rho_R;
   R Bn_L = Bx_L*n0 + By_L*n1 + Bz_L*n2;
   R Bn_R = Bx_R*n0 + By_R*n1 + Bz_R*n2;
   R Bn = R(.5)*(Bn_L+Bn_R);
   R signBn = Bn > R(0.0) ? R(1.0) : R(-1.0);
   R denom = rrh_L+rrh_R;
   R vx_ss = ( rrh_L*vx_L + rrh_R*vx_R + ( Bx_R - Bx_L )*signBn )/denom;
   R vy_ss = ( rrh_L*vy_L + rrh_R*vy_R + ( By_R - By_L )*signBn )/denom;
   R vz_ss = ( rrh_L*vz_L + rrh_R*vz_R + ( Bz_R - Bz_L )*signBn )/denom;
   R vn_ss = vx_ss*n0+vy_ss*n1+vz_ss*n2;
   vx_ss += (vel[2]-vn_ss)*n0;
   vy_ss += (vel[2]-vn_ss)*n1;
   vz_ss += (vel[2]-vn_ss)*n2;
   R Bx_ss = ( rrh_L*Bx_R + rrh_R*Bx_L + rrh_L*rrh_R*( vx_R - vx_L )*signBn )/denom;
   R By_ss = ( rrh_L*By_R + rrh_R*By_L + rrh_L*rrh_R*( vy_R - vy_L )*signBn )/denom;
   R Bz_ss = ( rrh_L*Bz_R + rrh_R*Bz_L + rrh_L*rrh_R*( vz_R - vz_L )*signBn )/denom;
   R Bn_ss = Bx_ss*n0+By_ss*n1+Bz_ss*n2;
   Bx_ss += (Bn-Bn_ss)*n0;
   By_ss += (Bn-Bn_ss)*n1;
   Bz_ss += (Bn-Bn_ss)*n2;
   R vB_ss = vx_ss*Bx_ss + vy_ss*By_ss + vz_ss*Bz_ss;
   R vBstar, e_star;
   if( LR == 0 ){ vBstar = vx_L*Bx_L + vy_L*By_L + vz_L*Bz_L; e_star = UsL[TAU]; }
   else         { vBstar = vx_R*Bx_R + vy_R*By_R + vz_R*Bz_R; e_star = UsR[TAU]; }
   R plusminus = LR == 1 ? R(1.0) : R(-1.0);
   R e_ss = e_star + plusminus*rrh_K*( vBstar - vB_ss )*signBn;
   Uss[DDD] = rhostar_K;
   Uss[SRR] = rhostar_K*vx_ss;
   Uss[LLL] = rhostar_K*vy_ss;
   Uss[SZZ] = rhostar_K*vz_ss;
   Uss[TAU] = e_ss;
   Uss[BRR] = Bx_ss; Uss[BPP] = By_ss; Uss[BZZ] = Bz_ss;
}

/* get_Ustar_HLLD (hlld.c:279-401): F and U of the face */
template<int Q, int DIM, class R>
__device__ __forceinline__ void hlld_solve(const DiskParams &P, R w, const R *primL,
                                          const R *primR, R *F, R *U, R r){
   const R n0 = DIM==1 ? R(1.0) : R(0.0), n1 = DIM==0 ? R(1.0) : R(0.0), n2 = DIM==2 ? R(1.0) : R(0.0);
   const R hr = R(1.0), hp = r, hz = R(1.0);      /* get_scale_factor(x, 1 / 0 / 2) */
   R pL[Q], pR[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){ pL[q] = primL[q]; pR[q] = primR[q]; }
   pL[URR] *= hr; pR[URR] *= hr;
   pL[UPP] *= hp; pR[UPP] *= hp;
   pL[UZZ] *= hz; pR[UZZ] *= hz;
   R vel[5], Pt_star;
   hlld_velocities<R>(P, pL, pR, n0, n1, n2, vel, &Pt_star);
   /* The two sides of the contact run the same operations on mirrored
    * inputs, so they are one code path here on the side K the face's frame
    * lies on (left: w < S_M) and the other side O: neighbouring faces on
    * different sides (w close to S_M, the common case on a moving mesh) do
    * not serialise the warp, and every value is the one the branch of that
    * side computes. */
   const bool left = w < vel[2];
   R pK[Q], pO[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){ pK[q] = left ? pL[q] : pR[q]; pO[q] = left ? pR[q] : pL[q]; }
   const R S_K = left ? vel[0] : vel[4], S_O = left ? vel[4] : vel[0];
   const R Ss_K = left ? vel[1] : vel[3];
   /* 0: outside the fast wave, 1: between the fast and the Alfven wave,
    * 2: between the Alfven wave and the contact */
   const int region = left ? ( w < vel[0] ? 0 : ( w < vel[1] ? 1 : 2 ) )
                           : ( w > vel[4] ? 0 : ( w > vel[3] ? 1 : 2 ) );
   R UK[8];
   hlld_flux<R>(P, pK, F, n0, n1, n2);
   hlld_prim_to_cons<R>(P, pK, UK);
   if( region == 0 ){
#pragma unroll
      for( int q=0 ; q<8 ; ++q ) U[q] = UK[q];
   }else{
      R UsK[8];
      hlld_single_star<R>(P, pK, UsK, S_K, vel[2], Pt_star, n0, n1, n2);
      if( region == 1 ){
#pragma unroll
         for( int q=0 ; q<8 ; ++q ){ U[q] = UsK[q]; F[q] += S_K*( U[q] - UK[q] ); }
      }else{
         R UsO[8], UsL[8], UsR[8];
         hlld_single_star<R>(P, pO, UsO, S_O, vel[2], Pt_star, n0, n1, n2);
#pragma unroll
         for( int q=0 ; q<8 ; ++q ){ UsL[q] = left ? UsK[q] : UsO[q]; UsR[q] = left ? UsO[q] : UsK[q]; }
         hlld_double_star<R>(UsL, UsR, U, vel, n0, n1, n2, left ? 0 : 1);
#pragma unroll
         for( int q=0 ; q<8 ; ++q ) F[q] += Ss_K*( U[q] - UsK[q] ) + S_K*( UsK[q] - UK[q] );
      }
   }
#pragma unroll
   for( int q=8 ; q<Q ; ++q ){ U[q] = pK[q]*U[DDD]; F[q] = pK[q]*F[DDD]; }
   const R brfac = R(1.0)/r, bpfac = R(1.0), bzfac = R(1.0);   /* bfield_scale_factor */
   F[SRR] *= hr; F[LLL] *= hp; F[SZZ] *= hz;
   F[BRR] *= brfac/hr; F[BPP] *= bpfac/hp; F[BZZ] *= bzfac/hz;
   U[SRR] *= hr; U[LLL] *= hp; U[SZZ] *= hz;
   U[BRR] *= brfac/hr; U[BPP] *= bpfac/hp; U[BZZ] *= bzfac/hz;
}

/* solve_riemann(), riemann.c:216-318, HLL / HLLC / HLLD (riemann 0 / 1 /
 * 2; HLLD needs MHD).  Returns G_q = (Flux_q - w*Ustr_q)*dAdt, the amount
 * subtracted from cons_L and added to cons_R (riemann.c:312-315), and, when
 * eb is given (MHD), the inputs of flux_to_E (Hydro/mhd.c:293-316):
 * eb = (Flux[BRR], Flux[BPP], Ustr[BRR], Flux[BZZ], Ustr[BZZ]). */
/* Kinematic viscosity of euler.c's visc_flux / visc_source / mindt:
 * Viscosity, or with Use_As_Alpha alpha c h, h = c r^1.5 (euler.c:224-229) */
__device__ __forceinline__ double visc_nu(const DiskParams &P, const double *prim, double r){
   if( !P.visc_alpha ) return P.visc_nu;
   double c = sqrt(P.gam*prim[PPP]/prim[RHO]);
   double h = c*pow(r, 1.5);
   return P.visc_nu*c*h;
}

/* the viscous limit of euler.c's mindt (:357-375): dt <= dx^2 / (2 nu),
 * dx the cell's shortest get_dL (cylindrical: r dphi with r the mid radius,
 * dr, dz) */
__device__ __forceinline__ double visc_dt_limit(const DiskParams &P, const double *prim, double r,
                                                double dt, double rp, double rm, double zp,
                                                double zm, double dph){
   double dL0 = (.5*(rp+rm))*dph, dL1 = rp - rm, dL2 = zp - zm;
   double dx = dL0;
   if( dx > dL1 ) dx = dL1;
   if( dx > dL2 ) dx = dL2;
   double nu = visc_nu(P, prim, r);
   double dt_visc = 0.5*dx*dx/nu;
   if( dt > dt_visc ) dt = dt_visc;
   return dt;
}

/* visc_flux (euler.c:217-259) at a face with centre x, normal n (orthonormal
 * basis), from the averaged state and gradients (riemann.c:295-309); om is
 * the energy frame's Omega at x (get_om) */
template<int Q>
__device__ __forceinline__ void visc_flux(const DiskParams &P, const double *prim,
                                          const double *gradr, const double *gradp,
                                          const double *gradz, double r, double om,
                                          const double *n, double *vF){
   double nu = visc_nu(P, prim, r);
   double rho = prim[RHO];
   double vr = prim[URR];
   double omg = prim[UPP];
   double om_off = omg - om;
   double vz = prim[UZZ];
   double divV_o_d = (gradr[URR] + gradp[UPP] + gradz[UZZ] + vr/r) / 3.0;
   double srr = gradr[URR] - divV_o_d;
   double spp = r*(r*gradp[UPP] + vr - r*divV_o_d);
   double szz = gradz[UZZ] - divV_o_d;
   double srp = 0.5*(r*r*gradr[UPP] + gradp[URR]);
   double srz = 0.5*(gradr[UZZ] + gradz[URR]);
   double spz = 0.5*(gradp[UZZ] + r*r*gradz[UPP]);
   double nc[3] = {n[0], n[1]/r, n[2]};
   double srn = srr*nc[0] + srp*nc[1] + srz*nc[2];
   double spn = srp*nc[0] + spp*nc[1] + spz*nc[2];
   double szn = srz*nc[0] + spz*nc[1] + szz*nc[2];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) vF[q] = 0.0;
   vF[SRR] = -2 * nu * rho * srn;
   vF[LLL] = -2 * nu * rho * spn;
   vF[SZZ] = -2 * nu * rho * szn;
   vF[TAU] = -2 * nu * rho * ( vr*srn + om_off*spn + vz*szn);
}

template<int Q, int NC, int DIM, class R>
__device__ __forceinline__ void solve_riemann(const DiskParams &P, const R *primL,
                                              const R *primR, R r, R om,
                                              R w, R dAdt, R *G, R *eb = nullptr,
                                              const double *vF = nullptr){
   R Flux[Q], Ustr[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){ Flux[q] = R(0.0); Ustr[q] = R(0.0); }
   if constexpr ( NC == 8 ){
      if( P.riemann == 2 ){
         hlld_solve<Q,DIM,R>(P, w, primL, primR, Flux, Ustr, r);
#pragma unroll
         for( int q=0 ; q<Q ; ++q ) G[q] = (Flux[q] - w*Ustr[q])*dAdt;
         if( eb ){ eb[0] = Flux[BRR]; eb[1] = Flux[BPP]; eb[2] = Ustr[BRR];
                   eb[3] = Flux[BZZ]; eb[4] = Ustr[BZZ]; }
         return;
      }
   }
   R Sl, Sr, Ss, Bpack[5];
   vel<NC,DIM,R>(P, primL, primR, r, &Sl, &Sr, &Ss, Bpack);
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
      getUstar<Q,NC,DIM,R>(P, pk, Ustr, r, om, Sk, Ss, Bpack);
      flux<Q,NC,DIM,R>(P, pk, Fk, r, om);
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) Flux[q] = Fk[q] + Sk*( Ustr[q] - Uk[q] );
   }
   if( vF ){                                     /* riemann.c:295-310 */
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) Flux[q] += (R)vF[q];
   }
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) G[q] = (Flux[q] - w*Ustr[q])*dAdt;
   if constexpr ( NC == 8 ){
      if( eb ){ eb[0] = Flux[BRR]; eb[1] = Flux[BPP]; eb[2] = Ustr[BRR];
                eb[3] = Flux[BZZ]; eb[4] = Ustr[BZZ]; }
   }
}

/* ------------------------------------------------------------ planets */
__device__ __forceinline__ double fgrav(double M, double r, double eps, int type){
   if( type == 0 ){                                   /* PLPOINTMASS, planet.c:58-62 */
      /* M*pow(r,n-1.)/pow( pow(r,n) + pow(eps,n) ,1.+1./n) with n = PHI_ORDER
       * = 2 (a global in planet.c, so the reference calls pow at run time):
       * pow(r,1.) is r exactly, pow(x,2.) is written x*x (glibc's pow(x,2.)
       * equals it except for a last-bit difference in about 1e-3 of
       * arguments) and pow(x,1.5) is x*sqrt(x) (within about an ulp of
       * glibc's correctly rounded pow) -- differences of the order of CUDA's
       * pow against glibc's, which the parity tolerance covers. */
      double x = r*r + eps*eps;
      return( M*r/(x*sqrt(x)) );
   }
   return 0.0;
}
/* adjust_gas (planet.c:76-96) with phigrav of a point mass, PHI_ORDER 2
 * (planet.c:36-42): the set-up gas of Include_Atmos */
__device__ __forceinline__ void adjust_gas(const Planet &pl, const double *x, double *prim, double gam){
   double r = x[0], phi = x[1];
   double cosp = cos(phi), sinp = sin(phi);
   double dx = r*cosp - pl.r*cos(pl.phi);
   double dy = r*sinp - pl.r*sin(pl.phi);
   double script_r = sqrt(dx*dx + dy*dy);
   double pot = pl.type == 0 ? pl.M/pow(pow(script_r, 2.0) + pow(pl.eps, 2.0), 1./2.0) : 0.0;
   double c2 = gam*prim[PPP]/prim[RHO];
   double factor = 1. + (gam-1.)*pot/c2;
   prim[RHO] *= factor;
   prim[PPP] *= pow(factor, gam);
}
/* addNoise (noise.c:15-50) with the cell's draws x[0..3] (made on the host
 * from glibc's rand() in the reference's order); cylindrical covariant
 * phi velocity r*Omega for type 3 (geometry_functions.c:19-24) */
__device__ __forceinline__ void add_noise(int type, double absMag, double relMag, double *prim,
                                          const double *x, const double *xr){
   if( type == 1 ){
      prim[URR] = (1.0+xr[0]*relMag)*prim[URR] + xr[1]*absMag;
      prim[UPP] = (1.0+xr[2]*relMag)*prim[UPP] + xr[3]*absMag;
   }else if( type == 2 ){
      prim[PPP] = (1.0+xr[0]*relMag)*prim[PPP] + xr[1]*absMag;
   }else if( type == 3 ){
      double Vc1 = prim[UPP]*x[0];
      prim[URR] = xr[0]*relMag*Vc1 + xr[1]*absMag;
      prim[UZZ] = xr[2]*relMag*Vc1 + xr[3]*absMag;
   }
}
/* planetaryForce(), planet.c:99-150, modes 0 and 1 */
/* the same with sin and cos of the cell's phi given (one sincos per cell
 * for all planets) */
__device__ __forceinline__ void planetary_force_sc(int grav2D, const Planet &pl, double r,
                                                   double sinp, double cosp, double z, double *fr,
                                                   double *fp, double *fz, int mode = 0){
   double rp = pl.r;
   double cpp = pl.cphi, spp = pl.sphi;             /* cos, sin of the planet's phi */
   if( grav2D == 1 ) z = 0.0;
   else if( grav2D == 2 ){ rp = r; cpp = cosp; spp = sinp; z = 1.0; }
   double dx = r*cosp-rp*cpp;
   double dy = r*sinp-rp*spp;
   double script_r = sqrt(dx*dx+dy*dy+z*z);
   double script_r_perp = sqrt(dx*dx+dy*dy);
   double f1 = -fgrav( pl.M , script_r , pl.eps , pl.type );
   double cosa = dx/script_r_perp;
   double sina = dy/script_r_perp;
   double cosap = cosa*cosp+sina*sinp;
   double sinap = sina*cosp-cosa*sinp;
   if( mode == 1 ){                    /* components along the planet's direction */
      cosap = cosa*cpp+sina*spp;
      sinap = sina*cpp-cosa*spp;
   }
   if( script_r_perp <= 0.0 ){ cosap = 0.0; sinap = 0.0; }
   double sint = script_r_perp/script_r;
   double cost = z/script_r;
   *fr = cosap*f1*sint;
   *fp = sinap*f1*sint;
   *fz = f1*cost;
}
__device__ __forceinline__ void planetary_force(int grav2D, const Planet &pl, double r,
                                                double phi, double z, double *fr,
                                                double *fp, double *fz, int mode = 0){
   double sinp, cosp;
   sincos(phi, &sinp, &cosp);
   planetary_force_sc(grav2D, pl, r, sinp, cosp, z, fr, fp, fz, mode);
}

/* ------------------------------------------------------------ initial */
template<int Q, int NC>
__device__ __forceinline__ void initial(const DiskParams &P, double *prim, const double *x){
   if( P.ic_module == 1 ) disco_ic_mhd_shear_eval(&P.ic_mhd, NC, Q, prim, x);
   else if( P.ic_module == 2 ) disco_ic_gr_torus_eval(&P.ic_gr, NC, Q, prim, x);
   else disco_ic_kepler_noise_eval(&P.ic, NC, Q, prim, x);
}

/* positive doubles order like their bit patterns */
__device__ __forceinline__ unsigned long long dbits(double x){
   return (unsigned long long)__double_as_longlong(x);
}

} // namespace disco
