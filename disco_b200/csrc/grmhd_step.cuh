/*
 * The grmhd2 Hydro module's per-state physics for the device timestep (FP64,
 * built with --fmad=false): everything onestep() asks of the module when
 * HYDRO = grmhd2, METRIC = schw_ks_rpz (or the new kerr_ks_rpz), FRAME =
 * normal and Riemann_Solver 0 (HLL):
 *
 *   gr_flux        flux                 Hydro/grmhd2.c:272-335
 *   gr_hll_speeds  vel, outer speeds    Hydro/grmhd2.c:542-612, 655-656
 *   gr_hll         solve_riemann (HLL)  riemann.c:216-258, 300-318
 *   gr_source      source               Hydro/grmhd2.c:383-478
 *   gr_omega       get_omega            Hydro/grmhd2.c:64-86
 *   gr_mindt       mindt                Hydro/grmhd2.c:748-832
 *   gr_cons2prim   cons2prim + noble2d  Hydro/grmhd2.c:253-270, 1096-1313
 *   metric terms   schw_ks_rpz.c:84-189 (derivatives), Frame/normal.c:23-44
 *
 * Each is written in the module's own operation order, so with the same
 * inputs the device rounds every step exactly as the reference's C: only
 * +, -, *, / and sqrt occur.  For the Kerr module (spin a, no reference
 * counterpart) the metric derivatives the source needs come from the
 * closed-form metric evaluated on dual numbers (exact derivatives of the
 * same expressions).
 */
#pragma once
#include "grmhd.cuh"

namespace disco {

/* noble2d's constants (grmhd2.c:1098-1100): tol 1e-12, 10 extra, cap 30 */
__device__ __forceinline__ GRParams gr_params(const DiskParams &P){
   GRParams G;
   G.gam = P.gam; G.rho_floor = P.rho_floor; G.p_floor = P.p_floor;
   G.M = P.gr_M; G.a = P.gr_a; G.tol = 1.0e-12;
   G.metric = P.gr_metric; G.nextra = 10; G.max_iter = 30; G.pad = 0;
   return G;
}

/* metric_jacobian (alpha sqrt(gamma)): r for both Kerr-Schild modules */
__device__ __forceinline__ double gr_jacobian(const double *x){ return x[0]; }

/* ------------------------------------------------------------- flux */
__device__ __forceinline__ void gr_flux(const GRParams &G, const Metric3 &g, const double *prim,
                                        const double *x, const double *n, double *F){
   const double r = x[0];
   const double al = g.al, jac = g.jac, sqrtgam = g.sqrtgam;
   const double *be = g.be, *gam = g.gam, *igam = g.igam, *U = g.U;
   const double rho = prim[RHO], Pp = prim[PPP];
   const double l[3] = {prim[URR], prim[UPP], prim[UZZ]};
   const double B[3] = {prim[BRR]/sqrtgam, prim[BPP]/(r*sqrtgam), prim[BZZ]/sqrtgam};
   double igaml[3], u[3], v[3];
   for( int i=0 ; i<3 ; ++i ){
      igaml[i] = 0.0;
      for( int j=0 ; j<3 ; ++j ) igaml[i] += igam[3*i+j]*l[j];
   }
   const double u2 = l[0]*igaml[0] + l[1]*igaml[1] + l[2]*igaml[2];
   const double w = sqrt(1.0 + u2);
   const double u0 = w/al;
   for( int i=0 ; i<3 ; ++i ) u[i] = igaml[i] - be[i]*u0;
   for( int i=0 ; i<3 ; ++i ) v[i] = u[i]/u0;
   const double lt = -al*w + be[0]*l[0] + be[1]*l[1] + be[2]*l[2];
   const double uU = U[0]*lt + U[1]*l[0] + U[2]*l[1] + U[3]*l[2];
   const double uB = l[0]*B[0] + l[1]*B[1] + l[2]*B[2];
   double bd[3];
   for( int k=0 ; k<3 ; ++k ) bd[k] = (gam[3*k]*B[0] + gam[3*k+1]*B[1] + gam[3*k+2]*B[2] + l[k]*uB) / w;
   double B2 = 0.0, UB = 0.0;
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ){
      B2 += gam[3*i+j]*B[i]*B[j];
      UB += gam[3*i+j] * B[i] * (U[0]*be[j] + U[j+1]);
   }
   const double b2 = (B2 + uB*uB) / (w*w);
   const double Ub = (UB + uU*uB) / w;
   const double un = u[0]*n[0] + u[1]*n[1] + u[2]*n[2];
   const double Bn = B[0]*n[0] + B[1]*n[1] + B[2]*n[2];
   const double Un = U[1]*n[0] + U[2]*n[1] + U[3]*n[2];
   const double vn = v[0]*n[0] + v[1]*n[1] + v[2]*n[2];
   const double hn = n[0] + r*n[1] + n[2];
   const double bn = (Bn + uB*un)/w;
   const double gl = G.gam;
   const double rhoh = rho + gl/(gl-1.0)*Pp + b2;
   const double rhoe = Pp / (gl-1.0);
   const double Pt = Pp + 0.5*b2;
   F[DDD] = jac * hn * rho*un;
   F[SRR] = jac * hn * (rhoh*un*l[0] + Pt*n[0] - bd[0]*bn);
   F[LLL] = jac * hn * (rhoh*un*l[1] + Pt*n[1] - bd[1]*bn);
   F[SZZ] = jac * hn * (rhoh*un*l[2] + Pt*n[2] - bd[2]*bn);
   F[TAU] = jac * hn * (-(rhoe+0.5*b2)*uU*un - Pt*(uU*un+Un) - rho*(uU+1.0)*un + Ub*bn);
   F[BRR] = sqrtgam * hn * (B[0]*vn - Bn*v[0])/r;
   F[BPP] = sqrtgam * hn * (B[1]*vn - Bn*v[1]);
   F[BZZ] = sqrtgam * hn * (B[2]*vn - Bn*v[2]);
   F[8] = prim[8]*F[DDD];
}

/* flux() and prim2cons(dV = 1) of the same state at the same point: the two
 * reference functions compute the same intermediates (u^i, w, b^mu, b^2,
 * ...) with the same expressions, so evaluating them once gives both results
 * bit for bit */
__device__ __forceinline__ void gr_flux_cons(const GRParams &G, const Metric3 &g, const double *prim,
                                             const double *x, const double *n, double *F, double *Uc){
   const double r = x[0];
   const double al = g.al, jac = g.jac, sqrtgam = g.sqrtgam;
   const double *be = g.be, *gam = g.gam, *igam = g.igam, *U = g.U;
   const double rho = prim[RHO], Pp = prim[PPP];
   const double l[3] = {prim[URR], prim[UPP], prim[UZZ]};
   const double B[3] = {prim[BRR]/sqrtgam, prim[BPP]/(r*sqrtgam), prim[BZZ]/sqrtgam};
   double igaml[3], u[3], v[3];
#pragma unroll
   for( int i=0 ; i<3 ; ++i ){
      igaml[i] = 0.0;
#pragma unroll
      for( int j=0 ; j<3 ; ++j ) igaml[i] += igam[3*i+j]*l[j];
   }
   const double u2 = l[0]*igaml[0] + l[1]*igaml[1] + l[2]*igaml[2];
   const double w = sqrt(1.0 + u2);
   const double u0 = w/al;
#pragma unroll
   for( int i=0 ; i<3 ; ++i ) u[i] = igaml[i] - be[i]*u0;
#pragma unroll
   for( int i=0 ; i<3 ; ++i ) v[i] = u[i]/u0;
   const double lt = -al*w + be[0]*l[0] + be[1]*l[1] + be[2]*l[2];
   const double uU = U[0]*lt + U[1]*l[0] + U[2]*l[1] + U[3]*l[2];
   const double uB = l[0]*B[0] + l[1]*B[1] + l[2]*B[2];
   const double b0 = uB / al;
   double bd[3];
#pragma unroll
   for( int k=0 ; k<3 ; ++k ) bd[k] = (gam[3*k]*B[0] + gam[3*k+1]*B[1] + gam[3*k+2]*B[2] + l[k]*uB) / w;
   double B2 = 0.0, UB = 0.0;
#pragma unroll
   for( int i=0 ; i<3 ; ++i )
#pragma unroll
      for( int j=0 ; j<3 ; ++j ){
         B2 += gam[3*i+j]*B[i]*B[j];
         UB += gam[3*i+j] * B[i] * (U[0]*be[j] + U[j+1]);
      }
   const double b2 = (B2 + uB*uB) / (w*w);
   const double Ub = (UB + uU*uB) / w;
   const double gl = G.gam;
   const double rhoh = rho + gl/(gl-1.0)*Pp + b2;
   const double rhoe = Pp / (gl-1.0);
   /* prim2cons, grmhd2.c:88-180 */
   Uc[DDD] = jac * rho*u0 * 1.0;
   Uc[SRR] = jac * (rhoh*u0*l[0] - b0*bd[0]) * 1.0;
   Uc[LLL] = jac * (rhoh*u0*l[1] - b0*bd[1]) * 1.0;
   Uc[SZZ] = jac * (rhoh*u0*l[2] - b0*bd[2]) * 1.0;
   Uc[TAU] = jac * (-(rhoe+0.5*b2)*uU*u0 - (Pp+0.5*b2)*(uU*u0+U[0])
                         - rho*(uU+1.0)*u0 + Ub*b0) * 1.0;
   Uc[BRR] = sqrtgam * B[0]/r * 1.0;
   Uc[BPP] = sqrtgam * B[1] * 1.0;
   Uc[BZZ] = sqrtgam * B[2] * 1.0;
   Uc[8] = prim[8]*Uc[DDD];
   /* flux, grmhd2.c:272-335 */
   const double un = u[0]*n[0] + u[1]*n[1] + u[2]*n[2];
   const double Bn = B[0]*n[0] + B[1]*n[1] + B[2]*n[2];
   const double Un = U[1]*n[0] + U[2]*n[1] + U[3]*n[2];
   const double vn = v[0]*n[0] + v[1]*n[1] + v[2]*n[2];
   const double hn = n[0] + r*n[1] + n[2];
   const double bn = (Bn + uB*un)/w;
   const double Pt = Pp + 0.5*b2;
   F[DDD] = jac * hn * rho*un;
   F[SRR] = jac * hn * (rhoh*un*l[0] + Pt*n[0] - bd[0]*bn);
   F[LLL] = jac * hn * (rhoh*un*l[1] + Pt*n[1] - bd[1]*bn);
   F[SZZ] = jac * hn * (rhoh*un*l[2] + Pt*n[2] - bd[2]*bn);
   F[TAU] = jac * hn * (-(rhoe+0.5*b2)*uU*un - Pt*(uU*un+Un) - rho*(uU+1.0)*un + Ub*bn);
   F[BRR] = sqrtgam * hn * (B[0]*vn - Bn*v[0])/r;
   F[BPP] = sqrtgam * hn * (B[1]*vn - Bn*v[1]);
   F[BZZ] = sqrtgam * hn * (B[2]*vn - Bn*v[2]);
   F[8] = prim[8]*F[DDD];
}

/* ------------------------------------------------------------- HLL speeds */
/* one side's fast speeds along n (grmhd2.c:551-612 for one of the two states) */
__device__ __forceinline__ void gr_side_speeds(const GRParams &G, const Metric3 &g, double sqrtgam_v,
                                               const double *prim, const double *n, double r,
                                               double bn, double ign, double hn,
                                               double *sl, double *sr){
   const double gl = G.gam;
   const double *gam = g.gam, *igam = g.igam;
   const double rho = prim[RHO], P = prim[PPP];
   const double l[3] = {prim[URR], prim[UPP], prim[UZZ]};
   const double B[3] = {prim[BRR]/sqrtgam_v, prim[BPP]/(r*sqrtgam_v), prim[BZZ]/sqrtgam_v};
   const double cs2 = gl*P/(rho+gl/(gl-1.0)*P);
   double uS[3], u2 = 0.0;
   for( int i=0 ; i<3 ; ++i ){
      uS[i] = 0.0;
      for( int j=0 ; j<3 ; ++j ) uS[i] += igam[3*i+j]*l[j];
      u2 += uS[i]*l[i];
   }
   const double w = sqrt(1.0+u2);
   const double v2 = u2/(w*w);
   const double uB = l[0]*B[0] + l[1]*B[1] + l[2]*B[2];
   double B2 = 0.0;
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ) B2 += gam[3*i+j]*B[i]*B[j];
   const double b2 = (B2 + uB*uB) / (w*w);
   const double va2 = b2 / (rho + gl/(gl-1.0)*P + b2);
   const double cf2 = cs2 + va2 - cs2*va2;
   const double vSn = (uS[0]*n[0]+uS[1]*n[1]+uS[2]*n[2]) / w;
   const double dv = sqrt(cf2*(ign - vSn*vSn - cf2*(ign*v2-vSn*vSn))) / w;
   const double al = g.al;
   *sl = hn * (al * (vSn*(1.0-cf2) - dv) / (1.0-v2*cf2) - bn);
   *sr = hn * (al * (vSn*(1.0-cf2) + dv) / (1.0-v2*cf2) - bn);
}

/* vel()'s Sl, Sr (the contact speed it also returns only serves HLLC) */
__device__ __forceinline__ void gr_hll_speeds(const GRParams &G, const Metric3 &g, const double *primL,
                                              const double *primR, const double *n, const double *x,
                                              double *Sl, double *Sr){
   const double r = x[0];
   const double sqrtgam_v = gr_jacobian(x) / (g.al * r);
   const double bn = (g.be[0]*n[0]+g.be[1]*n[1]+g.be[2]*n[2]);
   const double ign = g.igam[3*0+0]*n[0] + g.igam[3*1+1]*n[1] + g.igam[3*2+2]*n[2];
   const double hn = n[0] + r*n[1] + n[2];
   double sl1, sr1, sl2, sr2;
   gr_side_speeds(G, g, sqrtgam_v, primL, n, r, bn, ign, hn, &sl1, &sr1);
   gr_side_speeds(G, g, sqrtgam_v, primR, n, r, bn, ign, hn, &sl2, &sr2);
   *Sr = sr1 > sr2 ? sr1 : sr2;
   *Sl = sl1 < sl2 ? sl1 : sl2;
}

/* ------------------------------------------------------------- HLL flux */
/* G[q] = (F - w U*) dA dt of one face, solve_riemann with Riemann_Solver 0:
 * the upwind state's flux outside the fan, the HLL average inside.  g is
 * the metric at x (a per-annulus or per-track table: it depends on r, z). */
__device__ __forceinline__ void gr_hll(const DiskParams &P, const Metric3 &g, const double *primL,
                                       const double *primR, const double *x, const double *n,
                                       double w, double dAdt, double *Gq){
   const GRParams G = gr_params(P);
   double Sl, Sr;
   gr_hll_speeds(G, g, primL, primR, n, x, &Sl, &Sr);
   double Flux[GR_Q], Ustr[GR_Q];
   if( w < Sl ){
      gr_flux_cons(G, g, primL, x, n, Flux, Ustr);
   }else if( w > Sr ){
      gr_flux_cons(G, g, primR, x, n, Flux, Ustr);
   }else{
      double Fl[GR_Q], Fr[GR_Q], Ul[GR_Q], Ur[GR_Q];
      const double aL = Sr, aR = -Sl;
      gr_flux_cons(G, g, primL, x, n, Fl, Ul);
      gr_flux_cons(G, g, primR, x, n, Fr, Ur);
#pragma unroll
      for( int q=0 ; q<GR_Q ; ++q ){
         Flux[q] = ( aL*Fl[q] + aR*Fr[q] + aL*aR*( Ul[q] - Ur[q] ) )/( aL + aR );
         Ustr[q] = ( aR*Ul[q] + aL*Ur[q] + Fl[q] - Fr[q] )/( aL + aR );
      }
   }
#pragma unroll
   for( int q=0 ; q<GR_Q ; ++q ) Gq[q] = (Flux[q] - w*Ustr[q])*dAdt;
}

/* ------------------------------------------------------------- metric derivatives */
/* schw_ks_rpz.c:84-167: d g_{mu nu} / d x^i for i = 1 (r) and 3 (z), the
 * lapse's and the shift's gradients, M the mass. */
__device__ __forceinline__ void schw_der_g(const double *x, double M, int i, double *dg){
   for( int mu=0 ; mu<16 ; ++mu ) dg[mu] = 0.0;
   const double r = x[0], z = x[2];
   const double R = sqrt(r*r+z*z);
   const double st = r/R, ct = z/R;
   const double MoR2 = M/(R*R), MoR3 = M/(R*R*R), MoR4 = M/(R*R*R*R);
   if( i == 1 ){
      dg[0]  = -2*MoR2 * st;
      dg[1]  =  2*MoR2 * (1.0-2*st*st);
      dg[3]  = -4*MoR3*z * st;
      dg[5]  =  2*MoR3*r * (2.0-3.0*st*st);
      dg[7]  =  2*MoR3*z * (1.0-3.0*st*st);
      dg[10] =  2*r;
      dg[15] = -6*MoR4*z*z * st;
   }else{
      dg[0]  = -2*MoR2 * ct;
      dg[1]  = -4*MoR3*r * ct;
      dg[3]  =  2*MoR2 * (1.0-2*ct*ct);
      dg[5]  = -6*MoR4*r*r * ct;
      dg[7]  =  2*MoR3*r * (1.0-3.0*ct*ct);
      dg[15] =  2*MoR3*z * (2.0-3.0*ct*ct);
   }
   dg[4] = dg[1]; dg[12] = dg[3]; dg[13] = dg[7];
}
__device__ __forceinline__ void schw_der_lapse(const double *x, double M, double *da){
   const double r = x[0], z = x[2];
   const double R = sqrt(r*r+z*z);
   const double st = r/R, ct = z/R;
   const double MoR2 = M/(R*R);
   const double a = 1.0/sqrt(1.0+2*M/R);
   da[0] = 0.0;
   da[1] = a*a*a * MoR2 * st;
   da[2] = 0.0;
   da[3] = a*a*a * MoR2 * ct;
}
__device__ __forceinline__ void schw_der_shift(const double *x, double M, double *db){
   const double r = x[0], z = x[2];
   const double R = sqrt(r*r+z*z);
   const double st = r/R, ct = z/R;
   const double denom = 1.0/(R*R + 2*M*R);
   const double d_denom = -denom*denom * 2*(R+M);
   for( int i=0 ; i<12 ; ++i ) db[i] = 0.0;
   db[3] = 2*M * denom + 2*M*r * d_denom*st;
   db[5] = 2*M*z * d_denom*st;
   db[9] = 2*M*r * d_denom*ct;
   db[11] = 2*M * denom + 2*M*z * d_denom*ct;
}

/* first-order dual numbers: value and derivative along one direction */
struct Dual { double v, d; };
__device__ __forceinline__ Dual operator+(Dual a, Dual b){ return {a.v + b.v, a.d + b.d}; }
__device__ __forceinline__ Dual operator-(Dual a, Dual b){ return {a.v - b.v, a.d - b.d}; }
__device__ __forceinline__ Dual operator*(Dual a, Dual b){ return {a.v*b.v, a.d*b.v + a.v*b.d}; }
__device__ __forceinline__ Dual operator/(Dual a, Dual b){ return {a.v/b.v, (a.d*b.v - a.v*b.d)/(b.v*b.v)}; }
__device__ __forceinline__ Dual operator*(double s, Dual a){ return {s*a.v, s*a.d}; }
__device__ __forceinline__ Dual operator+(double s, Dual a){ return {s + a.v, a.d}; }
__device__ __forceinline__ Dual dsqrt(Dual a){ double q = sqrt(a.v); return {q, a.d/(2.0*q)}; }
__device__ __forceinline__ Dual dconst(double v){ return {v, 0.0}; }

/* The Kerr-Schild fields of metric_kerr (grmhd.cuh) on duals: lapse,
 * shift^i, gamma_ij at (r, z). */
__device__ __forceinline__ void kerr_fields_dual(Dual r, Dual z, double M, double a,
                                                 Dual &al, Dual *be, Dual *gam){
   const Dual rho2 = r*r + z*z;
   const Dual b = rho2 - dconst(a*a);
   const Dual R2 = 0.5*(b + dsqrt(b*b + (4.0*a*a)*(z*z)));
   const Dual R = dsqrt(R2);
   const Dual f = (2.0*M)*R*R2/(R2*R2 + (a*a)*(z*z));
   const Dual den = R2 + dconst(a*a);
   const Dual l[3] = { R*r/den, dconst(0.0) - (a*r*r)/den, z/R };
   const Dual lu[3] = { l[0], l[1]/(r*r), l[2] };
   const Dual flat[3] = { dconst(1.0), r*r, dconst(1.0) };
   const Dual c = f/(1.0 + f);
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j )
      gam[3*i+j] = (i == j ? flat[i] : dconst(0.0)) + f*l[i]*l[j];
   for( int i=0 ; i<3 ; ++i ) be[i] = c*lu[i];
   al = dconst(1.0)/dsqrt(1.0 + f);
}

/* the 4-metric g_{mu nu} from lapse, shift and 3-metric, differentiated */
__device__ __forceinline__ void kerr_der(const double *x, double M, double a, int dir, double *dg,
                                         double *dal, double *dbe){
   Dual r = {x[0], dir == 1 ? 1.0 : 0.0}, z = {x[2], dir == 3 ? 1.0 : 0.0};
   Dual al, be[3], gam[9];
   kerr_fields_dual(r, z, M, a, al, be, gam);
   Dual bl[3];
   for( int i=0 ; i<3 ; ++i ) bl[i] = gam[3*i]*be[0] + gam[3*i+1]*be[1] + gam[3*i+2]*be[2];
   Dual g00 = dconst(0.0) - al*al + (bl[0]*be[0] + bl[1]*be[1] + bl[2]*be[2]);
   dg[0] = g00.d;
   for( int i=0 ; i<3 ; ++i ){ dg[i+1] = bl[i].d; dg[4*(i+1)] = bl[i].d; }
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ) dg[4*(i+1)+j+1] = gam[3*i+j].d;
   *dal = al.d;
   for( int i=0 ; i<3 ; ++i ) dbe[i] = be[i].d;
}

/* ------------------------------------------------------------- tables */
/* The metric depends on (r, z) only, so every place the step evaluates it
 * is a fixed point of the grid: per annulus its centroid (phi faces,
 * cons->prim, mesh Omega) and the midpoint of its corners (source, mindt,
 * with the frame's and the 4-metric's derivatives there), per r- or z-track
 * the face centre.  They are computed once per batch into these tables with
 * the same functions, so the step reads bit-identical values. */
struct GRAnn {
   Metric3 c;            /* at (centroid r, centroid z) */
   Metric3 m;            /* at (midpoint r, midpoint z) */
   double dU[16];        /* frame_der_U at the midpoint */
   double dgr[16], dgz[16];   /* d g_{mu nu}/dr, /dz at the midpoint */
};

__device__ __forceinline__ void gr_ann_table(const DiskParams &P, double rp, double rm, double zp,
                                             double zm, GRAnn &T){
   const GRParams G = gr_params(P);
   const double xc[3] = {centroid_r(rp, rm), 0.0, centroid_z(zp, zm)};
   metric_at(G, xc, T.c);
   const double x[3] = {0.5*(rm+rp), 0.0, 0.5*(zm+zp)};
   metric_at(G, x, T.m);
   double da[4], db[12];
   if( G.metric == GR_METRIC_KERR ){
      double b1[3], b3[3];
      kerr_der(x, G.M, G.a, 1, T.dgr, &da[1], b1);
      kerr_der(x, G.M, G.a, 3, T.dgz, &da[3], b3);
      da[0] = 0.0; da[2] = 0.0;
      for( int j=0 ; j<3 ; ++j ){ db[j] = 0.0; db[3+j] = b1[j]; db[6+j] = 0.0; db[9+j] = b3[j]; }
   }else{
      schw_der_g(x, G.M, 1, T.dgr);
      schw_der_g(x, G.M, 3, T.dgz);
      schw_der_lapse(x, G.M, da);
      schw_der_shift(x, G.M, db);
   }
   /* frame_der_U (Frame/normal.c:23-44): killing directions t and phi */
   const double ia = 1.0/T.m.al;
   for( int i=0 ; i<16 ; ++i ) T.dU[i] = 0.0;
   for( int i=1 ; i<4 ; i+=2 ){
      T.dU[4*i] = -ia*ia*da[i];
      for( int j=0 ; j<3 ; ++j ) T.dU[4*i+j+1] = T.m.be[j]*ia*ia*da[i] - db[3*i+j]*ia;
   }
}

/* ------------------------------------------------------------- source */
/* source() of grmhd2.c:383-478 into cons (SRR, LLL, SZZ, TAU), at the
 * midpoint of the cell's corners, from the annulus table. */
__device__ __forceinline__ void gr_source(const DiskParams &P, const GRAnn &T, const double *prim,
                                          double *cons, double r, double dVdt){
   const Metric3 &g = T.m;
   const double al = g.al, jac = g.jac, sqrtgam = g.sqrtgam;
   const double *be = g.be, *gam = g.gam, *igam = g.igam, *U = g.U;
   const double rho = prim[RHO], Pp = prim[PPP];
   double l[4] = {0.0, prim[URR], prim[UPP], prim[UZZ]};
   const double B[3] = {prim[BRR]/sqrtgam, prim[BPP]/(r*sqrtgam), prim[BZZ]/sqrtgam};
   double ig[16];
   const double ia2 = 1.0/(al*al);
   ig[0] = -ia2;
#pragma unroll
   for( int mu=0 ; mu<3 ; ++mu ){
      ig[mu+1] = be[mu]*ia2;
      ig[4*(mu+1)] = ig[mu+1];
#pragma unroll
      for( int nu=0 ; nu<3 ; ++nu ) ig[4*(mu+1)+nu+1] = igam[3*mu+nu]-be[mu]*be[nu]*ia2;
   }
   double igaml[3];
   igaml[0] = igam[0]*l[1] + igam[1]*l[2] + igam[2]*l[3];
   igaml[1] = igam[3]*l[1] + igam[4]*l[2] + igam[5]*l[3];
   igaml[2] = igam[6]*l[1] + igam[7]*l[2] + igam[8]*l[3];
   const double u2 = l[1]*igaml[0] + l[2]*igaml[1] + l[3]*igaml[2];
   const double w = sqrt(1.0 + u2);
   double u[4];
   u[0] = w/al;
#pragma unroll
   for( int i=0 ; i<3 ; ++i ) u[i+1] = igaml[i] - be[i]*u[0];
   l[0] = -al*w + be[0]*l[1] + be[1]*l[2] + be[2]*l[3];
   const double uB = l[1]*B[0] + l[2]*B[1] + l[3]*B[2];
   double b[4], bd[4];
   b[0] = uB / al;
   b[1] = (B[0]+u[1]*uB)/w;
   b[2] = (B[1]+u[2]*uB)/w;
   b[3] = (B[2]+u[3]*uB)/w;
   bd[1] = (gam[0]*B[0] + gam[1]*B[1] + gam[2]*B[2] + l[1]*uB) / w;
   bd[2] = (gam[3]*B[0] + gam[4]*B[1] + gam[5]*B[2] + l[2]*uB) / w;
   bd[3] = (gam[6]*B[0] + gam[7]*B[1] + gam[8]*B[2] + l[3]*uB) / w;
   double B2 = 0.0, beB = 0.0;
#pragma unroll
   for( int i=0 ; i<3 ; ++i )
#pragma unroll
      for( int j=0 ; j<3 ; ++j ){
         beB += gam[3*i+j]*be[i]*B[j];
         B2 += gam[3*i+j]*B[i]*B[j];
      }
   bd[0] = (beB + l[0]*uB) / w;
   const double b2 = (B2 + uB*uB) / (w*w);
   const double gl = P.gam;
   const double rhoh = rho + gl/(gl-1.0)*Pp + b2;
   const double Pt = Pp + 0.5*b2;
   double Sk[3] = {0.0, 0.0, 0.0};
#pragma unroll
   for( int mu=0 ; mu<4 ; ++mu )
#pragma unroll
      for( int nu=0 ; nu<4 ; ++nu )
         Sk[0] += (rhoh*u[mu]*u[nu] + ig[4*mu+nu]*Pt - b[mu]*b[nu]) * T.dgr[4*mu+nu];
   Sk[0] *= 0.5;                                   /* Sk[1]: phi is a killing direction */
#pragma unroll
   for( int mu=0 ; mu<4 ; ++mu )
#pragma unroll
      for( int nu=0 ; nu<4 ; ++nu )
         Sk[2] += (rhoh*u[mu]*u[nu] + ig[4*mu+nu]*Pt - b[mu]*b[nu]) * T.dgz[4*mu+nu];
   Sk[2] *= 0.5;
   double S0 = -U[1]*Sk[0] - U[2]*Sk[1] - U[3]*Sk[2];
#pragma unroll
   for( int mu=0 ; mu<4 ; ++mu )
#pragma unroll
      for( int nu=0 ; nu<4 ; ++nu ){
         if( mu == nu ) S0 += -(rhoh*u[mu]*l[nu] + Pt - b[mu]*bd[nu]) * T.dU[4*mu+nu];
         else           S0 += -(rhoh*u[mu]*l[nu] - b[mu]*bd[nu]) * T.dU[4*mu+nu];
      }
   cons[SRR] += jac * Sk[0] * dVdt;
   cons[LLL] += jac * Sk[1] * dVdt;
   cons[SZZ] += jac * Sk[2] * dVdt;
   cons[TAU] += jac * S0 * dVdt;
}

/* ------------------------------------------------------------- mesh Omega */
__device__ __forceinline__ double gr_omega(const Metric3 &g, const double *prim){
   const double l[3] = {prim[URR], prim[UPP], prim[UZZ]};
   double u2 = 0.0;
#pragma unroll
   for( int i=0 ; i<3 ; ++i )
#pragma unroll
      for( int j=0 ; j<3 ; ++j ) u2 += g.igam[3*i+j]*l[i]*l[j];
   const double w = sqrt(1.0 + u2);
   return g.al*(g.igam[3]*l[0]+g.igam[4]*l[1]+g.igam[5]*l[2])/w - g.be[1];
}
/* the same with the metric evaluated at x (set-up kernels) */
__device__ __forceinline__ double gr_omega_at(const DiskParams &P, const double *prim, const double *x){
   const GRParams G = gr_params(P);
   Metric3 g;
   metric_at(G, x, g);
   return gr_omega(g, prim);
}

/* ------------------------------------------------------------- mindt */
/* g: the metric at the midpoint of the corners (GRAnn::m) */
__device__ __forceinline__ double gr_mindt(const DiskParams &P, const Metric3 &g, const double *prim,
                                           double wc, const double *xp, const double *xm, int *err){
   const GRParams G = gr_params(P);
   const double x[3] = {0.5*(xm[0]+xp[0]), 0.5*(xm[1]+xp[1]), 0.5*(xm[2]+xp[2])};
   const double r = x[0];
   const double al = g.al, *be = g.be, *gam = g.gam, *igam = g.igam;
   const double sqrtgam = gr_jacobian(x) / (r*al);
   const double gl = G.gam;
   const double rho = prim[RHO], Pp = prim[PPP];
   const double l[3] = {prim[URR], prim[UPP], prim[UZZ]};
   const double B[3] = {prim[BRR]/sqrtgam, prim[BPP]/(r*sqrtgam), prim[BZZ]/sqrtgam};
   const double cs = sqrt(gl*Pp/(rho+gl/(gl-1)*Pp));
   double uS[3], u2 = 0.0;
   for( int i=0 ; i<3 ; ++i ){
      uS[i] = 0.0;
      for( int j=0 ; j<3 ; ++j ) uS[i] += igam[3*i+j]*l[j];
      u2 += uS[i]*l[i];
   }
   const double w = sqrt(1.0+u2);
   double vS[3];
   for( int i=0 ; i<3 ; ++i ) vS[i] = uS[i]/w;
   const double v2 = u2/(w*w);
   const double uB = l[0]*B[0] + l[1]*B[1] + l[2]*B[2];
   double B2 = 0.0;
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ) B2 += gam[3*i+j]*B[i]*B[j];
   const double b2 = (B2 + uB*uB) / (w*w);
   const double va2 = b2 / (rho + gl/(gl-1.0)*Pp + b2);
   const double cf = sqrt(cs*cs + va2 - cs*cs*va2);
   const double sig = 1-cf*cf;
   const double dvr = cf * sqrt(igam[0]*(1-cf*cf*v2) - sig*vS[0]*vS[0]) / w;
   const double vrl = fabs(al * (vS[0]*sig - dvr) / (1-v2*cf*cf) - be[0]);
   const double vrr = fabs(al * (vS[0]*sig + dvr) / (1-v2*cf*cf) - be[0]);
   const double dvp = cf * sqrt(igam[4]*(1-cf*cf*v2) - sig*vS[1]*vS[1]) / w;
   const double vpl = fabs(r * (al * (vS[1]*sig - dvp) / (1-v2*cf*cf) - be[1] -wc));
   const double vpr = fabs(r * (al * (vS[1]*sig + dvp) / (1-v2*cf*cf) - be[1] -wc));
   const double dvz = cf * sqrt(igam[8]*(1-cf*cf*v2) - sig*vS[2]*vS[2]) / w;
   const double vzl = fabs(al * (vS[2]*sig - dvz) / (1-v2*cf*cf) - be[2]);
   const double vzr = fabs(al * (vS[2]*sig + dvz) / (1-v2*cf*cf) - be[2]);
   const double maxvr = vrr > vrl ? vrr : vrl;
   const double maxvp = vpr > vpl ? vpr : vpl;
   const double maxvz = vzr > vzl ? vzr : vzl;
   const double dtr = (xp[0]-xm[0])/maxvr;                                  /* get_dL(.,.,1) */
   const double dtp = (.5*(xp[0]+xm[0]))*get_dp(xp[1], xm[1], P.Pmax, err)/maxvp;   /* get_dL 0 */
   const double dtz = (xp[2]-xm[2])/maxvz;                                  /* get_dL(.,.,2) */
   double dt = dtr;
   dt = dt < dtp ? dt : dtp;
   dt = dt < dtz ? dt : dtz;
   return dt;
}

/* ------------------------------------------------------------- cons -> prim */
/* cons2prim (grmhd2.c:253-270): the conserved densities cons/dV, noble2d
 * warm-started from the cell's current prim (grmhd2.c:1167-1175), then the
 * recovery.  prim is read as the guess and overwritten; returns the
 * Newton iterations. */
__device__ __forceinline__ int gr_cons2prim(const DiskParams &P, const Metric3 &g, const double *cons,
                                            double *prim, const double *x, double dV){
   const GRParams G = gr_params(P);
   double c1[GR_Q];
#pragma unroll
   for( int q=0 ; q<GR_Q ; ++q ) c1[q] = cons[q]/dV;
   C2PInv I;
   c2p_invariants(G, g, c1, prim, x, I);
   double v2 = I.v20, eta = I.eta0;
   int ok;
   const int it = c2p_newton(G, I, &v2, &eta, &ok);
   c2p_recover(G, g, I, v2, eta, c1, prim, x);
   return it;
}

} /* namespace disco */
