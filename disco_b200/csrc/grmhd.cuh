/*
 * GRMHD state conversions on the device (FP64), for the cons -> prim solve
 * of Hydro/grmhd2.c, plus the learned initial guess.
 *
 *   metric  schw_ks_rpz: Schwarzschild in Kerr-Schild cylindrical
 *           coordinates, Hydro/Metric/schw_ks_rpz.c:20-81, same expressions;
 *           kerr_ks_rpz: the Kerr (spin a) generalisation, a new module (the
 *           reference reads Metric_Par3 "a" but no metric uses it): with
 *           g = eta + f l l, f = 2 M R^3/(R^4 + a^2 z^2), R the oblate
 *           spheroidal radius, the cylindrical covector is
 *           l_i = (R r/(R^2+a^2), -a r^2/(R^2+a^2), z/R), so
 *           gamma_ij = diag(1, r^2, 1) + f l_i l_j, beta^i = f l^i/(1+f),
 *           alpha = (1+f)^-1/2, sqrt(gamma) = r (1+f)^1/2; at a = 0 every
 *           term reduces to schw_ks_rpz.
 *   frame   normal observer U = (1/alpha, -beta/alpha), Frame/normal.c:9-21
 *   p2c     prim2cons, grmhd2.c:88-180
 *   c2p     cons2prim_solve_adiabatic_noble2d, grmhd2.c:1096-1313: 2x2
 *           Newton in (v^2, eta) from a guess, stop when |d eta/eta| < tol,
 *           then Nextra more iterations, at most max_iter.
 * Only +, -, *, / and sqrt appear, so with --fmad=false the Schwarzschild
 * path rounds exactly as the reference.
 *
 * The learned guess replaces the plain guess (the cell's previous prims,
 * grmhd2.c:1167-1175) by the plain guess plus a small MLP's correction in
 * (log eta, v^2), predicted from the solve's invariants and the plain
 * guess's residual; Newton then runs to the same tol with the same tail,
 * and falls back to the plain guess if it fails.
 */
#pragma once
#include "disco_device.cuh"

namespace disco {

#define GR_Q 9
enum { GR_METRIC_SCHW = 0, GR_METRIC_KERR = 1 };

/* MLP 8 -> 64 -> 64 -> 2, tanh hidden units */
#define MLP_IN 8
#define MLP_H 64
#define MLP_OUT 2
/* parameter block: W1[H][IN] b1[H] W2[H][H] b2[H] W3[OUT][H] b3[OUT];
 * normalisation: in_shift[IN] in_scale[IN] out_shift[OUT] out_scale[OUT] */
#define MLP_NW1 (MLP_H*MLP_IN)
#define MLP_NW2 (MLP_H*MLP_H)
#define MLP_NW3 (MLP_OUT*MLP_H)
#define MLP_NPARAM (MLP_NW1 + MLP_H + MLP_NW2 + MLP_H + MLP_NW3 + MLP_OUT)
#define MLP_NNORM (2*MLP_IN + 2*MLP_OUT)

struct GRParams {
   double gam, rho_floor, p_floor, M, a, tol;
   int metric, nextra, max_iter, pad;
};

struct Metric3 {
   double al, be[3], gam[9], igam[9], jac, sqrtgam, U[4];
};

/* schw_ks_rpz.c:20-81, expression for expression */
__host__ __device__ __forceinline__ void metric_schw(const double *x, double M, Metric3 &g){
   double r = x[0], z = x[2];
   {  double R = sqrt(x[0]*x[0] + x[2]*x[2]);
      g.al = 1.0/sqrt(1.0 + 2*M/R); }
   {  double R = sqrt(r*r+z*z);
      double a2 = 1.0 / (1.0 + 2*M/R);
      g.be[0] = 2*M*r/(R*R) * a2; g.be[1] = 0.0; g.be[2] = 2*M*z/(R*R) * a2; }
   {  double R = sqrt(r*r+z*z);
      double H = 2*M/R, st = r/R, ct = z/R;
      g.gam[0] = 1.0 + H*st*st; g.gam[1] = 0.0; g.gam[2] = H*st*ct;
      g.gam[3] = 0.0; g.gam[4] = r*r; g.gam[5] = 0.0;
      g.gam[6] = H*st*ct; g.gam[7] = 0.0; g.gam[8] = 1.0 + H*ct*ct; }
   {  double R = sqrt(r*r+z*z);
      double H = 2*M/R, st = r/R, ct = z/R, a2 = 1.0/(1.0 + H);
      g.igam[0] = (1.0 + H*ct*ct) * a2; g.igam[1] = 0.0; g.igam[2] = -H*st*ct*a2;
      g.igam[3] = 0.0; g.igam[4] = 1.0/(r*r); g.igam[5] = 0.0;
      g.igam[6] = -H*st*ct*a2; g.igam[7] = 0.0; g.igam[8] = (1.0 + H*st*st) * a2; }
   g.jac = x[0] / r;                         /* metric_jacobian(x)/r */
   g.sqrtgam = g.jac / g.al;
   double ia = 1.0/g.al;                     /* frame_U, Frame/normal.c:9-21 */
   g.U[0] = ia; g.U[1] = -ia*g.be[0]; g.U[2] = -ia*g.be[1]; g.U[3] = -ia*g.be[2];
}

/* Kerr-Schild (spin a) in cylindrical coordinates, closed form */
__host__ __device__ __forceinline__ void metric_kerr(const double *x, double M, double a, Metric3 &g){
   double r = x[0], z = x[2];
   double rho2 = r*r + z*z;
   double b = rho2 - a*a;
   double R2 = 0.5*(b + sqrt(b*b + 4.0*a*a*z*z));
   double R = sqrt(R2);
   double f = 2.0*M*R*R2/(R2*R2 + a*a*z*z);
   double den = R2 + a*a;
   double l[3] = { R*r/den, -a*r*r/den, z/R };          /* covariant */
   double lu[3] = { l[0], l[1]/(r*r), l[2] };           /* raised with diag(1, r^2, 1) */
   double flat[3] = {1.0, r*r, 1.0};
   double c = f/(1.0 + f);
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ){
      g.gam[3*i+j] = (i == j ? flat[i] : 0.0) + f*l[i]*l[j];
      g.igam[3*i+j] = (i == j ? 1.0/flat[i] : 0.0) - c*lu[i]*lu[j];
   }
   for( int i=0 ; i<3 ; ++i ) g.be[i] = c*lu[i];
   g.al = 1.0/sqrt(1.0 + f);
   g.jac = 1.0;                              /* alpha sqrt(gamma) / r */
   g.sqrtgam = g.jac / g.al;
   double ia = 1.0/g.al;
   g.U[0] = ia; g.U[1] = -ia*g.be[0]; g.U[2] = -ia*g.be[1]; g.U[3] = -ia*g.be[2];
}

__host__ __device__ __forceinline__ void metric_at(const GRParams &P, const double *x, Metric3 &g){
   if( P.metric == GR_METRIC_KERR ) metric_kerr(x, P.M, P.a, g);
   else metric_schw(x, P.M, g);
}

/* prim2cons, grmhd2.c:88-180 (per volume dV; 1 for the Riemann states) */
__host__ __device__ __forceinline__ void gr_prim2cons(const GRParams &P, const Metric3 &g,
                                                       const double *prim, double *cons,
                                                       const double *x, double dV = 1.0){
   double r = x[0];
   double gl = P.gam;
   double al = g.al, jac = g.jac, sqrtgam = g.sqrtgam;
   const double *be = g.be, *gam = g.gam, *igam = g.igam, *U = g.U;
   double rho = prim[RHO], Pp = prim[PPP];
   double l[3] = {prim[URR], prim[UPP], prim[UZZ]};
   double B[3] = {prim[BRR]/sqrtgam, prim[BPP]/(r*sqrtgam), prim[BZZ]/sqrtgam};
   double w, u0, u2, igaml[3];
   for( int i=0 ; i<3 ; ++i ){
      igaml[i] = 0.0;
      for( int j=0 ; j<3 ; ++j ) igaml[i] += igam[3*i+j]*l[j];
   }
   u2 = l[0]*igaml[0] + l[1]*igaml[1] + l[2]*igaml[2];
   w = sqrt(1.0 + u2);
   u0 = w/al;
   double l0 = -al*w + be[0]*l[0] + be[1]*l[1] + be[2]*l[2];
   double uU = U[0]*l0 + U[1]*l[0] + U[2]*l[1] + U[3]*l[2];
   double uB, b0, bd[3], B2, b2, UB, Ub;
   uB = l[0]*B[0] + l[1]*B[1] + l[2]*B[2];
   b0 = uB / al;
   bd[0] = (gam[0]*B[0] + gam[1]*B[1] + gam[2]*B[2] + l[0]*uB) / w;
   bd[1] = (gam[3]*B[0] + gam[4]*B[1] + gam[5]*B[2] + l[1]*uB) / w;
   bd[2] = (gam[6]*B[0] + gam[7]*B[1] + gam[8]*B[2] + l[2]*uB) / w;
   B2 = 0.0; UB = 0.0;
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ){
      B2 += gam[3*i+j]*B[i]*B[j];
      UB += gam[3*i+j] * B[i] * (U[0]*be[j] + U[j+1]);
   }
   b2 = (B2 + uB*uB) / (w*w);
   Ub = (UB + uU*uB) / w;
   double rhoh = rho + gl/(gl-1.0)*Pp + b2;
   double rhoe = Pp / (gl-1.0);
   cons[DDD] = jac * rho*u0 * dV;
   cons[SRR] = jac * (rhoh*u0*l[0] - b0*bd[0]) * dV;
   cons[LLL] = jac * (rhoh*u0*l[1] - b0*bd[1]) * dV;
   cons[SZZ] = jac * (rhoh*u0*l[2] - b0*bd[2]) * dV;
   cons[TAU] = jac * (-(rhoe+0.5*b2)*uU*u0 - (Pp+0.5*b2)*(uU*u0+U[0])
                           - rho*(uU+1.0)*u0 + Ub*b0) * dV;
   cons[BRR] = sqrtgam * B[0]/r * dV;
   cons[BPP] = sqrtgam * B[1] * dV;
   cons[BZZ] = sqrtgam * B[2] * dV;
   cons[8] = prim[8]*cons[DDD];
}

/* The solve's invariants (grmhd2.c:1124-1150) and the plain guess
 * (:1167-1175). */
struct C2PInv {
   double D, S[3], tau, B[3], s2, Q, psi, BS, B2, e, n, v20, eta0;
};
__host__ __device__ __forceinline__ void c2p_invariants(const GRParams &P, const Metric3 &g,
                                                         const double *cons, const double *prim,
                                                         const double *x, C2PInv &I){
   double r = x[0];
   const double *be = g.be, *gam = g.gam, *igam = g.igam, *U = g.U;
   double sqrtgam = g.sqrtgam, al = g.al;
   I.D = cons[DDD];
   I.S[0] = cons[SRR]; I.S[1] = cons[LLL]; I.S[2] = cons[SZZ];
   I.tau = cons[TAU];
   I.B[0] = r*cons[BRR]/sqrtgam; I.B[1] = cons[BPP]/sqrtgam; I.B[2] = cons[BZZ]/sqrtgam;
   double D = I.D;
   double s2 = 0.0, Us = 0.0, BS = 0.0, B2 = 0.0;
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ) s2 += igam[3*i+j]*I.S[i]*I.S[j];
   s2 /= D*D;
   for( int i=0 ; i<3 ; ++i ) Us += I.S[i]*(be[i]*U[0] + U[i+1]);
   Us /= D;
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ) B2 += gam[3*i+j]*I.B[i]*I.B[j];
   I.Q = sqrtgam * B2 / D;
   for( int i=0 ; i<3 ; ++i ) BS += I.B[i]*I.S[i];
   I.psi = sqrtgam * BS*BS / (D*D*D);
   I.s2 = s2; I.BS = BS; I.B2 = B2;
   I.e = (I.tau/D + Us + 1.0) / (al*U[0]);
   I.n = (P.gam-1.0)/P.gam;
   double u2 = 0.0;
   double l[3] = {prim[URR], prim[UPP], prim[UZZ]};
   for( int i=0 ; i<3 ; ++i ) for( int j=0 ; j<3 ; ++j ) u2 += igam[3*i+j]*l[i]*l[j];
   double w = sqrt(1.0 + u2);
   I.v20 = u2 / (1.0+u2);
   I.eta0 = w * (1.0 + P.gam/(P.gam-1.0)*prim[PPP]/prim[RHO]);
}

/* Newton-Raphson of grmhd2.c:1177-1236 from (v2, eta); returns iterations,
 * sets *ok when it stopped on the tolerance (not on max_iter). */
__host__ __device__ __forceinline__ int c2p_newton(const GRParams &P, const C2PInv &I,
                                                   double *pv2, double *peta, int *ok){
   double prec = P.tol;
   int max_iter = P.max_iter;
   int Nextra = P.nextra;
   double Q = I.Q, psi = I.psi, s2 = I.s2, e = I.e, n = I.n;
   double v2, v21 = *pv2, eta, eta1 = *peta, w;
   int i = 0, clean = -1;
   while( 1 ){
      v2 = v21;
      eta = eta1;
      w = 1.0/sqrt(1.0-v2);
      double fa = (eta+Q)*(eta+Q)*v2 - psi*(2*eta+Q)/(eta*eta) - s2;
      double fb = eta - n*(1-v2)*(eta-w) + 0.5*Q*(1+v2) - 0.5*psi/(eta*eta) - e;
      double dfadv2 = (eta+Q)*(eta+Q);
      double dfadet = 2*(eta+Q)*(v2 + psi/(eta*eta*eta));
      double dfbdv2 = n * (eta-0.5*w) + 0.5*Q;
      double dfbdet = 1 - n*(1-v2) + psi/(eta*eta*eta);
      double detj = dfadv2*dfbdet - dfbdv2*dfadet;
      v21  = v2  - ( dfbdet*fa - dfadet*fb)/detj;
      eta1 = eta - (-dfbdv2*fa + dfadv2*fb)/detj;
      i++;
      if( v21 > 1.0 ) v21 = 0.5*(v2 + 1.0);
      if( v21 < 0.0 ) v21 = 0.5*v2;
      if( eta1 < 1.0 ) eta1 = 0.5*(eta+1.0);
      double err = (eta1-eta)/eta;
      if( fabs(err) < prec && clean < 0 ) clean = Nextra+1;
      if( clean >= 0 ) clean--;
      if( clean == 0 || i == max_iter ) break;
   }
   *pv2 = v21; *peta = eta1;
   *ok = (clean == 0) && (eta1 == eta1) && (v21 == v21);
   return i;
}

/* Prim recovery, grmhd2.c:1238-1276 */
__host__ __device__ __forceinline__ void c2p_recover(const GRParams &P, const Metric3 &g,
                                                     const C2PInv &I, double v2, double eta,
                                                     const double *cons, double *prim, const double *x){
   double r = x[0];
   const double *gam = g.gam;
   double al = g.al, jac = g.jac, sqrtgam = g.sqrtgam;
   double D = I.D, BS = I.BS, B2 = I.B2, n = I.n, gl = P.gam;
   const double *S = I.S, *B = I.B;
   double w = 1.0/sqrt(1-v2);
   double u0 = w/al;
   double h = eta/w;
   double rho = D / (jac*u0);
   if( rho < P.rho_floor ) rho = P.rho_floor;
   double Pp = n * rho * (h-1.0);
   if( Pp < P.p_floor*rho ) Pp = P.p_floor*rho;
   h = 1.0 + gl/(gl-1.0) * Pp/rho;
   double Bd[3];
   Bd[0] = gam[0]*B[0] + gam[1]*B[1] + gam[2]*B[2];
   Bd[1] = gam[3]*B[0] + gam[4]*B[1] + gam[5]*B[2];
   Bd[2] = gam[6]*B[0] + gam[7]*B[1] + gam[8]*B[2];
   double l0 = (S[0] + sqrtgam*BS*Bd[0]/(D*h*w)) / (D*h + sqrtgam*B2/w);
   double l1 = (S[1] + sqrtgam*BS*Bd[1]/(D*h*w)) / (D*h + sqrtgam*B2/w);
   double l2 = (S[2] + sqrtgam*BS*Bd[2]/(D*h*w)) / (D*h + sqrtgam*B2/w);
   prim[RHO] = rho; prim[URR] = l0; prim[UPP] = l1; prim[UZZ] = l2; prim[PPP] = Pp;
   prim[BRR] = sqrtgam   * B[0];
   prim[BPP] = sqrtgam*r * B[1];
   prim[BZZ] = sqrtgam   * B[2];
   prim[8] = cons[8]/cons[DDD];
}

/* Scaled Newton residuals at the warm start (fa, fb of grmhd2.c:1185-1187
 * at (v2_0, eta_0)): ra = fa/(eta_0+Q)^2, rb = fb/eta_0.  Returns their size
 * sigma = |ra| + |rb| + 1e-14, the scale of the correction the guess needs. */
__host__ __device__ __forceinline__ double c2p_warm_residual(const C2PInv &I, double *ra, double *rb){
   const double v2 = I.v20, eta = I.eta0, Q = I.Q, psi = I.psi, n = I.n;
   const double w = 1.0/sqrt(1.0-v2);
   const double fa = (eta+Q)*(eta+Q)*v2 - psi*(2*eta+Q)/(eta*eta) - I.s2;
   const double fb = eta - n*(1-v2)*(eta-w) + 0.5*Q*(1+v2) - 0.5*psi/(eta*eta) - I.e;
   *ra = fa/((eta+Q)*(eta+Q));
   *rb = fb/eta;
   return fabs(*ra) + fabs(*rb) + 1e-14;
}

__host__ __device__ __forceinline__ float flog(float x){
#ifdef __CUDA_ARCH__
   return __logf(x);
#else
   return logf(x);
#endif
}

/* The network's 8 inputs: log e, log(1+s2), log(1+Q), log(1+|psi|),
 * log eta_0, log sigma, ra/sigma, rb/sigma.  The solution depends on the
 * invariants (s2, e, Q, psi) alone; the warm start enters through eta_0 and
 * its residual.  Returns sigma: the network predicts the corrections
 * (log eta - log eta_0, v2 - v2_0) divided by sigma, which keeps its
 * targets of order one whether the previous prims are close or far. */
__host__ __device__ __forceinline__ double mlp_features(const C2PInv &I, float *f){
   double ra, rb;
   const double sig = c2p_warm_residual(I, &ra, &rb);
   f[0] = flog((float)I.e);
   f[1] = flog(1.0f + (float)I.s2);
   f[2] = flog(1.0f + (float)I.Q);
   f[3] = flog(1.0f + (float)fabs(I.psi));
   f[4] = flog((float)I.eta0);
   f[5] = flog((float)sig);
   f[6] = (float)(ra/sig);
   f[7] = (float)(rb/sig);
   return sig;
}

} // namespace disco
