/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * CPU restatement of the GRMHD cons -> prim path that the device solver
 * disco_b200/csrc/disco_c2p.cu implements, and of the learned guess's
 * network, written for checking only:
 *
 *   orc_gr_prim2cons   Hydro/grmhd2.c:88-180 (prim2cons, dV = 1)
 *   orc_gr_cons2prim   Hydro/grmhd2.c:253-270 -> :1096-1313 (noble2d), with
 *                      the tolerance (:1098 prec), the tail (:1100 Nextra)
 *                      and the cap (:1099 max_iter) as parameters, and the
 *                      iteration count returned
 *   metric 0           Hydro/Metric/schw_ks_rpz.c:20-81, frame Frame/normal.c:9-21
 *   metric 1           Kerr-Schild of spin a in cylindrical coordinates (a new
 *                      module; at a = 0 it is metric 0), restated from the
 *                      Kerr-Schild form g = eta + f l l
 *   orc_mlp_*          the 8 -> 64 -> 64 -> 2 tanh network of the learned
 *                      guess, forward and backward in double, with the BF16
 *                      roundings of the device GEMM operands applied at the
 *                      same points
 *
 * Metric 0 and the solve are pinned bit for bit against the reference's own
 * grmhd2.c built by the Makefile's c2p target (tests/test_c2p_oracle.py).
 * States are AoS: 9 values per state (RHO PPP URR UPP UZZ BRR BPP BZZ X for
 * prims, DDD TAU SRR LLL SZZ BRR BPP BZZ X for cons), x 3 per state.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#include "../disco_b200/csrc/gr_torus.h"

enum { P_RHO = 0, P_PPP = 1, P_URR = 2, P_UPP = 3, P_UZZ = 4, P_BRR = 5, P_BPP = 6, P_BZZ = 7 };
enum { C_DDD = 0, C_TAU = 1, C_SRR = 2, C_LLL = 3, C_SZZ = 4 };

static struct {
   double gam, rho_floor, p_floor, M, a, tol;
   int metric, nextra, max_iter;
} G = {5.0/3.0, 1e-10, 1e-10, 1.0, 0.0, 1e-12, 0, 10, 30};

void orc_gr_setup(double gam, double rho_floor, double p_floor, double M, double a,
                  int metric, double tol, int nextra, int max_iter){
   G.gam = gam; G.rho_floor = rho_floor; G.p_floor = p_floor; G.M = M; G.a = a;
   G.metric = metric; G.tol = tol; G.nextra = nextra; G.max_iter = max_iter;
}

typedef struct { double al, be[3], gam[9], igam[9], jac, sqrtgam, U[4]; } geo_t;

/* Schwarzschild-KS, each quantity as its own function computes it in
 * schw_ks_rpz.c (lapse :20, shift :26, gam :38, igam :60, jacobian :82) */
static double schw_lapse(const double *x){
   double R = sqrt(x[0]*x[0] + x[2]*x[2]);
   return 1.0/sqrt(1.0 + 2*G.M/R);
}
static void schw_shift(const double *x, double *b){
   double r = x[0], z = x[2], R = sqrt(r*r+z*z);
   double a2 = 1.0/(1.0 + 2*G.M/R);
   b[0] = 2*G.M*r/(R*R)*a2; b[1] = 0.0; b[2] = 2*G.M*z/(R*R)*a2;
}
static void schw_gam(const double *x, double *g){
   double r = x[0], z = x[2], R = sqrt(r*r+z*z);
   double H = 2*G.M/R, st = r/R, ct = z/R;
   g[0] = 1.0 + H*st*st; g[1] = 0.0; g[2] = H*st*ct;
   g[3] = 0.0; g[4] = r*r; g[5] = 0.0;
   g[6] = H*st*ct; g[7] = 0.0; g[8] = 1.0 + H*ct*ct;
}
static void schw_igam(const double *x, double *g){
   double r = x[0], z = x[2], R = sqrt(r*r+z*z);
   double H = 2*G.M/R, st = r/R, ct = z/R, a2 = 1.0/(1.0+H);
   g[0] = (1.0 + H*ct*ct)*a2; g[1] = 0.0; g[2] = -H*st*ct*a2;
   g[3] = 0.0; g[4] = 1.0/(r*r); g[5] = 0.0;
   g[6] = -H*st*ct*a2; g[7] = 0.0; g[8] = (1.0 + H*st*st)*a2;
}

/* Kerr-Schild in cylindrical (r, phi, z): R from R^4 - (rho^2 - a^2) R^2
 * - a^2 z^2 = 0, f = 2 M R^3/(R^4 + a^2 z^2), null covector
 * l = (R r/(R^2+a^2), -a r^2/(R^2+a^2), z/R); gamma = flat + f l l,
 * gamma^-1 = flat^-1 - f/(1+f) l^ l^ (l has unit flat norm), beta^i =
 * f/(1+f) l^i, alpha^2 = 1/(1+f), alpha sqrt(gamma) = r. */
static void kerr_geo(const double *x, geo_t *g){
   double r = x[0], z = x[2], a = G.a, M = G.M;
   double rho2 = r*r + z*z;
   double b = rho2 - a*a;
   double R2 = 0.5*(b + sqrt(b*b + 4.0*a*a*z*z));
   double R = sqrt(R2);
   double f = 2.0*M*R*R2/(R2*R2 + a*a*z*z);
   double den = R2 + a*a;
   double l[3], lu[3], flat[3], c;
   int i, j;
   l[0] = R*r/den; l[1] = -a*r*r/den; l[2] = z/R;
   lu[0] = l[0]; lu[1] = l[1]/(r*r); lu[2] = l[2];
   flat[0] = 1.0; flat[1] = r*r; flat[2] = 1.0;
   c = f/(1.0 + f);
   for( i=0 ; i<3 ; ++i ) for( j=0 ; j<3 ; ++j ){
      g->gam[3*i+j] = (i == j ? flat[i] : 0.0) + f*l[i]*l[j];
      g->igam[3*i+j] = (i == j ? 1.0/flat[i] : 0.0) - c*lu[i]*lu[j];
   }
   for( i=0 ; i<3 ; ++i ) g->be[i] = c*lu[i];
   g->al = 1.0/sqrt(1.0 + f);
   g->jac = 1.0;
}

static void geo_at(const double *x, geo_t *g){
   double ia;
   if( G.metric == 1 ){
      kerr_geo(x, g);
   }else{
      g->al = schw_lapse(x);
      schw_shift(x, g->be);
      schw_gam(x, g->gam);
      schw_igam(x, g->igam);
      g->jac = x[0]/x[0];
   }
   g->sqrtgam = g->jac/g->al;
   /* normal.c:9-21: U = (1/alpha, -beta/alpha) */
   ia = 1.0/(G.metric == 1 ? g->al : schw_lapse(x));
   g->U[0] = ia; g->U[1] = -ia*g->be[0]; g->U[2] = -ia*g->be[1]; g->U[3] = -ia*g->be[2];
}

/* grmhd2.c:88-180 */
static void p2c_one(const double *prim, double *cons, const double *x){
   geo_t g;
   double r = x[0], gl = G.gam;
   double rho, Pp, l[3], B[3], w, u0, u2, igaml[3], l0, uU, uB, b0, bd[3], B2, b2, UB, Ub, rhoh, rhoe;
   int i, j;
   geo_at(x, &g);
   rho = prim[P_RHO]; Pp = prim[P_PPP];
   l[0] = prim[P_URR]; l[1] = prim[P_UPP]; l[2] = prim[P_UZZ];
   B[0] = prim[P_BRR]/g.sqrtgam; B[1] = prim[P_BPP]/(r*g.sqrtgam); B[2] = prim[P_BZZ]/g.sqrtgam;
   for( i=0 ; i<3 ; ++i ){
      igaml[i] = 0.0;
      for( j=0 ; j<3 ; ++j ) igaml[i] += g.igam[3*i+j]*l[j];
   }
   u2 = l[0]*igaml[0] + l[1]*igaml[1] + l[2]*igaml[2];
   w = sqrt(1.0 + u2);
   u0 = w/g.al;
   l0 = -g.al*w + g.be[0]*l[0] + g.be[1]*l[1] + g.be[2]*l[2];
   uU = g.U[0]*l0 + g.U[1]*l[0] + g.U[2]*l[1] + g.U[3]*l[2];
   uB = l[0]*B[0] + l[1]*B[1] + l[2]*B[2];
   b0 = uB/g.al;
   for( i=0 ; i<3 ; ++i )
      bd[i] = (g.gam[3*i]*B[0] + g.gam[3*i+1]*B[1] + g.gam[3*i+2]*B[2] + l[i]*uB)/w;
   B2 = 0.0; UB = 0.0;
   for( i=0 ; i<3 ; ++i ) for( j=0 ; j<3 ; ++j ){
      B2 += g.gam[3*i+j]*B[i]*B[j];
      UB += g.gam[3*i+j]*B[i]*(g.U[0]*g.be[j] + g.U[j+1]);
   }
   b2 = (B2 + uB*uB)/(w*w);
   Ub = (UB + uU*uB)/w;
   rhoh = rho + gl/(gl-1.0)*Pp + b2;
   rhoe = Pp/(gl-1.0);
   cons[C_DDD] = g.jac*rho*u0*1.0;
   cons[C_SRR] = g.jac*(rhoh*u0*l[0] - b0*bd[0])*1.0;
   cons[C_LLL] = g.jac*(rhoh*u0*l[1] - b0*bd[1])*1.0;
   cons[C_SZZ] = g.jac*(rhoh*u0*l[2] - b0*bd[2])*1.0;
   cons[C_TAU] = g.jac*(-(rhoe+0.5*b2)*uU*u0 - (Pp+0.5*b2)*(uU*u0+g.U[0])
                        - rho*(uU+1.0)*u0 + Ub*b0)*1.0;
   cons[P_BRR] = g.sqrtgam*B[0]/r*1.0;
   cons[P_BPP] = g.sqrtgam*B[1]*1.0;
   cons[P_BZZ] = g.sqrtgam*B[2]*1.0;
   cons[8] = prim[8]*cons[C_DDD];
}

void orc_gr_prim2cons(long n, const double *prim, const double *x, double *cons){
   long i;
   for( i=0 ; i<n ; ++i ) p2c_one(prim + 9*i, cons + 9*i, x + 3*i);
}

/* Invariants of the solve (grmhd2.c:1124-1150) and the warm-start guess
 * (:1167-1175). inv: s2, e, Q, psi, BS, B2, D, n */
typedef struct { double s2, e, Q, psi, BS, B2, D, n, S[3], B[3], v20, eta0; } inv_t;

static void invariants(const double *cons, const double *prim, const double *x,
                       const geo_t *g, inv_t *I){
   double r = x[0], D = cons[C_DDD], s2 = 0, Us = 0, BS = 0, B2 = 0, u2 = 0, l[3], w;
   int i, j;
   I->S[0] = cons[C_SRR]; I->S[1] = cons[C_LLL]; I->S[2] = cons[C_SZZ];
   I->B[0] = r*cons[P_BRR]/g->sqrtgam; I->B[1] = cons[P_BPP]/g->sqrtgam; I->B[2] = cons[P_BZZ]/g->sqrtgam;
   for( i=0 ; i<3 ; ++i ) for( j=0 ; j<3 ; ++j ) s2 += g->igam[3*i+j]*I->S[i]*I->S[j];
   s2 /= D*D;
   for( i=0 ; i<3 ; ++i ) Us += I->S[i]*(g->be[i]*g->U[0] + g->U[i+1]);
   Us /= D;
   for( i=0 ; i<3 ; ++i ) for( j=0 ; j<3 ; ++j ) B2 += g->gam[3*i+j]*I->B[i]*I->B[j];
   I->Q = g->sqrtgam*B2/D;
   for( i=0 ; i<3 ; ++i ) BS += I->B[i]*I->S[i];
   I->psi = g->sqrtgam*BS*BS/(D*D*D);
   I->e = (cons[C_TAU]/D + Us + 1.0)/(g->al*g->U[0]);
   I->n = (G.gam-1.0)/G.gam;
   I->s2 = s2; I->BS = BS; I->B2 = B2; I->D = D;
   l[0] = prim[P_URR]; l[1] = prim[P_UPP]; l[2] = prim[P_UZZ];
   for( i=0 ; i<3 ; ++i ) for( j=0 ; j<3 ; ++j ) u2 += g->igam[3*i+j]*l[i]*l[j];
   w = sqrt(1.0 + u2);
   I->v20 = u2/(1.0+u2);
   I->eta0 = w*(1.0 + G.gam/(G.gam-1.0)*prim[P_PPP]/prim[P_RHO]);
}

/* grmhd2.c:1177-1236; returns the iteration count */
static int newton(const inv_t *I, double *pv2, double *peta, int *ok){
   double Q = I->Q, psi = I->psi, s2 = I->s2, e = I->e, n = I->n;
   double v2 = 0, eta = 0, v21 = *pv2, eta1 = *peta, w;
   int it = 0, clean = -1;
   for( ;; ){
      double fa, fb, dfadv2, dfadet, dfbdv2, dfbdet, detj, err;
      v2 = v21; eta = eta1;
      w = 1.0/sqrt(1.0-v2);
      fa = (eta+Q)*(eta+Q)*v2 - psi*(2*eta+Q)/(eta*eta) - s2;
      fb = eta - n*(1-v2)*(eta-w) + 0.5*Q*(1+v2) - 0.5*psi/(eta*eta) - e;
      dfadv2 = (eta+Q)*(eta+Q);
      dfadet = 2*(eta+Q)*(v2 + psi/(eta*eta*eta));
      dfbdv2 = n*(eta-0.5*w) + 0.5*Q;
      dfbdet = 1 - n*(1-v2) + psi/(eta*eta*eta);
      detj = dfadv2*dfbdet - dfbdv2*dfadet;
      v21 = v2 - (dfbdet*fa - dfadet*fb)/detj;
      eta1 = eta - (-dfbdv2*fa + dfadv2*fb)/detj;
      it++;
      if( v21 > 1.0 ) v21 = 0.5*(v2 + 1.0);
      if( v21 < 0.0 ) v21 = 0.5*v2;
      if( eta1 < 1.0 ) eta1 = 0.5*(eta+1.0);
      err = (eta1-eta)/eta;
      if( fabs(err) < G.tol && clean < 0 ) clean = G.nextra + 1;
      if( clean >= 0 ) clean--;
      if( clean == 0 || it == G.max_iter ) break;
   }
   *pv2 = v21; *peta = eta1;
   *ok = (clean == 0) && v21 == v21 && eta1 == eta1;
   return it;
}

/* grmhd2.c:1238-1276 */
static void recover(const inv_t *I, const geo_t *g, double v2, double eta,
                    const double *cons, double *prim, const double *x){
   double r = x[0], gl = G.gam, D = I->D, w, u0, h, rho, Pp, Bd[3], den;
   int i;
   w = 1.0/sqrt(1-v2);
   u0 = w/g->al;
   h = eta/w;
   rho = D/(g->jac*u0);
   if( rho < G.rho_floor ) rho = G.rho_floor;
   Pp = I->n*rho*(h-1.0);
   if( Pp < G.p_floor*rho ) Pp = G.p_floor*rho;
   h = 1.0 + gl/(gl-1.0)*Pp/rho;
   for( i=0 ; i<3 ; ++i ) Bd[i] = g->gam[3*i]*I->B[0] + g->gam[3*i+1]*I->B[1] + g->gam[3*i+2]*I->B[2];
   prim[P_RHO] = rho;
   for( i=0 ; i<3 ; ++i ){
      den = D*h + g->sqrtgam*I->B2/w;
      prim[P_URR+i] = (I->S[i] + g->sqrtgam*I->BS*Bd[i]/(D*h*w))/den;
   }
   prim[P_PPP] = Pp;
   prim[P_BRR] = g->sqrtgam*I->B[0];
   prim[P_BPP] = g->sqrtgam*r*I->B[1];
   prim[P_BZZ] = g->sqrtgam*I->B[2];
   prim[8] = cons[8]/cons[C_DDD];
}

/* Warm-start solve: prim holds the previous prims on entry. iters/ok may be
 * NULL. fin (nullable, 2 per state) receives the final (v2, eta). */
void orc_gr_cons2prim(long n, const double *cons, const double *x, double *prim,
                      int *iters, int *ok, double *fin){
   long i;
   for( i=0 ; i<n ; ++i ){
      geo_t g; inv_t I; int k, o;
      double v2, eta;
      geo_at(x + 3*i, &g);
      invariants(cons + 9*i, prim + 9*i, x + 3*i, &g, &I);
      v2 = I.v20; eta = I.eta0;
      k = newton(&I, &v2, &eta, &o);
      recover(&I, &g, v2, eta, cons + 9*i, prim + 9*i, x + 3*i);
      if( iters ) iters[i] = k;
      if( ok ) ok[i] = o;
      if( fin ){ fin[2*i] = v2; fin[2*i+1] = eta; }
   }
}

/* Newton from a given (v2, eta) guess per state; prim is output only. */
void orc_gr_newton_from(long n, const double *cons, const double *x, const double *guess,
                        double *prim, int *iters, int *ok){
   long i;
   for( i=0 ; i<n ; ++i ){
      geo_t g; inv_t I; int o;
      double v2 = guess[2*i], eta = guess[2*i+1], dummy[9] = {1, 1, 0, 0, 0, 0, 0, 0, 0};
      geo_at(x + 3*i, &g);
      invariants(cons + 9*i, dummy, x + 3*i, &g, &I);
      iters[i] = newton(&I, &v2, &eta, &o);
      ok[i] = o;
      recover(&I, &g, v2, eta, cons + 9*i, prim + 9*i, x + 3*i);
   }
}

/* The network's 8 raw features of a state and its warm start: log e,
 * log(1+s2), log(1+Q), log(1+|psi|), log eta_0, log sigma, ra/sigma,
 * rb/sigma, with ra = fa/(eta_0+Q)^2 and rb = fb/eta_0 the scaled Newton
 * residuals (grmhd2.c:1185-1187) at the warm start and sigma = |ra| + |rb|
 * + 1e-14; sig (nullable) receives sigma and warm (nullable, 2 per state)
 * the warm start (v2_0, eta_0).  Float logs, as the device. */
void orc_gr_features(long n, const double *cons, const double *x, const double *prim,
                     float *feat, double *sig, double *warm){
   long i;
   for( i=0 ; i<n ; ++i ){
      geo_t g; inv_t I; float *f = feat + 8*i;
      double v2, eta, w, fa, fb, ra, rb, sg;
      geo_at(x + 3*i, &g);
      invariants(cons + 9*i, prim + 9*i, x + 3*i, &g, &I);
      v2 = I.v20; eta = I.eta0;
      w = 1.0/sqrt(1.0-v2);
      fa = (eta+I.Q)*(eta+I.Q)*v2 - I.psi*(2*eta+I.Q)/(eta*eta) - I.s2;
      fb = eta - I.n*(1-v2)*(eta-w) + 0.5*I.Q*(1+v2) - 0.5*I.psi/(eta*eta) - I.e;
      ra = fa/((eta+I.Q)*(eta+I.Q));
      rb = fb/eta;
      sg = fabs(ra) + fabs(rb) + 1e-14;
      f[0] = logf((float)I.e); f[1] = logf(1.0f + (float)I.s2); f[2] = logf(1.0f + (float)I.Q);
      f[3] = logf(1.0f + (float)fabs(I.psi)); f[4] = logf((float)eta);
      f[5] = logf((float)sg); f[6] = (float)(ra/sg); f[7] = (float)(rb/sg);
      if( sig ) sig[i] = sg;
      if( warm ){ warm[2*i] = v2; warm[2*i+1] = eta; }
   }
}

void orc_gr_torus(const gr_torus_par *tp, long n, const double *x, const uint64_t *cell, double *prim){
   long i;
   for( i=0 ; i<n ; ++i ) gr_torus_prim(tp, x + 3*i, cell[i], prim + 9*i);
}

/* ---------------- network: 8 -> 64 -> 64 -> 2, tanh ---------------- */
#define NI 8
#define NH 64
#define NO 2

/* float -> bf16 -> float, round to nearest even (finite inputs); with
 * orc_mlp_exact(1) the rounding is skipped, which makes the loss smooth for
 * a finite-difference check of the backward formulas */
static int mlp_exact = 0;
void orc_mlp_exact(int on){ mlp_exact = on; }
static double bf16r(float v){
   uint32_t u; float o;
   if( mlp_exact ) return v;
   memcpy(&u, &v, 4);
   u += 0x7fffu + ((u >> 16) & 1u);
   u &= 0xffff0000u;
   memcpy(&o, &u, 4);
   return o;
}

/* param block: W1[NH][NI] b1[NH] W2[NH][NH] b2[NH] W3[NO][NH] b3[NO] (the
 * W entries are the BF16 weights, given as float); norm: in_shift[NI]
 * in_scale[NI] out_shift[NO] out_scale[NO]. grad (nullable) receives
 * d(loss)/d(param) in the same layout; loss = sum (y - t)^2 / (2 n) over
 * normalised outputs; out (nullable) receives the normalised outputs. */
double orc_mlp_loss_grad(long n, const float *param, const float *norm, const float *feat,
                         const float *target, double *grad, double *out){
   const float *W1 = param, *b1 = W1 + NH*NI, *W2 = b1 + NH, *b2 = W2 + NH*NH,
               *W3 = b2 + NH, *b3 = W3 + NO*NH;
   double *gW1 = grad, *gb1 = grad + NH*NI, *gW2 = gb1 + NH, *gb2 = gW2 + NH*NH,
          *gW3 = gb2 + NH, *gb3 = gW3 + NO*NH;
   long np = NH*NI + NH + NH*NH + NH + NO*NH + NO, s;
   double loss = 0.0;
   int i, j, k, o;
   if( grad ) for( s=0 ; s<np ; ++s ) grad[s] = 0.0;
   for( s=0 ; s<n ; ++s ){
      double xin[NI], h1[NH], g1[NH], h2[NH], g2[NH], y[NO], dy[NO], da2[NH], da1[NH];
      for( i=0 ; i<NI ; ++i ) xin[i] = bf16r((feat[NI*s+i] - norm[i])*norm[NI+i]);
      for( j=0 ; j<NH ; ++j ){
         double a = b1[j];
         for( i=0 ; i<NI ; ++i ) a += (double)W1[NI*j+i]*xin[i];
         h1[j] = tanh(a); g1[j] = mlp_exact ? h1[j] : bf16r((float)h1[j]);
      }
      for( k=0 ; k<NH ; ++k ){
         double a = b2[k];
         for( j=0 ; j<NH ; ++j ) a += (double)W2[NH*k+j]*g1[j];
         h2[k] = tanh(a); g2[k] = mlp_exact ? h2[k] : bf16r((float)h2[k]);
      }
      for( o=0 ; o<NO ; ++o ){
         double a = b3[o];
         for( k=0 ; k<NH ; ++k ) a += (double)W3[NH*o+k]*g2[k];
         y[o] = a;
         if( out ) out[NO*s+o] = a;
         if( target ){
            double d = a - target[NO*s+o];
            loss += d*d;
            dy[o] = d/(double)n;
         }
      }
      if( !grad || !target ) continue;
      for( o=0 ; o<NO ; ++o ){
         gb3[o] += dy[o];
         for( k=0 ; k<NH ; ++k ) gW3[NH*o+k] += dy[o]*g2[k];
      }
      for( k=0 ; k<NH ; ++k ){
         double d = 0.0;
         for( o=0 ; o<NO ; ++o ) d += (double)W3[NH*o+k]*dy[o];
         da2[k] = d*(1.0 - h2[k]*h2[k]);
         gb2[k] += da2[k];
         for( j=0 ; j<NH ; ++j ) gW2[NH*k+j] += da2[k]*g1[j];
      }
      for( j=0 ; j<NH ; ++j ){
         double d = 0.0;
         for( k=0 ; k<NH ; ++k ) d += (double)W2[NH*k+j]*da2[k];
         da1[j] = d*(1.0 - h1[j]*h1[j]);
         gb1[j] += da1[j];
         for( i=0 ; i<NI ; ++i ) gW1[NI*j+i] += da1[j]*xin[i];
      }
   }
   return target ? loss/(2.0*(double)n) : 0.0;
}
