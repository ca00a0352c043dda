/*
 * disco_c2p -- C ABI of the B200-native GRMHD cons -> prim solve and its
 * learned initial guess.
 *
 * In the reference, calc_prim (misc.c:290-325) calls the Hydro module's
 *
 *     void cons2prim( const double *cons, double *prim,
 *                     const double *x, double dV );      Hydro/grmhd2.c:253-270
 *
 * once per real cell; for grmhd2 that is the Noble-2D Newton solve
 * (grmhd2.c:1096-1313) in (v^2, eta) started from the cell's previous prims,
 * stopped once |d eta/eta| < 1e-12 and then run 10 more iterations (at most
 * 30), followed by the prim recovery.  prim2cons (grmhd2.c:88-180) is its
 * inverse.  The metric is a compile-time module (Hydro/Metric/*.c); here it
 * is a run-time choice: DISCO_GR_SCHW_KS is schw_ks_rpz.c, DISCO_GR_KERR_KS
 * is a Kerr-Schild metric of spin a (new; equal to schw_ks_rpz at a = 0).
 * The frame is Frame/normal.c.
 *
 * disco_gr_cons2prim does calc_prim's loop for n cells in one launch.  All
 * cell arrays are DEVICE pointers in structure-of-arrays order: prim[q*n+i],
 * cons[q*n+i] (q = 0..8: RHO PPP URR UPP UZZ BRR BPP BZZ X for prims, DDD TAU
 * SRR LLL SZZ BRR BPP BZZ X for cons, NUM_C 8 + NUM_N 1), x[d*n+i] (r, phi,
 * z), per unit volume (dV = 1: divide by dV first, as cons2prim does).
 *
 * The learned guess (DISCO_GUESS_LEARNED) replaces the warm start with the
 * prediction of an 8 -> 64 -> 64 -> 2 tanh network (BF16 weights, FP32
 * accumulation on the tensor cores) from the solve's invariants and the warm
 * start.  Newton then runs to the same tolerance with the same tail; a cell
 * whose learned start does not converge is solved again from the warm start
 * (a fallback, counted).  The network is trained on the GPU by
 * disco_gr_mlp_train from (features, targets) pairs that plain solves write
 * (the `pairs` argument of disco_gr_cons2prim).
 *
 * Every function returns DISCO_OK or a DISCO_ERR_* code of disco_b200.h.
 */
#ifndef DISCO_C2P_H
#define DISCO_C2P_H

#ifdef __cplusplus
extern "C" {
#endif

enum disco_gr_metric { DISCO_GR_SCHW_KS = 0, DISCO_GR_KERR_KS = 1 };
enum disco_gr_guess  { DISCO_GUESS_PREVIOUS = 0, DISCO_GUESS_LEARNED = 1 };

/* Hydro and metric parameters.  gamma_law, rho_floor and p_floor are the
 * module's Adiabatic_Index, Density_Floor and Pressure_Floor
 * (grmhd2.c:53-58); M is Metric_Par2 (schw_ks_rpz.c:13-17); a is the spin of
 * the Kerr module.  tol, nextra and max_iter are the solve's prec, Nextra
 * and max_iter (grmhd2.c:1098-1100; the reference's values are 1e-12, 10, 30). */
typedef struct disco_gr_params {
   double gamma_law, rho_floor, p_floor;
   double M, a;
   double tol;
   int metric, nextra, max_iter, pad;
} disco_gr_params;

/* Iteration report of one disco_gr_cons2prim call.  iters counts Newton
 * iterations per cell, including those of a fallback solve; hist[k] counts
 * cells that took k iterations (k >= 63 in hist[63]).  n_fallback: cells
 * whose learned start failed and were solved again from the warm start;
 * n_fail: cells whose last solve stopped on max_iter. */
typedef struct disco_gr_stats {
   long long ncell, iters_sum;
   int iters_max, n_fallback, n_fail, pad;
   long long hist[64];
} disco_gr_stats;

/* The torus state module (disco_b200/csrc/gr_torus.h). */
typedef struct disco_gr_torus {
   double M, a, gam;
   double rc, wr, hr, K;
   double rho_atm, p_atm, B0, s_cut, amp;
   unsigned long long seed;
} disco_gr_torus;

/* Network sizes: parameters W1[64][8] b1[64] W2[64][64] b2[64] W3[2][64]
 * b3[2] (float; the W are held as BF16 on the device), normalisation
 * in_shift[8] in_scale[8] out_shift[2] out_scale[2].  A pair is 10 floats:
 * the 8 raw features (log D, log e, log1p s2, log1p Q, log1p|psi|, alpha,
 * v2_0, log eta_0) and the 2 raw targets (log eta - log eta_0, v2 - v2_0). */
#define DISCO_MLP_NPARAM 4866
#define DISCO_MLP_NNORM  20
#define DISCO_MLP_PAIR   10

typedef struct disco_gr disco_gr;

int  disco_gr_create(int device, const disco_gr_params *p, disco_gr **out);
void disco_gr_destroy(disco_gr *h);
/* Launch everything on this cudaStream_t (NULL: the legacy default stream). */
int  disco_gr_set_stream(disco_gr *h, void *stream);
const char *disco_gr_last_error(disco_gr *h);

/* Cell centres of an Nr x Nz x Np cylindrical grid (r log- or linearly
 * spaced edges in [rmin, rmax], z edges linear in [zmin, zmax], phi of cell
 * i at (i + 1/2) 2 pi/Np) into x[3n], n = Nr*Nz*Np, cell i + Np*(j + Nr*k). */
int  disco_gr_grid(disco_gr *h, int Nr, int Nz, int Np, double rmin, double rmax,
                   double zmin, double zmax, int log_r, double *x);
/* Torus prims at the n cell centres x (cell index = hash key). */
int  disco_gr_torus_prims(disco_gr *h, const disco_gr_torus *tp, long n, const double *x,
                          double *prim);
/* out = prim * (1 + eps u_q), u_q in [-1,1) hashed from (seed, cell, q). */
int  disco_gr_perturb(disco_gr *h, long n, const double *prim, double *out,
                      unsigned long long seed, double eps);

/* prim2cons (grmhd2.c:88-180) of n cells, dV = 1. */
int  disco_gr_prim2cons(disco_gr *h, long n, const double *prim, const double *x, double *cons);
/* cons2prim of n cells.  prim holds the previous prims on entry (the warm
 * start) and the solution on return.  iters (nullable, device, n bytes)
 * receives each cell's iteration count (saturated at 255); pairs (nullable,
 * device, 10 floats per cell) receives the training pair of each cell
 * (targets NaN where the solve did not converge); stats (nullable, host)
 * receives the report.  With guess = DISCO_GUESS_LEARNED the network must
 * have been set or trained first. */
int  disco_gr_cons2prim(disco_gr *h, long n, const double *cons, const double *x, double *prim,
                        int guess, unsigned char *iters, float *pairs, disco_gr_stats *stats);

/* Network state.  Host arrays.  set rounds the W to BF16 (nearest even);
 * get returns the W as the BF16 values widened to float. */
int  disco_gr_mlp_init(disco_gr *h, unsigned long long seed);
int  disco_gr_mlp_set(disco_gr *h, const float *param, const float *norm);
int  disco_gr_mlp_get(disco_gr *h, float *param, float *norm);
/* Fit the normalisation (mean and 1/std of the features, mean and std of the
 * targets) to the n pairs (device) with finite targets. */
int  disco_gr_mlp_fit_norm(disco_gr *h, long n, const float *pairs);
/* loss = sum over pairs and outputs of (y - t)^2 / (2 n) on normalised
 * targets, and its gradient (host, DISCO_MLP_NPARAM floats), over the n
 * pairs (device), computed by the training kernels. */
int  disco_gr_mlp_grad(disco_gr *h, long n, const float *pairs, float *grad, double *loss);
/* Adam on minibatches of `batch` pairs drawn (with replacement, hashed from
 * seed and step) from the n pairs (device); lr decays by cosine to lr/20.
 * loss_hist (nullable, host, `steps` doubles) receives each step's loss. */
int  disco_gr_mlp_train(disco_gr *h, long n, const float *pairs, int steps, int batch,
                        float lr, unsigned long long seed, double *loss_hist);
/* Which kernel disco_gr_mlp_grad / _train run: DISCO_MLP_TENSOR (the
 * default: the 128-sample group's four contractions as tcgen05.mma on the
 * tensor cores, BF16 operands, FP32 accumulation in tensor memory) or
 * DISCO_MLP_CUDA_CORES (the backward on the FP32 CUDA cores).  A tensor-
 * core wait that runs out (a bounded wait) returns DISCO_ERR_INTERNAL. */
#define DISCO_MLP_CUDA_CORES 0
#define DISCO_MLP_TENSOR 1
int  disco_gr_mlp_set_backend(disco_gr *h, int backend);

#ifdef __cplusplus
}
#endif
#endif
