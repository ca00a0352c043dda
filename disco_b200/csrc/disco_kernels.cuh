/*
 * Kernels of the B200 Disco timestep (hydro), templated on the bulk real
 * type R of the primitive variables, slopes and fluxes:
 *   R = double   the plain FP64 path, arithmetic identical to the reference
 *                (built with --fmad=false, same operation order);
 *   R = float    the mixed form: FP32 prim / PLM / Riemann arithmetic, FP64
 *                phi positions, mesh motion, face endpoints, dt reduction and
 *                a Kahan-compensated FP64 conserved update.
 *
 * Layout (device, one batch of one or more disks):
 *   cells      ragged SoA in annulus order; prim[q*Ncell + c] (R), cons (FP64),
 *              RKcons (FP64), ccarry (FP32 Kahan carry, mixed form), gradp,
 *              gradr (R);
 *              piph[c], dphi[c], wiph[c] (FP64)
 *   annuli     ann_off[a] .. ann_off[a]+ann_np[a]-1 are annulus a's cells
 *   tracks     track t joins annulus tr_a[t] (inner / lower) and tr_b[t]
 *              (outer / upper); its faces are tr_off[t] .. tr_off[t+1]-1
 *              (Np_a + Np_b of them, faces_alt.c:87-100).  Per disk the
 *              (Nr-1)*Nz r-tracks (tr_dim 1) come first, then the
 *              Nr*(Nz-1) z-tracks (tr_dim 2)
 *   faces      SoA: fL, fR (global cells), fLR, fphic, fdA, fdp (FP64),
 *              fS[q], fG[q] (R)
 *   consume    consL[c] = face of the r-track outside c that consumes c in the
 *              merge; consR[c] = same for the track inside c (consZL/consZR:
 *              the z-tracks above / below c).  They give each
 *              cell the contiguous runs of faces it belongs to, so every
 *              scatter of the reference (plm.c:82-110, riemann.c:312-315)
 *              becomes an order-preserving gather without atomics.
 *
 * Grids are block tables: cell kernels get one block per (annulus, chunk of
 * CB cells), face kernels one block per (track, chunk of FB faces).
 */
#pragma once
#include "disco_device.cuh"
#include "grmhd_step.cuh"

#include "tuned.h"
#if __has_include("tuned_mhd.h")
#include "tuned_mhd.h"
#endif

namespace disco {

/* threads per block of the cell kernels (one block per annulus chunk of CB
 * cells) and of the face kernels (FB faces of one track); tuned.h may set
 * them, the host's block tables and every launch follow */
#ifndef CB
#define CB 128
#endif
#ifndef FB
#define FB CB
#endif
/* Resident blocks per SM asked of the compiler for the step kernels (the
 * register budget per thread follows: 65536 / (CB * MB)).  The kernels
 * are latency-bound, so warps in flight matter more than the spills the
 * tighter budget costs: on ragged64 the hydro step went from 7.26 to
 * 5.41 ms (FP64) and 5.60 to 4.57 ms (mixed) with MB 8-12 against the
 * compiler's choice (MB 1).  tuned.h holds the per-kernel values the
 * autotuner (disco_b200/autotune.py) measured on a B200, per precision
 * (DISCO_MIXED_TU marks the FP32 translation unit); a -DMB_x on the
 * command line overrides them, and the defaults below fill the rest.  The
 * MHD instantiations (HLLD needs about 160 registers) take MB_MHD_* from
 * tuned_mhd.h, the same autotuner's values for Q = 9 measured on the
 * config-4 slab, else MB_MHD. */
#ifndef MB_FACES
#define MB_FACES 1
#endif
#ifndef MB_STEP
#define MB_STEP 8
#endif
#ifndef MB_MHD
#define MB_MHD 4
#endif
/* per kernel, for the MHD instantiations */
#ifndef MB_MHD_BEGIN
#define MB_MHD_BEGIN MB_MHD
#endif
#ifndef MB_MHD_GRAD
#define MB_MHD_GRAD MB_MHD
#endif
#ifndef MB_MHD_FLUX
#define MB_MHD_FLUX MB_MHD
#endif
#ifndef MB_MHD_UPDATE
#define MB_MHD_UPDATE MB_MHD
#endif
#ifndef MB_MHD_C2P
#define MB_MHD_C2P MB_MHD
#endif
#ifndef MB_BEGIN
#define MB_BEGIN 10
#endif
#ifndef MB_GRAD
#define MB_GRAD 12
#endif
#ifndef MB_FLUX
#define MB_FLUX MB_STEP
#endif
#ifndef MB_UPDATE
#define MB_UPDATE MB_STEP
#endif
#ifndef MB_C2P
#define MB_C2P MB_STEP
#endif
/* the grmhd2 (GR) instantiations of the step kernels: resident blocks per
 * SM measured on the config-3 torus (192 x 16 x 462 slice, Kerr a = 0.9)
 * for 2-6 blocks: 5 for the flux kernels and k_update (2-4 spill less but
 * hide less latency: 8.4-10.1 ms per step at 2-3 against 7.4 at 5), 6 for
 * k_begin and k_c2p */
#ifndef MB_GR
#define MB_GR 5
#endif
#ifndef MB_GR_LIGHT
#define MB_GR_LIGHT 6
#endif

template<class R>
struct ViewT {
   int Ncell, Nann, Ntr, Nf;
   const int *ann_off, *ann_np, *ann_disk, *ann_j, *ann_k;
   const int *tr_a, *tr_b, *tr_off, *tr_flux, *tr_j, *tr_k;
   const unsigned char *tr_dim;      /* 1: r-track (j,k)-(j+1,k); 2: z-track (j,k)-(j,k+1) */
   const double *tr_dxL, *tr_dxR;
   const double *tr_r, *tr_irf;       /* face centre radius of the track's faces, 1/(1/r) */
   const double *ann_rc;              /* centroid radius of the annulus (get_centroid(.,.,1)) */
   const int2 *cblk, *fblk;
   const int2 *ublk;                  /* k_update: (annulus, first cell) of chunks of CB-1 cells */
   const double *rj, *zk;
   const DiskParams *dp;
   DiskState *ds;
   R *prim, *gradp, *gradr, *gradz;   /* gradz only when a disk has Nz > 1 */
   double *cons, *RKcons;
   float *ccarry;       /* Kahan carry of cons (mixed form): below half an ulp of cons,
                         * so FP32 keeps 24 more bits of the sum than cons has */
   double *piph, *dphi, *wiph, *piph_new;
   int *I0;
   int *fL, *fR;
   unsigned char *fLR;
   double *fphic, *fdA, *fdp;
   R *fS, *fG;
   int *consL, *consR;                /* r-tracks outside / inside the cell */
   int *consZL, *consZR;              /* z-tracks above / below the cell */
   double *diag_part;   /* per cell block: nq sums + volume */
   const double *noise; /* addNoise draws, 4 per cell (set-up and restart), or NULL */
   /* *topo = 1 when the face lists and geometry were built from the current
    * piph (the second RK2 substep builds them after the cells have moved, so
    * the next step's first substep, with the same piph, keeps them and only
    * re-evaluates the face slopes); topo_reuse / topo_set select the
    * behaviour of one launch sequence. */
   int *topo;
   int topo_reuse, topo_set;
   /* move_cells + calc_dp of the first substep, done by k_c2p (1) or by the
    * constrained-transport update (0): k_update reads the neighbour cells'
    * pre-move dphi across its chunk edges, so it must not move any cell */
   int move_c2p;
   /* energy-frame Omega of omega.c:62-110, evaluated once by k_precompute at
    * the radii the step uses (same device expressions, so bit-identical to
    * evaluating them in place): annulus centroid (om, dOm/dr) and r-face */
   double *ann_om, *ann_om1, *tr_om;
   int nq;
   double dtfac;        /* 1 in the first substep, 0.5 in the second (timestep.c:39) */
   int *err;
   /* Constrained transport (Constrained_Transport 1; bfields.c), ct = the
    * CT_MODE (1: 2D, NUM_FACES 3; 2: 3D, NUM_FACES 5) or 0.  Per cell, SoA
    * [s*Ncell + c]: Phi / RKPhi, s = 0 the magnetic flux through the cell's
    * phi face at piph, s = 1 / 2 the flux through the r-face the cell owns in
    * the track inside / outside it (the face ending at its piph, LRtype 1 /
    * 0), s = 3 / 4 the same for the z-faces below / above it; ctE / ctB the
    * edge values E[0..7], B[0..7] (riemann.c:73-110, 175-213) before
    * averaging (FP32 in the mixed form, whose face fluxes stay FP64); pE, pB, pEr, pBz the phi face's (Ez, Br, Er, Bz) from
    * flux_to_E.  Per face (r and z): fEt / fBt (Erz, Brz), fEphi (E_phi),
    * fX the E dl dt of update_B_fluxes, fFlip the flag of check_flipped.
    * 3D: rk[m*Ncell + c] the position of cell c in the 4-way merge of the
    * edge line where it is list m (make_edge_adjust's c, cR, cU, cUR), and
    * lineX[line_off[l] + e] the E_phi dl dt of merged edge e of line l. */
   int ct, nfs;
   double *Phi, *RKPhi, *fX;            /* the face fluxes stay FP64 in both forms */
   /* grmhd2: the metric at the fixed points where the step evaluates it
    * (k_gr_tables; NULL for the Newtonian modules) */
   GRAnn *gr_ann;
   Metric3 *gr_tr;
   /* cons->prim inputs of the real cells, SoA [21][Ncell]: cons / dV (9), the
    * warm-start prims (9), x (3), written by each GR c2p when set
    * (disco_batch_set_gr_dump; NULL otherwise) */
   double *gr_dump;
   /* horizon_bin: a cell once excised stays out of the dt minimum (the
    * reference's real flag is never set back); NULL for other modules */
   unsigned char *xflag;
   R *ctE, *ctB, *pE, *pB, *pEr, *pBz, *fEt, *fBt, *fEphi;   /* edge arithmetic: R */
   /* 3D CT with a z boundary without ghosts: each pole cell's owned z-face
    * E (avg_Efields' z-pole average, k_ct_zpole); NULL otherwise */
   double *ctPole;
   unsigned char *fFlip;
   int *rk, *line_off;
   double *lineX;
};

template<class R>
__device__ __forceinline__ void raise_err(const ViewT<R> &v, int e){
   if( e ) atomicOr(v.err, e);
}

/* cons += x, plain in the FP64 path, Kahan-compensated in the mixed form */
template<class R>
__device__ __forceinline__ void acc(double &s, double &cc, double x){
   if constexpr ( sizeof(R) == sizeof(double) ){
      s += x;
   }else{
      double y = x - cc;
      double t = s + y;
      cc = (t - s) - y;
      s = t;
   }
}

/* ------------------------------------------------------------------ k_begin
 * First substep: RK snapshot (timestep.c:18-24), set_wcell (misc.c:101-168,
 * modes 0/1/2/4; mode 3's mean is k_wmean), the moved-and-wrapped piph of
 * move_cells + clean_pi (misc.c:256-268, 8-26) into piph_new.
 * Every substep: adjust_RK_cons (misc.c:226-244) and plm_phi (plm.c:15-51). */
template<int Q, int NC, class R, bool GR = false>
__device__ __forceinline__ void begin_body(const ViewT<R> &v, double RK, int first, int bid){
   /* the chunk's prims and dphi staged once, with one neighbour cell on each
    * side (slot t+1 = cell i0+t) */
   __shared__ R sp[Q][CB+2];
   __shared__ double sd[CB+2];
   int2 b = v.cblk[bid];
   int a = b.x, i0 = b.y, t = threadIdx.x, i = i0 + t;
   int np = v.ann_np[a];
   const int N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + i;
   int nact = np - i0 < CB ? np - i0 : CB;
   auto stage = [&](int slot, int cell){
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) sp[q][slot] = v.prim[q*N + cell];
      sd[slot] = v.dphi[cell];
   };
   if( t < nact ) stage(t+1, c);
   if( t == 0 ) stage(0, c0 + (i0 == 0 ? np-1 : i0-1));
   if( t == nact-1 ) stage(nact+1, c0 + (i0+nact == np ? 0 : i0+nact));
   __syncthreads();
   if( t >= nact ) return;
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];

   R pC[Q], pL[Q], pR[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){
      pC[q] = sp[q][t+1]; pL[q] = sp[q][t]; pR[q] = sp[q][t+2];
   }
   if( first ){
      double w = 0.0;
      if constexpr ( GR ){          /* get_omega of grmhd2, grmhd2.c:64-86 (set_wcell's x) */
         if( P.mesh_motion ){
            int j = v.ann_j[a], k = v.ann_k[a];
            const double *rj = v.rj + P.rj0 + 1, *zk = v.zk + P.zk0 + 1;
            double x[3] = {centroid_r(rj[j], rj[j-1]), 0.0, centroid_z(zk[k], zk[k-1])};
            double pc[Q], pr[Q];
#pragma unroll
            for( int q=0 ; q<Q ; ++q ){ pc[q] = (double)pC[q]; pr[q] = (double)pR[q]; }
            (void)x;
            w = .5*(gr_omega(v.gr_ann[a].c, pc) + gr_omega(v.gr_ann[a].c, pr));
         }
      }else{
         if( P.mesh_motion ) w = .5*((double)pC[UPP] + (double)pR[UPP]);   /* get_omega = prim[UPP] */
      }
      if( P.mesh_motion == 4 ){
         int j = v.ann_j[a];
         const double *rj = v.rj + P.rj0 + 1;
         w = mesh_om(P, centroid_r(rj[j], rj[j-1]));
      }
      v.wiph[c] = w;
      if( P.mesh_motion != 3 ){
         int err = 0;
         /* move_cells: never contracted to an FMA, so both forms move alike */
         double phi = __dadd_rn(v.piph[c], __dmul_rn(w, v.ds[d].dt));
         int n = 0;
         while( phi > P.Pmax ){ phi -= P.Pmax; if( ++n > WRAP_CAP ){ err |= ERRF_WRAP; break; } }
         while( phi < 0.0 ){ phi += P.Pmax; if( ++n > WRAP_CAP ){ err |= ERRF_WRAP; break; } }
         v.piph_new[c] = phi;
         raise_err(v, err);
      }
   }
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){
      double cq = v.cons[q*N + c];
      double rk;
      if( first ){ rk = cq; v.RKcons[q*N + c] = cq; }
      else rk = v.RKcons[q*N + c];
      /* with RK = 0 (the first substep) the average returns a finite cq
       * bit for bit, so the store is skipped */
      if( !(RK == 0.0 && isfinite(cq)) ) v.cons[q*N + c] = (1.-RK)*cq + RK*rk;
      if constexpr ( sizeof(R) != sizeof(double) ){
         /* the carry belongs to cons; averaged with it (RKcons keeps none) */
         if( !first ) v.ccarry[q*N + c] = (float)((1.-RK)*(double)v.ccarry[q*N + c]);
      }
   }
   if constexpr ( NC == 8 ){
      if( v.ct ){                   /* timestep.c:22 and adjust_RK_cons, misc.c:239-241 */
#pragma unroll
         for( int s=0 ; s<5 ; ++s ){
            if( s >= v.nfs ) break;
            double ph = v.Phi[s*N + c];
            double rk;
            if( first ){ rk = ph; v.RKPhi[s*N + c] = ph; }
            else rk = v.RKPhi[s*N + c];
            if( !(RK == 0.0 && isfinite(ph)) ) v.Phi[s*N + c] = (1.-RK)*ph + RK*rk;
         }
      }
   }
   const R dpL = (R)sd[t], dpC = (R)sd[t+1], dpR = (R)sd[t+2];
   const R PLM = (R)P.PLM;
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){
      R sL = pC[q] - pL[q];  sL /= R(.5)*( dpC + dpL );
      R sR = pR[q] - pC[q];  sR /= R(.5)*( dpR + dpC );
      R sC = pR[q] - pL[q];  sC /= R(.5)*( dpL + dpR ) + dpC;
      R aa = PLM*sL, bb = sC, cc = PLM*sR;                /* minmod, plm.c:6 */
      R m = aa;
      if( aa*bb < R(0.0) ) m = R(0.0);
      if( fabs(bb) < fabs(m) ) m = bb;
      if( bb*cc < R(0.0) ) m = R(0.0);
      if( fabs(cc) < fabs(m) ) m = cc;
      v.gradp[q*N + c] = m;
   }
}
template<int Q, int NC, class R, bool GR = false>
__global__ void __launch_bounds__(CB, GR ? MB_GR_LIGHT : (Q > 6 ? MB_MHD_BEGIN : MB_BEGIN)) k_begin(ViewT<R> v, double RK, int first){
   begin_body<Q,NC,R,GR>(v, RK, first, blockIdx.x);
}

/* Energy-frame Omega at the radii the step evaluates it (omega.c:62-110):
 * annulus centroids (sources, phi faces, c2p) and r-faces (trans_flux). */
template<class R>
__global__ void k_precompute(ViewT<R> v){
   int x = blockIdx.x*blockDim.x + threadIdx.x;
   if( x < v.Nann ){
      const DiskParams &P = v.dp[v.ann_disk[x]];
      const double *rj = v.rj + P.rj0 + 1;
      int j = v.ann_j[x];
      double r = centroid_r(rj[j], rj[j-1]);
      v.ann_om[x] = get_om(P, r);
      v.ann_om1[x] = get_om1(P, r);
   }
   if( x < v.Ntr ){
      const DiskParams &P = v.dp[v.ann_disk[v.tr_a[x]]];
      const double *rj = v.rj + P.rj0 + 1;
      int j = v.tr_j[x];
      v.tr_om[x] = get_om(P, v.tr_dim[x] == 1 ? .5*(rj[j]+rj[j]) : centroid_r(rj[j], rj[j-1]));
   }
}

/* grmhd2's metric tables (GRAnn per annulus, Metric3 per track at the face
 * centre: (r_{j+1/2}, centroid z) for r-faces, (centroid r, z_{k+1/2}) for
 * z-faces, addFace faces_alt.c:10-16), once per batch */
template<class R>
__global__ void k_gr_tables(ViewT<R> v){
   int x = blockIdx.x*blockDim.x + threadIdx.x;
   if( x < v.Nann ){
      const DiskParams &P = v.dp[v.ann_disk[x]];
      const double *rj = v.rj + P.rj0 + 1, *zk = v.zk + P.zk0 + 1;
      int j = v.ann_j[x], k = v.ann_k[x];
      gr_ann_table(P, rj[j], rj[j-1], zk[k], zk[k-1], v.gr_ann[x]);
   }
   if( x < v.Ntr ){
      const DiskParams &P = v.dp[v.ann_disk[v.tr_a[x]]];
      const double *rj = v.rj + P.rj0 + 1, *zk = v.zk + P.zk0 + 1;
      int j = v.tr_j[x], k = v.tr_k[x];
      double xf[3];
      if( v.tr_dim[x] == 1 ){ xf[0] = .5*(rj[j]+rj[j]); xf[2] = 0.5*(zk[k]+zk[k-1]); }
      else { xf[0] = centroid_r(rj[j], rj[j-1]); xf[2] = 0.5*(zk[k]+zk[k]); }
      xf[1] = 0.0;
      metric_at(gr_params(P), xf, v.gr_tr[x]);
   }
}

/* Mesh_Motion 3 (misc.c:138-152): annulus mean of w, summed in cell order
 * (one warp per annulus: lane 0 adds the values in cell order from shared
 * memory, the warp loads and writes), then the move of the first substep
 * (move != 0) or not (set-up). */
#define WM_WARPS 4
#define WM_CHUNK 256
template<class R>
__global__ void __launch_bounds__(32*WM_WARPS) k_wmean(ViewT<R> v, int move){
   __shared__ double s_w[WM_WARPS][WM_CHUNK];
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   const int a = blockIdx.x*WM_WARPS + warp;
   if( a >= v.Nann ) return;
   const int np = v.ann_np[a], c0 = v.ann_off[a];
   const int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   if( P.mesh_motion != 3 ) return;
   double w = 0.0;
   for( int base=0 ; base<np ; base+=WM_CHUNK ){
      const int n = np - base < WM_CHUNK ? np - base : WM_CHUNK;
      for( int t=lane ; t<n ; t+=32 ) s_w[warp][t] = v.wiph[c0+base+t];
      __syncwarp();
      if( lane == 0 ) for( int t=0 ; t<n ; ++t ) w += s_w[warp][t];
      __syncwarp();
   }
   w = __shfl_sync(0xffffffffu, w, 0);
   w /= (double)np;
   const double dt = v.ds[d].dt;
   int err = 0;
   for( int i=lane ; i<np ; i+=32 ){
      v.wiph[c0+i] = w;
      if( move ){
         double phi = __dadd_rn(v.piph[c0+i], __dmul_rn(w, dt));
         int n = 0;
         while( phi > P.Pmax ){ phi -= P.Pmax; if( ++n > WRAP_CAP ){ err |= ERRF_WRAP; break; } }
         while( phi < 0.0 ){ phi += P.Pmax; if( ++n > WRAP_CAP ){ err |= ERRF_WRAP; break; } }
         v.piph_new[c0+i] = phi;
      }
   }
   raise_err(v, err);
}

/* ------------------------------------------------------------------ k_I0
 * faces_alt.c:57-79: I0 = first cell in quadrant I after any cell in
 * quadrant IV (the cell whose upper edge is just past phi = 0).  One warp
 * per annulus, ballots over 32-cell chunks. */
template<class R>
__device__ __forceinline__ void I0_body(const ViewT<R> &v, int topo_reuse, int warp, int lane){
   if( warp >= v.Nann ) return;
   if( topo_reuse && *v.topo ) return;
   int a = warp;
   int np = v.ann_np[a], c0 = v.ann_off[a];
   const DiskParams &P = v.dp[v.ann_disk[a]];
   double convert = 2.*DISCO_PI/P.Pmax;
   int first4 = -1, res = 0;
   for( int base=0 ; base<np ; base+=32 ){
      int i = base + lane;
      bool q1 = false, q4 = false;
      if( i < np ){
         double s, cs;
         sincos(v.piph[c0+i]*convert, &s, &cs);
         q1 = (s > 0. && cs > 0.);
         q4 = (s < 0. && cs > 0.);
      }
      unsigned m4 = __ballot_sync(0xffffffffu, q4);
      unsigned m1 = __ballot_sync(0xffffffffu, q1);
      if( first4 < 0 && m4 ){
         int l4 = __ffs(m4) - 1;
         first4 = base + l4;
         unsigned after = (l4 == 31) ? 0u : (m1 & (0xffffffffu << (l4+1)));
         if( after ){ res = base + __ffs(after) - 1; break; }
      }else if( first4 >= 0 && m1 ){
         res = base + __ffs(m1) - 1; break;
      }
   }
   if( lane == 0 ) v.I0[a] = res;
}
template<class R>
__global__ void k_I0(ViewT<R> v){
   I0_body<R>(v, v.topo_reuse, (blockIdx.x*blockDim.x + threadIdx.x) >> 5, threadIdx.x & 31);
}

/* The first x in [lo, hi) where the monotone predicate p turns true (hi if
 * it never does) -- the binary search's answer -- found by galloping out
 * from a guess g and bisecting the bracket: a few probes when g is close,
 * as the position of a face or edge in the other annulus usually is.  The
 * guess only sets where the search starts (computed in FP32, it may be off
 * by one either way); the answer is the bisection's whatever it is. */
template<class Pr>
__device__ __forceinline__ int gallop_lb(int lo, int hi, int g, Pr p){
   if( g < lo ) g = lo;
   if( g > hi ) g = hi;
   int a, b;
   if( g < hi && !p(g) ){            /* the answer lies above g */
      a = g + 1; b = hi;
      for( int step=1 ; a + step - 1 < hi ; step <<= 1 ){
         const int x = a + step - 1;
         if( p(x) ){ b = x; break; }
         a = x + 1;
      }
   }else{                            /* at or below g */
      a = lo; b = g;
      for( int step=1 ; b - step >= lo ; step <<= 1 ){
         const int x = b - step;
         if( !p(x) ){ a = x + 1; break; }
         b = x;
      }
   }
   while( a < b ){
      const int mid = (a + b) >> 1;
      if( p(mid) ) b = mid; else a = mid + 1;
   }
   return a;
}

/* ------------------------------------------------------------------ faces
 * buildfaces (faces_alt.c:102-177) as a merge path: face d of a track is
 * the d-th step of the reference's two-pointer merge, found by binary
 * search on the diagonal over the two annuli's edges unrolled from I0.
 * Within one cell width the unrolled order equals the reference's wrapped
 * comparison, so (iL, iR, LRtype) are the reference's; the face's own
 * LR / LR_back and geometry are then evaluated exactly as :140-164 and
 * addFace (:10-34) do (FP64 in both forms).  Also stores the PLM face
 * slopes S_q of plm_trans (plm.c:82-89) when with_slopes is set: the
 * gather reads each twice (sum, limiter), and recomputing them there from
 * the two cells' scattered states was measured 5x slower than storing. */
template<int Q, class R>
__device__ __forceinline__ void faces_body(const ViewT<R> &v, int with_slopes, int topo_reuse, int bid){
   int2 b = v.fblk[bid];
   int t = b.x, dd = b.y + threadIdx.x;
   int A = v.tr_a[t], B = v.tr_b[t];
   int NA = v.ann_np[A], NB = v.ann_np[B];
   if( dd >= NA + NB ) return;
   const int N = v.Ncell;
   int f = v.tr_off[t] + dd;
   int cA0 = v.ann_off[A], cB0 = v.ann_off[B];
   int IA = v.I0[A], IB = v.I0[B];
   const DiskParams &P = v.dp[v.ann_disk[A]];
   double Pmax = P.Pmax;
   int err = 0;

   if( topo_reuse && *v.topo ){     /* same piph as the last build: slopes only */
      if( !with_slopes ) return;
      int cL = v.fL[f], cR = v.fR[f];
      double phic = v.fphic[f];
      R dxL = (R)v.tr_dxL[t], dxR = (R)v.tr_dxR[t];
      double phiL = v.piph[cL] - .5*v.dphi[cL], phiR = v.piph[cR] - .5*v.dphi[cR];
      R dpL = (R)get_signed_dp(phic, phiL, Pmax, &err);
      R dpR = (R)get_signed_dp(phiR, phic, Pmax, &err);
#pragma unroll
      for( int q=0 ; q<Q ; ++q ){
         R WL = v.prim[q*N + cL] + dpL*v.gradp[q*N + cL];
         R WR = v.prim[q*N + cR] - dpR*v.gradp[q*N + cR];
         v.fS[(size_t)q*v.Nf + f] = (WR-WL)/(dxR+dxL);
      }
      raise_err(v, err);
      return;
   }
   int lo = dd - NB > 0 ? dd - NB : 0;
   int hi = dd < NA ? dd : NA;
   /* the diagonal's split: both annuli's edges are unrolled from I0, so face
    * dd lies near phi = dd/(NA+NB) of the turn in both */
   lo = gallop_lb(lo, hi, __float2int_rz(__fdividef((float)dd*(float)NA, (float)(NA+NB))), [&](int mid){
      int ia = IA + mid;       if( ia >= NA ) ia -= NA;
      int ib = IB + dd - mid - 1; if( ib >= NB ) ib -= NB;
      return v.piph[cA0+ia] > v.piph[cB0+ib];
   });
   int ka = lo, kb = dd - lo;
   int ia = IA + ka; while( ia >= NA ) ia -= NA;
   int ib = IB + kb; while( ib >= NB ) ib -= NB;
   int cL = cA0 + ia, cR = cB0 + ib;

   double pL = v.piph[cL], pR = v.piph[cR];
   double dL = v.dphi[cL], dR = v.dphi[cR];
   double dphi = pL - pR;
   int n = 0;
   while( dphi > .5*Pmax ){ dphi -= Pmax; if( ++n > WRAP_CAP ){ err |= ERRF_WRAP; break; } }
   while( dphi <-.5*Pmax ){ dphi += Pmax; if( ++n > WRAP_CAP ){ err |= ERRF_WRAP; break; } }
   int LR = dphi > 0. ? 1 : 0;
   dphi = pL-dL - pR+dR;
   n = 0;
   while( dphi > .5*Pmax ){ dphi -= Pmax; if( ++n > WRAP_CAP ){ err |= ERRF_WRAP; break; } }
   while( dphi <-.5*Pmax ){ dphi += Pmax; if( ++n > WRAP_CAP ){ err |= ERRF_WRAP; break; } }
   int LR_back = dphi < 0. ? 1 : 0;
   double xp1 = LR == 0 ? pL : pR;
   double xm1 = LR_back == 0 ? pL-dL : pR-dR;

   int j = v.tr_j[t], k = v.tr_k[t];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   double dp = get_dp(xp1, xm1, Pmax, &err);
   double phic = get_dp(xp1, .5*dp, Pmax, &err);
   double dA;
   if( v.tr_dim[t] == 1 ){
      double r = .5*(rj[j]+rj[j]);
      double dz = zk[k]-zk[k-1];
      dA = r*dp*dz;                                       /* get_dA(.,.,1) */
   }else{
      double r = .5*(rj[j]+rj[j-1]);
      double dr = rj[j]-rj[j-1];
      dA = r*dr*dp;                                       /* get_dA(.,.,2) */
   }

   v.fL[f] = cL; v.fR[f] = cR; v.fLR[f] = (unsigned char)LR;
   v.fphic[f] = phic; v.fdA[f] = dA; v.fdp[f] = dp;
   if( v.tr_dim[t] == 1 ){ if( LR == 0 ) v.consL[cL] = f; else v.consR[cR] = f; }
   else                  { if( LR == 0 ) v.consZL[cL] = f; else v.consZR[cR] = f; }

   if( with_slopes ){
      R dxL = (R)v.tr_dxL[t], dxR = (R)v.tr_dxR[t];
      double phiL = pL - .5*dL, phiR = pR - .5*dR;
      R dpL = (R)get_signed_dp(phic, phiL, Pmax, &err);
      R dpR = (R)get_signed_dp(phiR, phic, Pmax, &err);
#pragma unroll
      for( int q=0 ; q<Q ; ++q ){
         R WL = v.prim[q*N + cL] + dpL*v.gradp[q*N + cL];
         R WR = v.prim[q*N + cR] - dpR*v.gradp[q*N + cR];
         v.fS[(size_t)q*v.Nf + f] = (WR-WL)/(dxR+dxL);
      }
   }
   raise_err(v, err);
}
template<int Q, class R>
__global__ void __launch_bounds__(FB, MB_FACES) k_faces(ViewT<R> v, int with_slopes){
   faces_body<Q,R>(v, with_slopes, v.topo_reuse, blockIdx.x);
}

/* The faces of track t in which cell c (k-th edge from I0 of its annulus,
 * cell index i) is the head on its side, in face order: run 1 is
 * [s1, e1]; the I0 cell also heads the faces after the other annulus wraps,
 * run 2 = [s2, e2] (empty when s2 > e2).  cons[] is consL or consR. */
struct Runs { int s1, e1, s2, e2; };
template<class R>
__device__ __forceinline__ Runs cell_runs(const ViewT<R> &v, const int *cons, int t,
                                          int c0, int np, int i, int I0){
   Runs RR;
   int c = c0 + i;
   if( i == I0 ){
      RR.s1 = v.tr_off[t];
      int prev = c0 + (I0 == 0 ? np-1 : I0-1);
      RR.s2 = cons[prev] + 1;
      RR.e2 = v.tr_off[t+1] - 1;
   }else{
      int prev = c0 + (i == 0 ? np-1 : i-1);
      RR.s1 = cons[prev] + 1;
      RR.s2 = 1; RR.e2 = 0;
   }
   RR.e1 = cons[c];
   return RR;
}

/* ------------------------------------------------------------------ k_grad
 * plm_trans (plm.c:56-195) for dim 1 (r) or 2 (z): sum S*dA over the
 * cell's faces in the reference's face order (inner / lower track first,
 * then outer / upper), divide by the cell's two face areas, then apply
 * every face's limiter. */
template<int Q, int DIM, class R>
__device__ __forceinline__ void grad_body(const ViewT<R> &v, int bid){
   int2 b = v.cblk[bid];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const int N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + i;
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   if( DIM == 2 && P.Nz == 1 ) return;
   R *grad = DIM == 1 ? v.gradr : v.gradz;
   int j = v.ann_j[a], k = v.ann_k[a];
   int Nr = P.Nr, Nz = P.Nz;
   int I0 = v.I0[a];
   R g[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) g[q] = R(0.0);
   if( P.PLM == 0.0 ){
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) grad[q*N + c] = R(0.0);
      return;
   }
   int tin, tout;
   const int *cin, *cout;
   if( DIM == 1 ){
      tin = j >= 1 ? P.trr0 + (j-1) + (Nr-1)*k : -1;
      tout = j <= Nr-2 ? P.trr0 + j + (Nr-1)*k : -1;
      cin = v.consR; cout = v.consL;
   }else{
      tin = k >= 1 ? P.trz0 + j + Nr*(k-1) : -1;
      tout = k <= Nz-2 ? P.trz0 + j + Nr*k : -1;
      cin = v.consZR; cout = v.consZL;
   }
   Runs Rin = {1,0,1,0}, Rout = {1,0,1,0};
   if( tin >= 0 ) Rin = cell_runs(v, cin, tin, c0, np, i, I0);
   if( tout >= 0 ) Rout = cell_runs(v, cout, tout, c0, np, i, I0);
   const size_t Nf = v.Nf;
#define ACC_RUN(s,e) for( int f=(s) ; f<=(e) ; ++f ){ R dA = (R)v.fdA[f]; \
      _Pragma("unroll") for( int q=0 ; q<Q ; ++q ) g[q] += v.fS[q*Nf + f]*dA; }
   ACC_RUN(Rin.s1, Rin.e1)
   ACC_RUN(Rin.s2, Rin.e2)
   ACC_RUN(Rout.s1, Rout.e1)
   ACC_RUN(Rout.s2, Rout.e2)
#undef ACC_RUN
   int err = 0;
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   double phip = v.piph[c];
   double phim = phip - v.dphi[c];
   double dph = get_dp(phip, phim, P.Pmax, &err);
   double dAp, dAm;
   if( DIM == 1 ){
      double dz = zk[k]-zk[k-1];
      dAp = (.5*(rj[j]+rj[j]))*dph*dz;
      dAm = (.5*(rj[j-1]+rj[j-1]))*dph*dz;
   }else{
      double r = .5*(rj[j]+rj[j-1]), dr = rj[j]-rj[j-1];
      dAp = r*dr*dph;
      dAm = r*dr*dph;
   }
   double dAtot = dAp + dAm;
   if( (DIM == 1 && j == 0) || (DIM == 2 && k == 0) ) dAtot = dAp;
   if( (DIM == 1 && j == Nr-1) || (DIM == 2 && k == Nz-1) ) dAtot = dAm;
   const R rdAtot = (R)dAtot;
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) g[q] /= rdAtot;
   const R PLM = (R)P.PLM;
#define LIM_RUN(s,e) for( int f=(s) ; f<=(e) ; ++f ){ \
      _Pragma("unroll") for( int q=0 ; q<Q ; ++q ){ R S = v.fS[q*Nf + f]; \
         if( S*g[q] < R(0.0) ) g[q] = R(0.0); else if( fabs(PLM*S) < fabs(g[q]) ) g[q] = PLM*S; } }
   LIM_RUN(Rin.s1, Rin.e1)
   LIM_RUN(Rin.s2, Rin.e2)
   LIM_RUN(Rout.s1, Rout.e1)
   LIM_RUN(Rout.s2, Rout.e2)
#undef LIM_RUN
   /* plm_geom_boundary at the axis (plm.c:184-185 -> geom_grad,
    * cylindrical.c:141-173): with no ghosts inside (NgRa 0) and the inner
    * edge at r = 0, the first annulus keeps only its v_r (and B_r) slope,
    * limited against prim/r at the centroid; the other slopes are zero.
    * (At an outer or z edge without ghosts geom_grad changes nothing.) */
   if( DIM == 1 && j == 0 && P.NgRa == 0 ){
      double xp0 = rj[0], xm0 = rj[-1];
      if( !(xp0 < 0.0 || fabs(xm0) > 1.0e-10*xp0) ){
         double r = centroid_r(xp0, xm0);
#pragma unroll
         for( int q=0 ; q<Q ; ++q ){
            if( q == URR || (Q > 6 && q == BRR) ){
               double SL = (double)v.prim[q*N + c]/r;
               double S = (double)g[q];
               if( S*SL < 0.0 ) g[q] = R(0.0);
               else if( fabs(P.PLM*SL) < fabs(S) ) g[q] = (R)(P.PLM*SL);
            }else{
               g[q] = R(0.0);
            }
         }
      }
   }
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) grad[q*N + c] = g[q];
   raise_err(v, err);
}
template<int Q, int DIM, class R>
__global__ void __launch_bounds__(CB, Q > 6 ? MB_MHD_GRAD : MB_GRAD) k_grad(ViewT<R> v){
   grad_body<Q,DIM,R>(v, blockIdx.x);
}
/* both directions of a 3D grid in one launch: the cell's annulus data are
 * read once and the two gathers' loads overlap */
template<int Q, class R>
__global__ void __launch_bounds__(CB, Q > 6 ? MB_MHD_GRAD : MB_GRAD) k_grad_rz(ViewT<R> v){
   grad_body<Q,1,R>(v, blockIdx.x);
   grad_body<Q,2,R>(v, blockIdx.x);
}

/* The viscous flux of a face, compiled only into the viscous instances of
 * k_flux_t / k_update (template VISC) so that the inviscid kernels keep
 * their registers.  trans_visc_flux: riemann_trans's
 * averaged state and gradients (riemann.c:127-131, 158-167, 295-309), the
 * face's own difference slope in the face's direction; phi_visc_flux:
 * riemann_phi's (riemann.c:45-64). */
template<int Q, int DIM, class R>
__device__ __forceinline__ void trans_visc_flux(const ViewT<R> &v, const DiskParams &P, int cL, int cR,
                                             R dpL, R dpR, R dxL, R dxR, const R *primL,
                                             const R *primR, double r, double om, double *vF){
   const int N = v.Ncell;
   double pa[Q], gr[Q], gp[Q], gz[Q];
   for( int q=0 ; q<Q ; ++q ){
      double g = (((double)v.prim[q*N+cR] - (double)v.gradp[q*N+cR]*(double)dpR)
                  - ((double)v.prim[q*N+cL] + (double)v.gradp[q*N+cL]*(double)dpL))
                 / ((double)dxL + (double)dxR);
      double zL = v.gradz ? (double)v.gradz[q*N+cL] : 0.0;
      double zR = v.gradz ? (double)v.gradz[q*N+cR] : 0.0;
      pa[q] = .5*((double)primL[q] + (double)primR[q]);
      gp[q] = .5*((double)v.gradp[q*N+cL] + (double)v.gradp[q*N+cR]);
      if( DIM == 1 ){ gr[q] = .5*(g + g); gz[q] = .5*(zL + zR); }
      else { gr[q] = .5*((double)v.gradr[q*N+cL] + (double)v.gradr[q*N+cR]); gz[q] = .5*(g + g); }
   }
   const double n[3] = {DIM == 1 ? 1.0 : 0.0, 0.0, DIM == 2 ? 1.0 : 0.0};
   visc_flux<Q>(P, pa, gr, gp, gz, r, om, n, vF);
}
template<int Q, class R>
__device__ __forceinline__ void phi_visc_flux(const ViewT<R> &v, const DiskParams &P, int cL, int cR,
                                           const R *primL, const R *primR, double r, double om,
                                           double *vF){
   const int N = v.Ncell;
   double pa[Q], gr[Q], gp[Q], gz[Q];
   double dh = 0.5*(v.dphi[cR] + v.dphi[cL]);
   for( int q=0 ; q<Q ; ++q ){
      double g = ((double)v.prim[q*N+cR] - (double)v.prim[q*N+cL]) / dh;
      pa[q] = .5*((double)primL[q] + (double)primR[q]);
      gr[q] = .5*((double)v.gradr[q*N+cL] + (double)v.gradr[q*N+cR]);
      gp[q] = .5*(g + g);
      gz[q] = v.gradz ? .5*((double)v.gradz[q*N+cL] + (double)v.gradz[q*N+cR]) : 0.0;
   }
   const double n[3] = {0.0, 1.0, 0.0};
   visc_flux<Q>(P, pa, gr, gp, gz, r, om, n, vF);
}
/* riemann_trans's solve with the viscous flux */
template<int Q, int NC, int DIM, class R>
__device__ __forceinline__ void trans_face_flux_visc(const ViewT<R> &v, const DiskParams &P, int cL,
                                                  int cR, R dpL, R dpR, R dxL, R dxR,
                                                  const R *primL, const R *primR, double r,
                                                  double om, double dAdt, R *G){
   double vF[Q];
   trans_visc_flux<Q,DIM,R>(v, P, cL, cR, dpL, dpR, dxL, dxR, primL, primR, r, om, vF);
   solve_riemann<Q,NC,DIM,R>(P, primL, primR, (R)r, (R)om, R(0.0), (R)dAdt, G, nullptr, vF);
}
/* visc_source (euler.c:261-295) for cell c: the increments of cons[SRR]
 * and cons[TAU] */
template<int Q, class R>
__device__ __forceinline__ double2 visc_source_cell(const ViewT<R> &v, const DiskParams &P, int c,
                                                 int a, double r, double dVdt){
   const int N = v.Ncell;
   double gr[Q], gp[Q], gz[Q], prim[Q];
   for( int q=0 ; q<Q ; ++q ) prim[q] = (double)v.prim[q*N + c];
   for( int q=0 ; q<Q ; ++q ){
      gr[q] = (double)v.gradr[q*N + c];
      gp[q] = (double)v.gradp[q*N + c];
      gz[q] = v.gradz ? (double)v.gradz[q*N + c] : 0.0;
   }
   double nu = visc_nu(P, prim, r);
   double rho = prim[RHO], vr = prim[URR];
   double divV_o_d = (gr[URR] + gp[UPP] + gz[UZZ] + vr/r) / 3.0;
   double spp = (r*gp[UPP] + vr - r*divV_o_d) / (r*r*r);
   double dS = (-2 * r * rho * nu * spp) * dVdt;
   double srp = 0.5*(r*r*gr[UPP] + gp[URR]);
   double spz = 0.5*(gp[UZZ] + r*r*gz[UPP]);
   double om_r = v.ann_om1[a], om_z = 0.0;
   double dT = (2 * rho * nu * (srp * om_r + spz * om_z)) * dVdt;
   return make_double2(dS, dT);
}

/* ------------------------------------------------------------------ k_flux_t
 * trans_flux (misc.c:431-509) -> riemann_trans (riemann.c:114-170) ->
 * solve_riemann for the faces of r-tracks (DIM 1) or z-tracks (DIM 2);
 * G_q = (F - w U*) dA dt per face.  The face centre cm is (r_{j+1/2}, phic,
 * z centroid) for r-faces and (r centroid, phic, z_{k+1/2}) for z-faces
 * (addFace, faces_alt.c:10-16). */
template<int Q, int NC, int DIM, class R, bool VISC = false, bool GR = false>
__device__ __forceinline__ void flux_body(const ViewT<R> &v, double dtfac, int bid){
   int2 b = v.fblk[bid];
   int t = b.x;
   if( v.tr_dim[t] != DIM || !v.tr_flux[t] ) return;
   int dd = b.y + threadIdx.x;
   int f = v.tr_off[t] + dd;
   if( f >= v.tr_off[t+1] ) return;
   const int N = v.Ncell;
   int cL = v.fL[f], cR = v.fR[f];
   int d = v.ann_disk[v.tr_a[t]];
   const DiskParams &P = v.dp[d];
   int err = 0;
   double dt = v.ds[d].dt*dtfac;
   double dAdt = v.fdA[f]*dt;
   R dxL = (R)v.tr_dxL[t], dxR = (R)v.tr_dxR[t];
   double phi = v.fphic[f];
   double phiL = v.piph[cL] - .5*v.dphi[cL];
   double phiR = v.piph[cR] - .5*v.dphi[cR];
   R dpL = (R)get_signed_dp(phi, phiL, P.Pmax, &err);
   R dpR = (R)get_signed_dp(phiR, phi, P.Pmax, &err);
   const R *grad = DIM == 1 ? v.gradr : v.gradz;
   R primL[Q], primR[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){
      primL[q] = v.prim[q*N+cL] + grad[q*N+cL]*dxL + v.gradp[q*N+cL]*dpL;
      primR[q] = v.prim[q*N+cR] - grad[q*N+cR]*dxR - v.gradp[q*N+cR]*dpR;
   }
   if constexpr ( NC == 8 ){                     /* normal B averaged, riemann.c:146-152 */
      const int BT = DIM == 1 ? BRR : BZZ;
      R Bavg = R(.5)*(primL[BT]+primR[BT]);
      primL[BT] = Bavg; primR[BT] = Bavg;
   }
   /* face cm[0]: .5 (r_j + r_j) on an r track, the annulus centroid on a z
    * track (the same for every face of the track, tabulated at set-up) */
   const double r = v.tr_r[t];
   R G[Q];
   if constexpr ( GR ){              /* grmhd2 + HLL at the face centre (addFace, faces_alt.c:10-16) */
      const double *zk = v.zk + P.zk0 + 1;
      int k = v.tr_k[t];
      double x[3] = {r, phi, DIM == 1 ? 0.5*(zk[k]+zk[k-1]) : 0.5*(zk[k]+zk[k])};
      const double n[3] = {DIM == 1 ? 1.0 : 0.0, 0.0, DIM == 2 ? 1.0 : 0.0};
      double pl[Q], pr[Q], g[Q];
#pragma unroll
      for( int q=0 ; q<Q ; ++q ){ pl[q] = (double)primL[q]; pr[q] = (double)primR[q]; }
      gr_hll(P, v.gr_tr[t], pl, pr, x, n, 0.0, dAdt, g);
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) G[q] = (R)g[q];
   }else if constexpr ( NC == 8 ){
      if( v.ct ){                    /* flux_to_E dim 1 / 2, Hydro/mhd.c:304-314 */
         R eb[5];
         solve_riemann<Q,NC,DIM,R>(P, primL, primR, (R)r, (R)v.tr_om[t], R(0.0), (R)dAdt, G, eb);
         const R rr = (R)r;
         const R irfac = (R)v.tr_irf[t];                /* 1/(1/r) */
         if( DIM == 1 ){
            v.fEt[f] = -eb[1]*rr;
            v.fBt[f] = eb[2]*irfac;
            if( v.ct == 2 ) v.fEphi[f] = eb[3];
         }else{
            v.fEt[f] = eb[1]*rr;
            v.fBt[f] = eb[4];
            v.fEphi[f] = -eb[0]*irfac;
         }
      }else{
         solve_riemann<Q,NC,DIM,R>(P, primL, primR, (R)r, (R)v.tr_om[t], R(0.0), (R)dAdt, G);
      }
   }else{
      bool visc = false;
      if constexpr ( VISC ) visc = P.visc;
      if( visc ){                    /* riemann_trans (riemann.c:127-131, 158-167) + visc */
         trans_face_flux_visc<Q,NC,DIM,R>(v, P, cL, cR, dpL, dpR, dxL, dxR, primL, primR, r,
                                          v.tr_om[t], dAdt, G);
      }else{
         solve_riemann<Q,NC,DIM,R>(P, primL, primR, (R)r, (R)v.tr_om[t], R(0.0), (R)dAdt, G);
      }
   }
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) v.fG[(size_t)q*v.Nf + f] = G[q];
   raise_err(v, err);
}
template<int Q, int NC, int DIM, class R, bool VISC = false, bool GR = false>
__global__ void __launch_bounds__(FB, GR ? MB_GR : (Q > 6 ? MB_MHD_FLUX : MB_FLUX)) k_flux_t(ViewT<R> v){
   flux_body<Q,NC,DIM,R,VISC,GR>(v, v.dtfac, blockIdx.x);
}

/* ------------------------------------------------------------------ phi faces
 * phi_flux (misc.c:368-426) -> riemann_phi (riemann.c:39-65): the face
 * between cells cL = i and cR = i+1 of a real annulus a, G_q = (F - w U*)
 * dA dt, with x = (annulus centroid r, phi, centroid z), dA = dr dz,
 * w = r wiph[cL]. */
template<int Q, int NC, class R>
__device__ __forceinline__ void phi_face_flux(const ViewT<R> &v, const DiskParams &P, int a,
                                              int cL, int cR, double r, double dAdt, R *G,
                                              R *eb = nullptr){
   const int N = v.Ncell;
   R primL[Q], primR[Q];
   R dL = (R)v.dphi[cL], dR = (R)v.dphi[cR];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ){
      primL[q] = v.prim[q*N+cL] + R(.5)*v.gradp[q*N+cL]*dL;
      primR[q] = v.prim[q*N+cR] - R(.5)*v.gradp[q*N+cR]*dR;
   }
   if constexpr ( NC == 8 ){                     /* B_phi averaged, riemann.c:54-58 */
      R Bp = R(.5)*(primL[BPP]+primR[BPP]);
      primL[BPP] = Bp; primR[BPP] = Bp;
   }
   double w = r*v.wiph[cL];
   solve_riemann<Q,NC,0,R>(P, primL, primR, (R)r, (R)v.ann_om[a], (R)w, (R)dAdt, G, eb);
}

/* the same from the two edge states already extrapolated (primL: cell cL's
 * right edge, primR: the next cell's left edge); primR is overwritten */
template<int Q, int NC, class R>
__device__ __forceinline__ void phi_face_flux_states(const ViewT<R> &v, const DiskParams &P, int a,
                                                     int cL, double r, double dAdt, const R *eL,
                                                     R *primR, R *G, R *eb = nullptr){
   R primL[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) primL[q] = eL[q];
   if constexpr ( NC == 8 ){                     /* B_phi averaged, riemann.c:54-58 */
      R Bp = R(.5)*(primL[BPP]+primR[BPP]);
      primL[BPP] = Bp; primR[BPP] = Bp;
   }
   double w = r*v.wiph[cL];
   solve_riemann<Q,NC,0,R>(P, primL, primR, (R)r, (R)v.ann_om[a], (R)w, (R)dAdt, G, eb);
}

/* Q values passed to and from the out-of-line viscous paths by value, so
 * that no array of the calling kernel has its address taken */
template<int Q, class R> struct QVec { R q[Q]; };

/* The phi face with the viscous flux (riemann_phi, riemann.c:45-64, +
 * visc_flux), in the viscous instance of k_update only.  The edge states
 * are extrapolated again here exactly as k_update does (cL's right edge,
 * cR's left edge). */
template<int Q, int NC, class R>
__device__ __forceinline__ QVec<Q,R> phi_face_flux_visc(const ViewT<R> &v, const DiskParams &P, int a,
                                                     int cL, int cR, double r, double dAdt){
   const int N = v.Ncell;
   R primL[Q], primR[Q];
   R dL = (R)v.dphi[cL], dR = (R)v.dphi[cR];
   for( int q=0 ; q<Q ; ++q ){
      primL[q] = v.prim[q*N + cL] + R(.5)*v.gradp[q*N + cL]*dL;
      primR[q] = v.prim[q*N + cR] - R(.5)*v.gradp[q*N + cR]*dR;
   }
   double w = r*v.wiph[cL];
   double vF[Q];
   phi_visc_flux<Q,R>(v, P, cL, cR, primL, primR, r, v.ann_om[a], vF);
   QVec<Q,R> G;
   solve_riemann<Q,NC,0,R>(P, primL, primR, (R)r, (R)v.ann_om[a], (R)w, (R)dAdt, G.q, nullptr, vF);
   return G;
}

/* ------------------------------------------------------------------ k_update
 * The flux gather and sources, per cell, in the reference's order:
 *   flux gather  riemann.c:312-315 applied as phi_flux then trans_flux do
 *   add_source   misc.c:538-580 (euler source + planet_src), pre-move cell,
 *                FP64 in both forms (the disk's force balance)
 * The move of the first substep (move_cells / clean_pi / calc_dp,
 * misc.c:256-288, to piph_new from k_begin) follows in k_c2p: the phi-face
 * states here read the pre-move dphi of the cells next to the chunk, which
 * another block owns, so no block of this kernel may move a cell.
 * calc_prim, the boundary, and the fused getmindt / diagnostics follow in
 * k_c2p (run inside this kernel instead, the extra registers cost more than
 * the saved re-read of cons: 1.73 against 1.69 ms per ragged64 step). */
template<int Q, int NC, class R, bool VISC = false, bool GR = false>
__device__ __forceinline__ void update_body(const ViewT<R> &v, int first, double dtfac, int bid){
   /* The block updates CB-1 cells i0 .. i0+CB-2 and its thread t solves the
    * phi face (i0+t-1, i0+t) into sG[.][t]: every thread one face, the
    * chunk's two outer faces included (the left one is also the previous
    * chunk's last). */
   __shared__ R sG[Q][CB];
   __shared__ R sW[Q][CB+1];      /* sW[.][s]: left-edge state of cell i0+s-1 */
   int2 b = v.ublk[bid];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   const int N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + i;
   int cprev = c0 + (i == 0 ? np-1 : i-1);
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   int j = v.ann_j[a], k = v.ann_k[a];
   bool real = j >= P.NgRa && j < P.Nr - P.NgRb && k >= P.NgZa && k < P.Nz - P.NgZb;
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   /* With constrained transport phi_flux also runs on the ghost annuli next
    * to the real ones (misc.c:382-397): their faces' E is needed, their cons
    * updates are not (the ghosts' cons never reach a real cell). */
   bool ctE = false;
   if constexpr ( NC == 8 ){
      if( v.ct ){
         int jmin = P.NgRa == 0 ? 0 : P.NgRa-1, jmax = P.NgRb == 0 ? P.Nr : P.Nr-P.NgRb+1;
         int kmin = P.NgZa == 0 ? 0 : P.NgZa-1, kmax = P.NgZb == 0 ? P.Nz : P.Nz-P.NgZb+1;
         ctE = j >= jmin && j < jmax && k >= kmin && k < kmax;
      }
   }
   if( real || ctE ){               /* uniform over the block: one annulus */
      double dA = (rj[j]-rj[j-1])*(zk[k]-zk[k-1]);       /* get_dA(.,.,0) */
      double dAdtp = dA*(v.ds[d].dt*dtfac);
      double rc = v.ann_rc[a];                          /* centroid_r(r_j, r_j-1) */
      /* riemann_phi's edge states (riemann.c:45-50): thread t extrapolates
       * cell i-1 to both of its phi edges; the left-edge state goes to its
       * neighbour through shared memory (the last thread also does cell i) */
      R eR[Q];
      const int tt = threadIdx.x;
      auto edges = [&](int cell, R *right, int slot){
         R dph = (R)v.dphi[cell];
#pragma unroll
         for( int q=0 ; q<Q ; ++q ){
            R pq = v.prim[q*N + cell], gq = v.gradp[q*N + cell];
            if( right ) right[q] = pq + R(.5)*gq*dph;
            sW[q][slot] = pq - R(.5)*gq*dph;
         }
      };
      /* slot s holds cell i0+s-1 (periodic); slots 0 .. smax are read */
      const int i0 = b.y;
      const int smax = (np - i0 < CB-1 ? np - i0 : CB-1) + 1;
      auto cell_of = [&](int sl){
         int x = i0 + sl - 1;
         if( x < 0 ) x += np; else if( x >= np ) x -= np;
         return c0 + x;
      };
      if( tt <= smax ) edges(cell_of(tt), eR, tt);
      if( tt == CB-1 && CB <= smax ) edges(cell_of(CB), nullptr, CB);
      __syncthreads();
      if( i <= np ){                 /* face (i-1, i): left cell cprev, right cell c (mod np) */
         R G[Q];
         R primR[Q];
#pragma unroll
         for( int q=0 ; q<Q ; ++q ) primR[q] = sW[q][tt+1];
         if constexpr ( GR ){      /* riemann_phi with grmhd2 + HLL, x = (r, piph, z) */
            double pl[Q], pr[Q], g[Q];
#pragma unroll
            for( int q=0 ; q<Q ; ++q ){ pl[q] = (double)eR[q]; pr[q] = (double)primR[q]; }
            double Bp = .5*(pl[BPP]+pr[BPP]);                 /* riemann.c:54-58 */
            pl[BPP] = Bp; pr[BPP] = Bp;
            double x[3] = {rc, v.piph[cprev], centroid_z(zk[k], zk[k-1])};
            const double n[3] = {0.0, 1.0, 0.0};
            gr_hll(P, v.gr_ann[a].c, pl, pr, x, n, rc*v.wiph[cprev], dAdtp, g);
#pragma unroll
            for( int q=0 ; q<Q ; ++q ) G[q] = (R)g[q];
         }else if( ctE ){           /* flux_to_E dim 0, Hydro/mhd.c:298-303 */
            R eb[5];
            phi_face_flux_states<Q,NC,R>(v, P, a, cprev, rc, dAdtp, eR, primR, G, eb);
            if( threadIdx.x > 0 ){  /* stored once: t = 0's face is the previous chunk's */
               const R irfac = (R)(1.0/(1.0/rc));
               v.pE[cprev] = eb[0]*irfac;
               v.pB[cprev] = eb[2]*irfac;
               if( v.ct == 2 ){ v.pEr[cprev] = -eb[3]; v.pBz[cprev] = eb[4]; }
            }
         }else{
            bool visc = false;
            if constexpr ( VISC ) visc = P.visc;
            if( visc ){
               QVec<Q,R> Gv = phi_face_flux_visc<Q,NC,R>(v, P, a, cprev, c0 + (i == np ? 0 : i),
                                                         rc, dAdtp);
#pragma unroll
               for( int q=0 ; q<Q ; ++q ) G[q] = Gv.q[q];
            }else{
               phi_face_flux_states<Q,NC,R>(v, P, a, cprev, rc, dAdtp, eR, primR, G);
            }
         }
#pragma unroll
         for( int q=0 ; q<Q ; ++q ) sG[q][threadIdx.x] = G[q];
      }
      __syncthreads();
   }
   if( threadIdx.x == CB-1 || i >= np ) return;
   int err = 0;
   double piph = v.piph[c], dphi = v.dphi[c];
   if( real ){
      const DiskState &S = v.ds[d];
      double dt = S.dt*dtfac;
      double cons[Q], cc[Q];
#pragma unroll
      for( int q=0 ; q<Q ; ++q ){
         cons[q] = v.cons[q*N + c];
         if constexpr ( sizeof(R) != sizeof(double) ) cc[q] = (double)v.ccarry[q*N + c];
         else cc[q] = 0.0;
      }
      /* The face fluxes: in the FP64 path added to cons one by one in the
       * reference's order; in the mixed form (FP32 fluxes) summed in a plain
       * FP64 accumulator, exact for a handful of FP32 values whose exponents
       * lie within 29 binades, then added to cons once, compensated. */
      double fs[Q];
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) fs[q] = 0.0;
      auto addf = [&](int q, double x){
         if constexpr ( sizeof(R) == sizeof(double) ) cons[q] += x;
         else fs[q] += x;
      };
      /* phi faces: loop order of phi_flux */
      const int t = threadIdx.x;
      if( i > 0 ){
#pragma unroll
         for( int q=0 ; q<Q ; ++q ){
            addf(q, (double)sG[q][t]);
            addf(q, -(double)sG[q][t+1]);
         }
      }else{
#pragma unroll
         for( int q=0 ; q<Q ; ++q ){
            addf(q, -(double)sG[q][t+1]);
            addf(q, (double)sG[q][t]);
         }
      }
      /* r faces: inner track (cell is R) then outer track (cell is L) */
      int I0 = v.I0[a];
      /* a real annulus at the axis (NoBC_Rmin, j = 0) has no inner track, one
       * at an outer edge without ghosts (NoBC_Rmax, j = Nr-1) no outer one */
      Runs Rin = {1,0,1,0}, Rout = {1,0,1,0};
      if( j >= 1 ) Rin = cell_runs(v, v.consR, P.trr0 + (j-1) + (P.Nr-1)*k, c0, np, i, I0);
      if( j <= P.Nr-2 ) Rout = cell_runs(v, v.consL, P.trr0 + j + (P.Nr-1)*k, c0, np, i, I0);
      const size_t Nf = v.Nf;
#define ADD_RUN(s,e,sg) for( int f=(s) ; f<=(e) ; ++f ){ \
      _Pragma("unroll") for( int q=0 ; q<Q ; ++q ) addf(q, sg (double)v.fG[q*Nf + f]); }
      ADD_RUN(Rin.s1, Rin.e1, +)
      ADD_RUN(Rin.s2, Rin.e2, +)
      ADD_RUN(Rout.s1, Rout.e1, -)
      ADD_RUN(Rout.s2, Rout.e2, -)
      /* z faces (trans_flux dim 2): lower track (cell is R) then upper */
      if( P.Nz > 1 ){
         if( k >= 1 ){
            Runs Zin = cell_runs(v, v.consZR, P.trz0 + j + P.Nr*(k-1), c0, np, i, I0);
            ADD_RUN(Zin.s1, Zin.e1, +)
            ADD_RUN(Zin.s2, Zin.e2, +)
         }
         if( k <= P.Nz-2 ){
            Runs Zout = cell_runs(v, v.consZL, P.trz0 + j + P.Nr*k, c0, np, i, I0);
            ADD_RUN(Zout.s1, Zout.e1, -)
            ADD_RUN(Zout.s2, Zout.e2, -)
         }
      }
#undef ADD_RUN
      if constexpr ( sizeof(R) != sizeof(double) ){
#pragma unroll
         for( int q=0 ; q<Q ; ++q ) acc<R>(cons[q], cc[q], fs[q]);
      }
      /* add_source with the pre-move cell */
      double prim[Q];
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) prim[q] = (double)v.prim[q*N + c];
      double rp = rj[j], rm = rj[j-1], zp = zk[k], zm = zk[k-1];
      double phim = piph - dphi;
      double dph = get_dp(piph, phim, P.Pmax, &err);
      double dV = dV_of(rp, rm, dph, zp, zm);
      double dVdt = dV*dt;
      double r = v.ann_rc[a];                            /* centroid_r(rp, rm) */
      if constexpr ( GR ){       /* grmhd2 source, grmhd2.c:383-478 */
         gr_source(P, v.gr_ann[a], prim, cons, 0.5*(rm+rp), dVdt);
      }else if constexpr ( NC == 8 ){  /* mhd source, mhd.c:225-263 */
         double rho = prim[RHO], Pp = prim[PPP];
         double r_1 = .5*(rp+rm);
         double r2_3 = (rp*rp + rp*rm + rm*rm)/3.;
         double vr = prim[URR], omega = prim[UPP];
         double Br = prim[BRR], Bp = prim[BPP], Bz = prim[BZZ];
         double B2 = Br*Br+Bp*Bp+Bz*Bz;
         double centrifugal;
         if( P.polar ){
            centrifugal = ( rho*omega*omega*r2_3 )/r_1*sin(.5*dph)/(.5*dph);
            centrifugal -= Bp*Bp/r_1;
         }else{
            centrifugal = rho*omega*omega*r - Bp*Bp/r;
         }
         double press_bal = (Pp+.5*B2)/r_1;
         acc<R>(cons[SRR], cc[SRR], dVdt*( centrifugal + press_bal ));
         double om = v.ann_om[a];
         double om1 = v.ann_om1[a];
         acc<R>(cons[TAU], cc[TAU], dVdt*rho*vr*( om*om*r2_3/r_1 - om1*(omega-om)*r2_3 ));
      }else{  /* euler source, euler.c:171-215 */
         double rho = prim[RHO], Pp = prim[PPP];
         double r_1 = .5*(rp+rm);
         double vr = prim[URR], omega = prim[UPP], vz = prim[UZZ];
         double centrifugal = rho*omega*omega*r;
         if( P.polar ) centrifugal *= sin(0.5*dph) / (0.5*dph);
         double press_bal = Pp/r_1;
         acc<R>(cons[SRR], cc[SRR], dVdt*( centrifugal + press_bal ));
         double om = v.ann_om[a];
         double om_r = v.ann_om1[a];
         double om_z = 0.0;
         acc<R>(cons[TAU], cc[TAU], dVdt*rho*( r*vr*om*om - r*r*(omega-om)*(vr*om_r + vz*om_z)));
      }
      double sphi = 0.0, cphi = 1.0;
      if( P.npl > 0 ) sincos(phim + 0.5*dph, &sphi, &cphi);   /* the cell's phi, all planets */
      for( int p=0 ; p<P.npl ; ++p ){   /* planet_src, planet.c:152-196 */
         double rho = prim[RHO], vr = prim[URR], vz = prim[UZZ], omega = prim[UPP];
         double x2 = centroid_z(zp, zm);
         double F0, F1, F2;
         planetary_force_sc(P.grav2D, S.pl[p], r, sphi, cphi, x2, &F0, &F1, &F2);
         double hr = 1.0, hp = r, hz = 1.0;
         if( P.polar ){ double adj = sin(0.5*dph)/(0.5*dph); F0 *= adj; F1 *= adj; }
         acc<R>(cons[SRR], cc[SRR], rho*hr*F0*dVdt);
         acc<R>(cons[LLL], cc[LLL], rho*hp*F1*dVdt);
         acc<R>(cons[SZZ], cc[SZZ], rho*hz*F2*dVdt);
         acc<R>(cons[TAU], cc[TAU], rho*( hr*F0*vr + hz*F2*vz + hp*F1*omega )*dVdt);
      }
      if constexpr ( NC == 5 && VISC ){
         if( P.visc ){                  /* visc_source, euler.c:261-295 */
            double2 st = visc_source_cell<Q,R>(v, P, c, a, r, dVdt);
            acc<R>(cons[SRR], cc[SRR], st.x);
            acc<R>(cons[TAU], cc[TAU], st.y);
         }
      }
#pragma unroll
      for( int q=0 ; q<Q ; ++q ){
         v.cons[q*N + c] = cons[q];
         if constexpr ( sizeof(R) != sizeof(double) ) v.ccarry[q*N + c] = (float)cc[q];
      }
   }
   (void)first;                     /* the move follows in k_c2p (or k_ct_update) */
   raise_err(v, err);
}
template<int Q, int NC, class R, bool VISC = false, bool GR = false>
__global__ void __launch_bounds__(CB, GR ? MB_GR : (Q > 6 ? MB_MHD_UPDATE : MB_UPDATE)) k_update(ViewT<R> v, int first){
   update_body<Q,NC,R,VISC,GR>(v, first, v.dtfac, blockIdx.x);
}

/* One cell's terms of add_diagnostics (analysis.c:52-107) with the
 * diag_disk2d quantities (Diagnostics/diag_disk2d.c:17-38), times dV, and
 * dV itself: every cell of the annulus, ghosts included, at the midpoint xc. */
template<int NQD>
__device__ __forceinline__ void diag_cell(const DiskParams &P, const DiskState &S,
                                          const double *prim,
                                          double rp, double rm, double zp, double zm,
                                          double piph, double phim, double *dq, int *err){
   double dph = get_dp(piph, phim, P.Pmax, err);
   double dV = dV_of(rp, rm, dph, zp, zm);
   double r = .5*(rp+rm), phi = .5*(piph+phim);
   double rho = prim[RHO], vr = prim[URR], omega = prim[UPP];
   double Fp = 0.0;
   if constexpr ( NQD == 5 ){         /* Diagnostics/diag_disk2d.c:17-40 */
      if( P.npl > 1 ){
         double Fr, Fz;
         planetary_force(P.grav2D, S.pl[1], r, phi, 0.0, &Fr, &Fp, &Fz);
      }
      dq[0] = rho*dV;
      dq[1] = 2.*DISCO_PI*r*rho*vr*dV;
      dq[2] = 2.*DISCO_PI*r*rho*(r*Fp)*dV;
      dq[3] = 2.*DISCO_PI*r*rho*( r*r*omega*vr )*dV;
      dq[4] = omega*dV;
   }else if constexpr ( NQD == 18 ){  /* Diagnostics/diag_mhdmri.c:17-59 */
      double Pp = prim[PPP], vp = prim[UPP], vz = prim[UZZ];
      double Br = prim[BRR], Bp = prim[BPP], Bz = prim[BZZ];
      double gam = P.gam;
      double cs2 = gam * Pp / rho;
      double B2 = Br*Br + Bp*Bp + Bz*Bz;
      double sr = rho*vr;
      double sp = r*r*rho*vp;
      double sz = rho*vz;
      double e = 0.5*rho*(vr*vr + r*r*vp*vp + vz*vz) + Pp/(gam-1.0) + 0.5*B2;
      const double qv[18] = {rho, Pp, vr, vp, vz, Br, Bp, Bz, rho, e, sr, sp, sz, rho*vr*vp,
                             Br*Bp, B2, sqrt(cs2), sqrt(B2/rho)};
#pragma unroll
      for( int m=0 ; m<18 ; ++m ) dq[m] = qv[m]*dV;
      (void)omega; (void)phi; (void)Fp;
   }else{                             /* Diagnostics/diag_euler.c:17-45 */
      double z = .5*(zp+zm);
      double vz = prim[UZZ], Pp = prim[PPP];
      if( P.npl > 1 ){
         double Fr, Fz;
         planetary_force(P.grav2D, S.pl[1], r, phi, z, &Fr, &Fp, &Fz);
      }
      dq[0] = rho*dV;
      dq[1] = 2.*DISCO_PI*r*rho*vr*dV;
      dq[2] = 2.*DISCO_PI*r*rho*vz*dV;
      dq[3] = 2.*DISCO_PI*r*rho*(r*Fp)*dV;
      dq[4] = 2.*DISCO_PI*r*rho*( r*r*omega*vr )*dV;
      dq[5] = omega*dV;
      dq[6] = 2*DISCO_PI*r * rho*r*r*omega*dV;
      dq[7] = Pp*dV;
   }
   dq[NQD] = dV;
}

/* the global slot of local diagnostic m (the volume goes to DIAG_VOL) */
template<int NQD>
__device__ __forceinline__ int diag_slot(int m){ return m == NQD ? DIAG_VOL : m; }

/* The per-block diagnostic sums as a pass of their own, for boundaries that
 * change ghost prims after calc_prim (zerograd): add_diagnostics sees the
 * state after the last boundary pass (timestep.c:40-42). */
template<int Q, class R, int NQD>
__global__ void __launch_bounds__(CB) k_diag_part(ViewT<R> v){
   __shared__ double s_red[CB/32][NQD+1];
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   const int N = v.Ncell;
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   int j = v.ann_j[a], k = v.ann_k[a];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   double dq[NQD+1];
#pragma unroll
   for( int m=0 ; m<=NQD ; ++m ) dq[m] = 0.0;
   int err = 0;
   if( i < np ){
      int c = v.ann_off[a] + i;
      double prim[Q];
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) prim[q] = (double)v.prim[q*N + c];
      double piph = v.piph[c];
      diag_cell<NQD>(P, v.ds[d], prim, rj[j], rj[j-1], zk[k], zk[k-1], piph, piph - v.dphi[c], dq, &err);
   }
   raise_err(v, err);
   int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
   for( int m=0 ; m<=NQD ; ++m ){
      double x = dq[m];
#pragma unroll
      for( int o=16 ; o>0 ; o>>=1 ) x += __shfl_down_sync(0xffffffffu, x, o);
      if( lane == 0 ) s_red[wid][m] = x;
   }
   __syncthreads();
   if( threadIdx.x == 0 ){
      for( int m=0 ; m<=NQD ; ++m ){
         double x = 0.0;
         for( int w=0 ; w<CB/32 ; ++w ) x += s_red[w][m];
         v.diag_part[(size_t)blockIdx.x*DIAG_SLOTS + diag_slot<NQD>(m)] = x;
      }
   }
}

/* The ghost cells a fixed boundary re-initialises from the Initial module,
 * and where it evaluates it:
 *   bc 1  Boundary/fixed.c:11-60: r ghosts (all k) at (midpoint r,
 *         piph - dphi/2, midpoint z)
 *   bc 2  Boundary/fixed3d.c -> boundary_functions.c:20-31, 161-265: r ghosts
 *         (all k) and z ghosts (all j) at the centroid (get_centroid_arr)
 * then subtract_omega (rotframe.c:15-17);
 *   bc 6  Boundary/accrete3d.c: the outer r ghosts and the z ghosts as bc 2
 *         (boundary_fixed_rout / _zbot / _ztop; the inner r ghosts are
 *         zero-gradient, k_zerograd)
 * then subtract_omega (rotframe.c:15-17);
 *   bc 3  Boundary/polar.c: outer r ghosts and z ghosts at the centroid,
 *         without subtract_omega;
 *   bc 8  Boundary/horizon.c:26-67: outer r ghosts and z ghosts at (midpoint r,
 *         piph - dphi/2, midpoint z), without subtract_omega;
 *   bc 9  Boundary/horizon3d.c: outer r ghosts and z ghosts as bc 6
 *         (Boundary/polar3d.c is bc 6 on a grid without inner ghosts);
 * plus, for bc 8 and 9, every annulus inside the excised region
 * (horizon_cut) re-initialised as the module does it.  Returns whether
 * prim was set. */
/* Whether annulus (j, k) lies in a horizon module's excised region: the
 * cells Boundary/horizon.c:70-109 re-initialises and marks not real inside
 * 0.7 * 2M (M = 1 there), or boundary_fixed_horizon's R < R_HOR = 1
 * (boundary_functions.c:622-656, horizon3d).  rj, zk are the disk's edge
 * arrays (index -1 valid). */
__device__ __forceinline__ bool horizon_cut(const DiskParams &P, int bc, int j, int k,
                                            const double *rj, const double *zk){
   if( bc == 8 ){
      const double rh = 2*1.0, cut = 0.7*rh;
      if( !(rj[-1] < cut && zk[-1] < cut && zk[P.Nz-1] > -cut) ) return false;
      double zp = zk[k], zm = zk[k-1];
      double zc = fabs(zp) < fabs(zm) ? zp : zm;
      if( fabs(zc) > cut && P.Nz > 1 ) return false;
      /* the reference walks j outwards and stops at the first annulus
       * outside; the test is monotone in j, so it is this annulus's own */
      double rp = rj[j], rm = rj[j-1];
      double rc = fabs(rp) < fabs(rm) ? rp : rm;
      return !((rc*rc+zc*zc > cut*cut && P.Nz > 1) || rc > cut);
   }
   if( bc == 9 ){
      const double R_HOR = 1.0;
      double zm = zk[k-1], zp = zk[k];
      double zo = fabs(zp) > fabs(zm) ? zp : zm;
      if( fabs(zo) > R_HOR ) return false;
      double ro = rj[j];
      double R = sqrt(zo*zo + ro*ro);
      return R < R_HOR;
   }
   return false;
}
/* Boundary/horizon_bin.c:83-171: cell (j, k) at phi inside one of the two
 * excision spheres of the module's fixed binary (M = 1, separation 10, q = 1:
 * centres at x = 5 and x = -5 in the plane, radius 0.8 r_H of each member),
 * tested in the module's order with its nearest-edge radius rc and z; the
 * per-annulus pre-checks first, then the cell's own distance. */
__device__ __forceinline__ bool horizon_bin_cut(const DiskParams &P, int j, int k, const double *rj,
                                                const double *zk, double phi){
   const double M = 1.0, a = 1.0e1, q = 1.0;
   const double M1 = M/(1+q), M2 = q*M/(1+q);
   const double a1 = q*a/(1+q), a2 = -a/(1+q);
   const double cuts[2] = {0.8*(2*M1), 0.8*(2*M2)};
   const double zp = zk[k], zm = zk[k-1];
   const double zc = fabs(zp) < fabs(zm) ? zp : zm;
   const double rp = rj[j], rm = rj[j-1];
   for( int s=0 ; s<2 ; ++s ){
      const double cut = cuts[s];
      /* the member's centre at x = as; its |x| = xs */
      const double as = s == 0 ? a1 : a2, xs = s == 0 ? a1 : -a2;
      if( !(rj[-1] < xs+cut && rj[P.Nr-1] > xs-cut && zk[-1] < cut && zk[P.Nz-1] > -cut) ) continue;
      if( fabs(zc) > cut && P.Nz > 1 ) continue;
      double rc, dr;
      if( s == 0 ){ rc = fabs(rp-a1) < fabs(rm-a1) ? rp : rm; dr = rc-a1; }
      else        { rc = fabs(rp+a2) < fabs(rm+a2) ? rp : rm; dr = rc+a2; }
      if( (dr*dr+zc*zc > cut*cut && P.Nz > 1) || fabs(dr) > cut ) continue;
      double sn, cs;
      sincos(phi, &sn, &cs);
      const double xc = rc*cs, yc = rc*sn;
      double d2;
      if( P.Nz > 1 ) d2 = (xc-as)*(xc-as) + yc*yc + zc*zc;
      else           d2 = (xc-as)*(xc-as) + yc*yc;
      if( d2 < cut*cut ) return true;
   }
   return false;
}

/* Whether a horizon module re-initialises cell (j, k, phi) and marks it not
 * real: horizon / horizon3d by annulus, horizon_bin by cell. */
__device__ __forceinline__ bool cell_excised(const DiskParams &P, int bc, int j, int k, const double *rj,
                                             const double *zk, double piph, double dphi){
   if( bc == 10 ) return horizon_bin_cut(P, j, k, rj, zk, piph - .5*dphi);
   return (bc == 8 || bc == 9) && horizon_cut(P, bc, j, k, rj, zk);
}

template<int Q, int NC>
__device__ __forceinline__ bool fixed_ghost_init(const DiskParams &P, int bc, int j, int k,
                                                 const double *rj, const double *zk,
                                                 double piph, double dphi, double *prim){
   bool rghost = j < P.NgRa || j >= P.Nr - P.NgRb;
   bool zghost = k < P.NgZa || k >= P.Nz - P.NgZb;
   if( (bc == 8 && (j >= P.Nr - P.NgRb || zghost || horizon_cut(P, bc, j, k, rj, zk))) ||
       (bc == 10 && (j >= P.Nr - P.NgRb || zghost || horizon_bin_cut(P, j, k, rj, zk, piph - .5*dphi))) ){
      double x[3] = { .5*(rj[j]+rj[j-1]), piph - .5*dphi, .5*(zk[k]+zk[k-1]) };
      initial<Q,NC>(P, prim, x);
      return true;
   }
   if( bc == 9 && (j >= P.Nr - P.NgRb || zghost || horizon_cut(P, bc, j, k, rj, zk)) ){
      /* set_cell_init (boundary_functions.c:21-31) */
      double x[3] = { centroid_r(rj[j], rj[j-1]), 0.5*(piph + (piph - dphi)), 0.5*(zk[k]+zk[k-1]) };
      initial<Q,NC>(P, prim, x);
      if( P.rotframe ) prim[UPP] -= P.RotOmega;
      return true;
   }
   if( bc == 1 && rghost ){
      double x[3] = { .5*(rj[j]+rj[j-1]), piph - .5*dphi, .5*(zk[k]+zk[k-1]) };
      initial<Q,NC>(P, prim, x);
   }else if( bc == 2 && (rghost || zghost) ){
      double x[3] = { centroid_r(rj[j], rj[j-1]), 0.5*(piph + (piph - dphi)), 0.5*(zk[k]+zk[k-1]) };
      initial<Q,NC>(P, prim, x);
   }else if( bc == 11 && ((j < P.NgRa && (P.side_fixed & 1)) || (j >= P.Nr - P.NgRb && (P.side_fixed & 2)) ||
                          (k < P.NgZa && (P.side_fixed & 4)) || (k >= P.Nz - P.NgZb && (P.side_fixed & 8))) ){
      /* the fixed sides of fixRrefZ, fixed_gap (boundary_fixed_rinn / _rout /
       * _zbot / _ztop: set_cell_init) */
      double x[3] = { centroid_r(rj[j], rj[j-1]), 0.5*(piph + (piph - dphi)), 0.5*(zk[k]+zk[k-1]) };
      initial<Q,NC>(P, prim, x);
   }else if( bc == 6 && (j >= P.Nr - P.NgRb || zghost) ){
      /* accrete3d: boundary_fixed_rout, _zbot, _ztop (set_cell_init); the
       * inner r ghosts are zero-gradient */
      double x[3] = { centroid_r(rj[j], rj[j-1]), 0.5*(piph + (piph - dphi)), 0.5*(zk[k]+zk[k-1]) };
      initial<Q,NC>(P, prim, x);
   }else if( bc == 3 && (j >= P.Nr - P.NgRb || zghost) ){
      /* Boundary/polar.c:10-77: the outer r ghosts, then every annulus of
       * the z ghost layers, re-evaluated at their centroids (the z pass
       * rewrites the corners with the same values); no subtract_omega */
      double x[3] = { centroid_r(rj[j], rj[j-1]), piph - .5*dphi, centroid_z(zk[k], zk[k-1]) };
      initial<Q,NC>(P, prim, x);
      return true;
   }else{
      return false;
   }
   if( P.rotframe ) prim[UPP] -= P.RotOmega;
   return true;
}

/* B_faces_to_cells type 1 under constrained transport (disco_ct.cuh) */
template<class R>
__device__ void ct_cons_B(const ViewT<R> &v, const DiskParams &P, int a, int c0, int np, int i,
                          int j, int k, double rp, double rm, double zp, double zm, double *cons,
                          int *err);

/* ------------------------------------------------------------------ c2p
 *   move         move_cells / calc_dp (misc.c:256-288) in the first substep
 *                without constrained transport (v.move_c2p; k_c2p)
 *   calc_prim    misc.c:290-325 (cons2prim, FP64) on real cells, from cons
 *   boundary     Boundary/fixed.c:11-60 / fixed3d (ghosts re-initialised)
 * and, on the last substep, the next step's getmindt (misc.c:39-84) and the
 * per-block sums of add_diagnostics (analysis.c:52-107).  Every thread of the
 * block (one annulus chunk) must call it: it ends in block reductions.
 * piph / dphi are the moved cell's; cons is read only on real cells. */
template<int Q, int NC, class R, int NQD, bool VISC, bool GR = false>
__device__ __forceinline__ void c2p_tail(const ViewT<R> &v, const DiskParams &P, int a, int c,
                                         int c0, int np, int i, int j, int k, int d, bool real,
                                         bool active, double piph, double dphi, double *cons,
                                         int last, int bc, int diag, int err, int topo_set,
                                         int bid){
   __shared__ double s_red[CB/32][NQD+1];
   __shared__ unsigned long long s_dt[CB/32];
   const int N = v.Ncell;
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   double prim[Q];
   double dtc = 1.0e300;
   double dq[NQD+1];
#pragma unroll
   for( int m=0 ; m<=NQD ; ++m ) dq[m] = 0.0;
   double rp = rj[j], rm = rj[j-1], zp = zk[k], zm = zk[k-1];
   bool excised = false;
   if( active ){
      double phim = piph - dphi;
      if( real ){
         double dph2 = get_dp(piph, phim, P.Pmax, &err);
         double dV2 = dV_of(rp, rm, dph2, zp, zm);
         if constexpr ( GR ){       /* grmhd2 cons2prim from the cell's current prims */
#pragma unroll
            for( int q=0 ; q<Q ; ++q ) prim[q] = (double)v.prim[q*N + c];
            double x[3] = {centroid_r(rp, rm), 0.5*(phim+piph), centroid_z(zp, zm)};
            if( v.gr_dump ){         /* the solve's inputs, as gr_cons2prim forms them */
               double *o = v.gr_dump + c;
#pragma unroll
               for( int q=0 ; q<Q ; ++q ){ o[(size_t)q*N] = cons[q]/dV2; o[(size_t)(Q+q)*N] = prim[q]; }
#pragma unroll
               for( int m=0 ; m<3 ; ++m ) o[(size_t)(2*Q+m)*N] = x[m];
            }
            gr_cons2prim(P, v.gr_ann[a].c, cons, prim, x, dV2);
         }else{
            cons2prim<Q,NC>(P, cons, prim, v.ann_rc[a], v.ann_om[a], dV2);   /* centroid_r(rp, rm) */
         }
         /* a horizon module then re-initialises the excised annuli (after
          * calc_prim, as boundary_trans follows it) and getmindt skips them */
         if( cell_excised(P, bc, j, k, rj, zk, piph, dphi) ){
            fixed_ghost_init<Q,NC>(P, bc, j, k, rj, zk, piph, dphi, prim);
            excised = true;
            if( v.xflag ) v.xflag[c] = 1;   /* horizon_bin: not real from now on */
         }
         if( v.xflag && v.xflag[c] ) excised = true;
#pragma unroll
         for( int q=0 ; q<Q ; ++q ){
            R pq = (R)prim[q];
            v.prim[q*N + c] = pq;
            prim[q] = (double)pq;       /* the stored state is what the next step sees */
         }
      }else{
         if( fixed_ghost_init<Q,NC>(P, bc, j, k, rj, zk, piph, dphi, prim) ){
#pragma unroll
            for( int q=0 ; q<Q ; ++q ){
               R pq = (R)prim[q];
               v.prim[q*N + c] = pq;
               prim[q] = (double)pq;
            }
         }else if( last ){
#pragma unroll
            for( int q=0 ; q<Q ; ++q ) prim[q] = (double)v.prim[q*N + c];
         }
      }
      if( last ){
         if( real && !excised && GR ){            /* mindt, grmhd2.c:748-832 */
            int cprev = c0 + (i == 0 ? np-1 : i-1);
            double w = .5*(v.wiph[cprev] + v.wiph[c]);
            double xp[3] = {rp, piph, zp}, xm[3] = {rm, phim, zm};
            double dtm = gr_mindt(P, v.gr_ann[a].m, prim, w, xp, xm, &err);
            if( dtm == dtm ) dtc = dtm;
         }else if( real && !excised ){            /* mindt, euler.c:332-380, mhd.c:452-486 */
            int cprev = c0 + (i == 0 ? np-1 : i-1);
            double w = .5*(v.wiph[cprev] + v.wiph[c]);
            double r = v.ann_rc[a];                      /* centroid_r(rp, rm) */
            double vp = (prim[UPP]-w)*r;
            double cs = sqrt(P.gam*prim[PPP]/prim[RHO]);
            if constexpr ( NC == 8 ){
               double b2 = (prim[BRR]*prim[BRR]+prim[BPP]*prim[BPP]+prim[BZZ]*prim[BZZ])/prim[RHO];
               cs = sqrt(cs*cs + b2);
            }
            double maxvr = cs + fabs(prim[URR]);
            double maxvp = cs + fabs(vp);
            double maxvz = cs + fabs(prim[UZZ]);
            double dtr = (rp-rm)/maxvr;
            double dtp = (.5*(rp+rm))*get_dp(piph, phim, P.Pmax, &err)/maxvp;
            double dtz = (zp-zm)/maxvz;
            double dtm = dtr;
            if( dtm > dtp ) dtm = dtp;
            if( dtm > dtz ) dtm = dtz;
            if constexpr ( VISC ){
               if( P.visc ) dtm = visc_dt_limit(P, prim, r, dtm, rp, rm, zp, zm,
                                                get_dp(piph, phim, P.Pmax, &err));
            }
            if( dtm == dtm ) dtc = dtm;
         }
         if( v.nq && diag ) diag_cell<NQD>(P, v.ds[d], prim, rp, rm, zp, zm, piph, phim, dq, &err);
      }
   }
   raise_err(v, err);
   if( topo_set && bid == 0 && threadIdx.x == 0 ) *v.topo = 1;
   if( !last ) return;
   /* block reductions (one annulus per block) */
   int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
   unsigned long long bits = dbits(dtc);
#pragma unroll
   for( int o=16 ; o>0 ; o>>=1 ){
      unsigned long long ob = __shfl_down_sync(0xffffffffu, bits, o);
      bits = ob < bits ? ob : bits;
   }
   if( lane == 0 ) s_dt[wid] = bits;
   if( v.nq && diag ){
#pragma unroll
      for( int m=0 ; m<=NQD ; ++m ){
         double x = dq[m];
#pragma unroll
         for( int o=16 ; o>0 ; o>>=1 ) x += __shfl_down_sync(0xffffffffu, x, o);
         if( lane == 0 ) s_red[wid][m] = x;
      }
   }
   __syncthreads();
   if( threadIdx.x == 0 ){
      unsigned long long mb = s_dt[0];
      for( int w=1 ; w<CB/32 ; ++w ) mb = s_dt[w] < mb ? s_dt[w] : mb;
      if( real ) atomicMin(&v.ds[d].dtmin, mb);
      if( v.nq && diag ){
         for( int m=0 ; m<=NQD ; ++m ){
            double x = 0.0;
            for( int w=0 ; w<CB/32 ; ++w ) x += s_red[w][m];
            v.diag_part[(size_t)bid*DIAG_SLOTS + diag_slot<NQD>(m)] = x;
         }
      }
   }
}

/* ------------------------------------------------------------------ k_c2p
 * c2p_tail on each cell after k_update, with constrained transport first
 * rebuilding B from the face fluxes (onestep.c:183-185). */
template<int Q, int NC, class R, int NQD = 5, bool VISC = false, bool GR = false>
__device__ __forceinline__ void c2p_body(const ViewT<R> &v, int last, int bc, int diag, int move_c2p,
                                         int topo_set, int bid){
   int2 b = v.cblk[bid];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   bool active = i < np;
   const int N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + (active ? i : 0);
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   int j = v.ann_j[a], k = v.ann_k[a];
   bool real = j >= P.NgRa && j < P.Nr - P.NgRb && k >= P.NgZa && k < P.Nz - P.NgZb;
   int err = 0;
   double cons[Q];
   double piph = 0.0, dphi = 0.0;
   if( active ){
      if( move_c2p ){               /* move_cells + calc_dp (misc.c:256-288) */
         piph = v.piph_new[c];
         dphi = get_dp(piph, v.piph_new[c0 + (i == 0 ? np-1 : i-1)], P.Pmax, &err);
         v.piph[c] = piph; v.dphi[c] = dphi;
      }else{
         piph = v.piph[c]; dphi = v.dphi[c];
      }
      if( real ){
#pragma unroll
         for( int q=0 ; q<Q ; ++q ) cons[q] = v.cons[q*N + c];
         if constexpr ( NC == 8 ){
            if( v.ct ){                  /* onestep.c:183-185 */
               const double *rj = v.rj + P.rj0 + 1;
               const double *zk = v.zk + P.zk0 + 1;
               ct_cons_B(v, P, a, c0, np, i, j, k, rj[j], rj[j-1], zk[k], zk[k-1], cons, &err);
               v.cons[BRR*N + c] = cons[BRR];
               v.cons[BPP*N + c] = cons[BPP];
               if( v.ct == 2 && P.Nz > 1 ) v.cons[BZZ*N + c] = cons[BZZ];
            }
         }
      }
   }
   c2p_tail<Q,NC,R,NQD,VISC,GR>(v, P, a, c, c0, np, i, j, k, d, real, active, piph, dphi, cons, last,
                                bc, diag, err, topo_set, bid);
}
/* LAST: 1 for the last substep (the next step's getmindt and the
 * diagnostics), 0 otherwise -- one instantiation each, so that the
 * substeps without the reductions keep fewer registers */
template<int Q, int NC, class R, int NQD = 5, bool VISC = false, bool GR = false, int LAST = 1>
__global__ void __launch_bounds__(CB, GR ? MB_GR_LIGHT : (Q > 6 ? MB_MHD_C2P : MB_C2P)) k_c2p(ViewT<R> v, int bc, int diag){
   c2p_body<Q,NC,R,NQD,VISC,GR>(v, LAST, bc, diag, v.move_c2p, v.topo_set, blockIdx.x);
}

/* The sequential walk of set_cells_copy_distant (boundary_functions.c:
 * 90-158) over ghost cells lo..hi-1 starting at source cell i1: records the
 * start and the number of source cells visited per ghost cell, returns the
 * cell the next ghost cell starts from.  Loops capped (ERRF_WRAP). */
__device__ __forceinline__ int zg_walk(const double *sp, const double *sd, const double *sp1,
                                       const double *sd1, int np1, double Pmax, int lo, int hi,
                                       int i1, int *st, int *cnt, int *err){
   for( int i=lo ; i<hi ; ++i ){
      double phip = sp[i], phim = sp[i] - sd[i];
      double phip1;
      int n = 0;
      st[i] = i1;
      do{
         phip1 = sp1[i1];
         double phim1 = sp1[i1] - sd1[i1];
         int w = 0;
         while( phip1 < phim ){ phip1 += Pmax; phim1 += Pmax; if( ++w > WRAP_CAP ){ *err |= ERRF_WRAP; break; } }
         while( phim1 > phip ){ phip1 -= Pmax; phim1 -= Pmax; if( ++w > WRAP_CAP ){ *err |= ERRF_WRAP; break; } }
         i1 = i1 < np1-1 ? i1+1 : 0;
         if( ++n > np1 + 1 ){ *err |= ERRF_WRAP; break; }
      }while( phip1 < phip );
      cnt[i] = n;
      i1 = i1 > 0 ? i1-1 : np1-1;
   }
   return i1;
}

/* ------------------------------------------------------------------ zerograd
 * boundary_zerograd_{rinn,rout,zbot,ztop} (boundary_functions.c:269-440):
 * a ghost annulus takes the phi-overlap-weighted average of the adjacent
 * annulus (set_cells_copy_distant, :90-158).  One block per (ghost, source)
 * annulus pair of one layer: thread 0 replays the reference's traversal on
 * the two annuli's edges in shared memory and records, per ghost cell, the
 * source cell it starts from and how many it visits; then every thread sums
 * its ghost cell's overlaps in that order and divides by its dphi.  Loops
 * are capped; a cap hit raises ERRF_WRAP.  sides[] names each pair's
 * boundary (0 inner r, 1 outer r, 2 lower z, 3 upper z); with `diode` the
 * copied normal velocity may only point out of the domain (the diode
 * argument of the same functions, used by outflow3d, zerograd_omk and
 * accrete3d), with `omk` the r ghosts then take Omega from the Initial
 * module (boundary_fixed_q_rinn / _rout with q = UPP, :662-718,
 * set_cell_init_q :33-47; zerograd_omk).  Higher bits of sides[]: 4 the
 * diode on this side only, 8 a mirror copy (boundary_reflect_*), 16 no-slip
 * (boundary_noslip_*, :914-1100), 32 a window-only entry with no copy. */
template<int Q, class R>
__global__ void k_zerograd(ViewT<R> v, const int2 *pairs, const unsigned char *sides, int diode,
                           int omk){
   extern __shared__ __align__(16) unsigned char zg_smem[];
   int2 pr = pairs[blockIdx.x];
   const int a = pr.x, a1 = pr.y;
   const int np = v.ann_np[a], np1 = v.ann_np[a1];
   const int c0 = v.ann_off[a], c10 = v.ann_off[a1];
   const DiskParams &P = v.dp[v.ann_disk[a]];
   const double Pmax = P.Pmax;
   if( sides[blockIdx.x] & 32 ){
      /* boundary_fixed_phi_rout(0.3 pi, 1.7 pi) (boundary_functions.c:809-843)
       * on a ghost annulus whose copies are all done (flowthrough.c:10-12):
       * set_cell_init on the cells whose centre lies in the window, no copy */
      const double phia = 0.3*DISCO_PI, phib = 1.7*DISCO_PI;
      const int j = v.ann_j[a], k = v.ann_k[a];
      const double *rj = v.rj + P.rj0 + 1;
      const double *zk = v.zk + P.zk0 + 1;
      const int N = v.Ncell;
      for( int i=threadIdx.x ; i<np ; i+=blockDim.x ){
         const double phip = v.piph[c0+i], dp = v.dphi[c0+i];
         double phi = phip - 0.5*dp;
         for( int w=0 ; phi < phia && w <= WRAP_CAP ; ++w ) phi += Pmax;
         if( phi < phib ){
            double x[3] = { centroid_r(rj[j], rj[j-1]), 0.5*(phip + (phip - dp)), 0.5*(zk[k]+zk[k-1]) };
            double tp[Q];
            initial<Q, (Q > 6 ? 8 : 5)>(P, tp, x);
            if( P.rotframe ) tp[UPP] -= P.RotOmega;
#pragma unroll
            for( int q=0 ; q<Q ; ++q ) v.prim[q*N + c0 + i] = (R)tp[q];
         }
      }
      return;
   }
   double *sp = reinterpret_cast<double*>(zg_smem);          /* ghost piph, dphi */
   double *sd = sp + np;
   double *sp1 = sd + np;                                    /* source piph, dphi */
   double *sd1 = sp1 + np1;
   int *st = reinterpret_cast<int*>(sd1 + np1);              /* start, count */
   int *cnt = st + np;
   __shared__ int s_first;
   for( int i=threadIdx.x ; i<np ; i+=blockDim.x ){ sp[i] = v.piph[c0+i]; sd[i] = v.dphi[c0+i]; }
   for( int i=threadIdx.x ; i<np1 ; i+=blockDim.x ){ sp1[i] = v.piph[c10+i]; sd1[i] = v.dphi[c10+i]; }
   __shared__ int s_rot;
   if( threadIdx.x == 0 ){ s_first = np1; s_rot = 0; }
   __syncthreads();
   /* the source annulus's edges are increasing from its smallest one on
    * (cyclically): that cell's index, for the binary searches below */
   for( int k=threadIdx.x+1 ; k<np1 ; k+=blockDim.x )
      if( sp1[k] < sp1[k-1] ) atomicMax(&s_rot, k);
   {  /* the first source cell (in index order) containing the ghost
       * annulus's first edge: every thread tests its cells, the minimum
       * index wins, as the reference's search loop would stop there */
      int err = 0;
      double phi0 = sp[0] - sd[0];
      for( int k=threadIdx.x ; k<np1 ; k+=blockDim.x ){
         double dphip = get_signed_dp(sp1[k], phi0, Pmax, &err);
         double dphim = dphip - sd1[k];
         if( dphip > 0 && dphim <= 0.0 ){ atomicMin(&s_first, k); break; }
      }
      raise_err(v, err);
   }
   __syncthreads();
   /* The walk of set_cells_copy_distant: ghost cell i starts at source cell
    * st[i] and visits cnt[i] cells; the next starts where it stopped.  Warp 0
    * splits the ghost cells into 32 runs; lane l walks run l from a guess of
    * its start (the source cell holding the upper edge of the cell before
    * the run).  Then each guess is checked against the end of the previous
    * run; from the first wrong guess on, lane 0 walks the rest again, so
    * st/cnt are those of the sequential walk in every case. */
   if( threadIdx.x < 32 ){
      const int lane = threadIdx.x;
      const int seg = (np + 31)/32;
      const int lo = lane*seg, hi = lo + seg < np ? lo + seg : np;
      __shared__ int s_guess[32], s_end[32], s_err[32];
      int err = 0, werr = 0;
      int start = -1;
      if( lo < np ){
         if( lane == 0 ){
            start = s_first < np1 ? s_first : 0;
         }else{
            /* a guess only (checked below): the source cell whose edge is
             * the first at or after the upper edge of the cell before the
             * run, by binary search over the source edges unrolled from
             * the smallest; past the largest it is the cell that wraps */
            const double pt = sp[lo-1];
            const int rot = s_rot;
            int l0 = 0, h0 = np1;
            while( l0 < h0 ){
               int mid = (l0 + h0) >> 1;
               int k = rot + mid; if( k >= np1 ) k -= np1;
               if( sp1[k] < pt ) l0 = mid + 1; else h0 = mid;
            }
            start = rot + (l0 < np1 ? l0 : 0);
            if( start >= np1 ) start -= np1;
         }
      }
      s_guess[lane] = start;
      int endi = -1;
      if( lo < np && start >= 0 ) endi = zg_walk(sp, sd, sp1, sd1, np1, Pmax, lo, hi, start, st, cnt, &werr);
      s_end[lane] = endi;
      s_err[lane] = werr;           /* counts only if this run's start is confirmed */
      __syncwarp();
      if( lane == 0 ){
         int bad = 32;
         for( int l=1 ; l<32 && l*seg < np ; ++l )
            if( s_guess[l] < 0 || s_guess[l] != s_end[l-1] ){ bad = l; break; }
         for( int l=0 ; l<bad ; ++l ) err |= s_err[l];
         if( bad < 32 ) zg_walk(sp, sd, sp1, sd1, np1, Pmax, bad*seg, np, s_end[bad-1], st, cnt, &err);
      }
      raise_err(v, err);
   }
   __syncthreads();
   const int N = v.Ncell;
   for( int i=threadIdx.x ; i<np ; i+=blockDim.x ){
      double phip = sp[i], phim = sp[i] - sd[i];
      double acc[Q];
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) acc[q] = 0.0;
      int i1 = st[i];
      for( int n=0 ; n<cnt[i] ; ++n ){
         double phip1 = sp1[i1], phim1 = sp1[i1] - sd1[i1];
         int w = 0;
         while( phip1 < phim && w <= WRAP_CAP ){ phip1 += Pmax; phim1 += Pmax; ++w; }
         while( phim1 > phip && w <= 2*WRAP_CAP ){ phip1 -= Pmax; phim1 -= Pmax; ++w; }
         double phi1 = phip < phip1 ? phip : phip1;
         double phi2 = phim > phim1 ? phim : phim1;
         double dphi = phi1 - phi2;
#pragma unroll
         for( int q=0 ; q<Q ; ++q ) acc[q] += (double)v.prim[q*N + c10 + i1]*dphi;
         i1 = i1 < np1-1 ? i1+1 : 0;
      }
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) acc[q] = acc[q]/sd[i];
      const int sflags = sides[blockIdx.x];
      const int side = sflags & 3;
      R out[Q];
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) out[q] = (R)acc[q];
      if( sflags & 16 ){              /* no-slip: reflect_prims in r, phi and z */
         out[URR] = -out[URR]; out[UPP] = -out[UPP]; out[UZZ] = -out[UZZ];
      }else if( sflags & 8 ){         /* mirror copy: reflect_prims (euler.c:405, mhd.c:507) */
         if( side <= 1 ) out[URR] = -out[URR];
         else            out[UZZ] = -out[UZZ];
      }
      if( diode || (sflags & 4) ){
         if( side == 0 && out[URR] > R(0) ) out[URR] = R(0);
         if( side == 1 && out[URR] < R(0) ) out[URR] = R(0);
         if( side == 2 && out[UZZ] > R(0) ) out[UZZ] = R(0);
         if( side == 3 && out[UZZ] < R(0) ) out[UZZ] = R(0);
      }
      if( omk && side <= 1 ){
         const int j = v.ann_j[a], k = v.ann_k[a];
         const double *rj = v.rj + P.rj0 + 1;
         const double *zk = v.zk + P.zk0 + 1;
         double x[3] = { centroid_r(rj[j], rj[j-1]), phip - 0.5*sd[i], centroid_z(zk[k], zk[k-1]) };
         double tp[Q];
         initial<Q, (Q > 6 ? 8 : 5)>(P, tp, x);
         if( P.rotframe ) tp[UPP] -= P.RotOmega;
         out[UPP] = (R)tp[UPP];
      }
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) v.prim[q*N + c0 + i] = out[q];
   }
}

/* ------------------------------------------------------------------ per disk */
/* Start of timestep(): planet_RK_copy, reset of the dt reduction. */
template<class R>
__device__ __forceinline__ void disk_begin_body(const ViewT<R> &v, int d, int use_next){
   DiskState &S = v.ds[d];
   const DiskParams &P = v.dp[d];
   if( use_next ) S.dt = S.dt_next;
   for( int p=0 ; p<P.npl ; ++p ){
      Planet &pl = S.pl[p];
      pl.RK_r = pl.r; pl.RK_phi = pl.phi; pl.RK_M = pl.M; pl.RK_omega = pl.omega; pl.RK_vr = pl.vr;
      sincos(pl.phi, &pl.sphi, &pl.cphi);
   }
   double dt0 = P.maxDT / P.CFL;
   if( dt0 <= 0.0 ) dt0 = 1.0e100;
   S.dtmin = dbits(dt0);
}
template<class R>
__global__ void k_disk_begin(ViewT<R> v, int ndisk, int use_next){
   int d = blockIdx.x*blockDim.x + threadIdx.x;
   if( d < ndisk ) disk_begin_body<R>(v, d, use_next);
}

/* cos / sin of the planets' phi at set-up (later kept by k_disk_begin/mid) */
template<class R>
__global__ void k_planet_trig(ViewT<R> v, int ndisk){
   int d = blockIdx.x*blockDim.x + threadIdx.x;
   if( d >= ndisk ) return;
   DiskState &S = v.ds[d];
   for( int p=0 ; p<v.dp[d].npl ; ++p ) sincos(S.pl[p].phi, &S.pl[p].sphi, &S.pl[p].cphi);
}

/* After substep 1 (onestep.c:163-166, timestep.c:38): planet adjust/move,
 * planet phi wrap (clean_pi, misc.c:27-34), t += dt. */
template<class R>
__device__ __forceinline__ void disk_mid_body(const ViewT<R> &v, int d, double RK, int first, int advance_t){
   DiskState &S = v.ds[d];
   const DiskParams &P = v.dp[d];
   double dt = S.dt;
   double dts = first ? dt : 0.5*dt;
   if( first ){
      for( int p=0 ; p<P.npl ; ++p ){
         Planet &pl = S.pl[p];
         pl.r     = (1.-RK)*pl.r     + RK*pl.RK_r;
         pl.phi   = (1.-RK)*pl.phi   + RK*pl.RK_phi;
         pl.M     = (1.-RK)*pl.M     + RK*pl.RK_M;
         pl.omega = (1.-RK)*pl.omega + RK*pl.RK_omega;
         pl.vr    = (1.-RK)*pl.vr    + RK*pl.RK_vr;
         if( P.planets_move ) pl.phi += pl.omega*dts;
         if( P.pl_eps_decay ) pl.eps = P.pl_smooth + exp(-S.t/30.);   /* movePlanets(t = t_n) */
      }
   }
   for( int p=0 ; p<P.npl ; ++p ){
      Planet &pl = S.pl[p];
      double phi = pl.phi;
      int n = 0;
      while( phi > P.Pmax && n++ < WRAP_CAP ){ phi -= P.Pmax; pl.RK_phi -= P.Pmax; }
      while( phi < 0.0 && n++ < WRAP_CAP ){ phi += P.Pmax; pl.RK_phi += P.Pmax; }
      pl.phi = phi;
      sincos(phi, &pl.sphi, &pl.cphi);
   }
   if( advance_t ) S.t += dt;
}
template<class R>
__global__ void k_disk_mid(ViewT<R> v, int ndisk, double RK, int first, int advance_t){
   int d = blockIdx.x*blockDim.x + threadIdx.x;
   if( d < ndisk ) disk_mid_body<R>(v, d, RK, first, advance_t);
}

/* End of timestep(): dt of the next step, diagnostics time (analysis.c:105),
 * count_steps. */
template<class R>
__device__ __forceinline__ void disk_end_body(const ViewT<R> &v, int d){
   DiskState &S = v.ds[d];
   const DiskParams &P = v.dp[d];
   double mn = __longlong_as_double((long long)S.dtmin);
   S.dt_next = mn*P.CFL;
   S.t_avg += S.dt;
   S.count_steps += 1;
   if( !(S.dt_next > 0.0) || S.dt_next != S.dt_next || S.dt_next >= 1.0e99 )
      atomicOr(v.err, ERRF_NONFINITE);
}
template<class R>
__global__ void k_disk_end(ViewT<R> v, int ndisk){
   int d = blockIdx.x*blockDim.x + threadIdx.x;
   if( d < ndisk ) disk_end_body<R>(v, d);
}

/* Per annulus: sum its blocks' diagnostic partials in block order. */
template<class R>
__device__ __forceinline__ void diag_finish_body(const ViewT<R> &v, double *Qrz, const int *ann_blk0,
                                                 const int *ann_nblk, int a){
   int d = v.ann_disk[a];
   double dt = v.ds[d].dt;
   double s[DIAG_SLOTS] = {0,0,0,0,0,0,0,0,0};
   const int nq = v.nq;
   for( int bb=0 ; bb<ann_nblk[a] ; ++bb ){
      const double *p = v.diag_part + (size_t)(ann_blk0[a]+bb)*DIAG_SLOTS;
      for( int m=0 ; m<DIAG_SLOTS ; ++m ) if( m < nq || m == DIAG_VOL ) s[m] += p[m];
   }
   for( int m=0 ; m<nq ; ++m ) Qrz[(size_t)a*nq + m] += s[m]*dt / s[DIAG_VOL];
}
template<class R>
__global__ void k_diag_finish(ViewT<R> v, double *Qrz, const int *ann_blk0, const int *ann_nblk){
   int a = blockIdx.x*blockDim.x + threadIdx.x;
   if( a < v.Nann ) diag_finish_body<R>(v, Qrz, ann_blk0, ann_nblk, a);
}

/* ------------------------------------------------------------------ report
 * report() (report.c:7-202) as device reductions: per cell block the sums
 * (and minimum) of its real cells' terms, then per disk the totals, the
 * annulus-mean minimum and the derived values, so a report needs no copy of
 * the state.  Sums are block trees in a fixed order, not the reference's
 * serial loop (agreement to rounding, about 1e-15 relative). */
enum { RP_PSIR, RP_PSII, RP_L1ISEN, RP_L1RHO, RP_L1P, RP_L1B, RP_BR2, RP_BRBP, RP_B2, RP_PDV,
       RP_MDOT, RP_VOL, RP_MASS, RP_SR, RP_S0, RP_TORQUE, RP_POWER, RP_TORQUE2, RP_FR,
       RP_RHOMIN, RP_ARHO, RP_AVOL, RP_N };

template<int Q, int NC, class R>
__global__ void __launch_bounds__(CB) k_report_part(ViewT<R> v, double *part){
   __shared__ double s_red[CB/32][RP_N];
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   const int N = v.Ncell;
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   const DiskState &S = v.ds[d];
   int j = v.ann_j[a], k = v.ann_k[a];
   bool real = j >= P.NgRa && j < P.Nr - P.NgRb && k >= P.NgZa && k < P.Nz - P.NgZb;
   double x[RP_N];
#pragma unroll
   for( int m=0 ; m<RP_N ; ++m ) x[m] = 0.0;
   x[RP_RHOMIN] = HUGE_VAL;
   int err = 0;
   if( real && i < np ){
      int c = v.ann_off[a] + i;
      const double *rj = v.rj + P.rj0 + 1;
      const double *zk = v.zk + P.zk0 + 1;
      double phip = v.piph[c], dphi = v.dphi[c];
      double phi = phip - .5*dphi;
      double phim = phip - dphi;
      double dV = dV_of(rj[j], rj[j-1], get_dp(phip, phim, P.Pmax, &err), zk[k], zk[k-1]);
      double r = centroid_r(rj[j], rj[j-1]);
      double rho = (double)v.prim[RHO*N + c], Pp = (double)v.prim[PPP*N + c];
      double vr = (double)v.prim[URR*N + c];
      double sn, cs;
      sincos(phi, &sn, &cs);
      const double rho0 = 1.0;
      x[RP_PSIR] = rho*dV*cs;
      x[RP_PSII] = rho*dV*sn;
      x[RP_L1ISEN] = fabs(Pp/pow(rho, P.gam)-1.)*dV;
      x[RP_L1RHO] = fabs(rho/rho0-1.)*dV;
      x[RP_L1P] = fabs(Pp/pow(rho, 5./3.)/0.01-1.)*dV;
      if constexpr ( NC == 8 ){
         double Br = (double)v.prim[BRR*N + c], Bp = (double)v.prim[BPP*N + c];
         double Bz = (double)v.prim[BZZ*N + c];
         x[RP_L1B] = fabs(Br)*dV;
         x[RP_BR2] = .5*Br*Br*dV;
         x[RP_BRBP] = Br*Bp*dV;
         x[RP_B2] = .5*(Br*Br+Bp*Bp+Bz*Bz)*dV;
      }
      x[RP_PDV] = Pp*dV;
      x[RP_MDOT] = 2.*DISCO_PI*r*rho*dV*vr;
      x[RP_VOL] = dV;
      x[RP_RHOMIN] = rho/rho0;
      x[RP_ARHO] = rho*dV;
      x[RP_AVOL] = dV;
      x[RP_MASS] = rho*dV;
      double r4 = pow(rho, 4.);
      x[RP_SR] = r4*r*dV;
      x[RP_S0] = r4*dV;
      if( P.npl > 1 ){
         double fr, fp, fz, fp2;
         const Planet &p1 = S.pl[1];
         planetary_force(P.grav2D, S.pl[0], r, phi, 0.0, &fr, &fp2, &fz, 1);
         planetary_force(P.grav2D, p1, r, phi, 0.0, &fr, &fp, &fz, 1);
         x[RP_TORQUE] = -(rho-1.0)*p1.r*fp*dV;
         x[RP_POWER] = -(rho-1.0)*( p1.r*p1.omega*fp + p1.vr*fr )*dV;
         x[RP_TORQUE2] = -(rho-1.0)*p1.r*fp2*dV;
         x[RP_FR] = -(rho-1.0)*fr*dV;
      }
   }
   raise_err(v, err);
   int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
   for( int m=0 ; m<RP_N ; ++m ){
      double y = x[m];
#pragma unroll
      for( int o=16 ; o>0 ; o>>=1 ){
         double z = __shfl_down_sync(0xffffffffu, y, o);
         y = m == RP_RHOMIN ? (z < y ? z : y) : y + z;
      }
      if( lane == 0 ) s_red[wid][m] = y;
   }
   __syncthreads();
   if( threadIdx.x == 0 ){
      for( int m=0 ; m<RP_N ; ++m ){
         double y = s_red[0][m];
         for( int w=1 ; w<CB/32 ; ++w ) y = m == RP_RHOMIN ? (s_red[w][m] < y ? s_red[w][m] : y) : y + s_red[w][m];
         part[(size_t)blockIdx.x*RP_N + m] = y;
      }
   }
}

/* one thread per disk: totals over its blocks in annulus order, the minimum
 * over radii of the annulus (all z) mean density, the derived values; out =
 * the 17 numbers of a report.dat line (report.c:189-193) */
template<class R>
__global__ void k_report_finish(ViewT<R> v, const double *part, const int *ann_blk0,
                                const int *ann_nblk, double *out, int ndisk){
   int d = blockIdx.x*blockDim.x + threadIdx.x;
   if( d >= ndisk ) return;
   const DiskParams &P = v.dp[d];
   const DiskState &S = v.ds[d];
   double tot[RP_N];
   for( int m=0 ; m<RP_N ; ++m ) tot[m] = 0.0;
   tot[RP_RHOMIN] = HUGE_VAL;
   double rhoavg_min = HUGE_VAL;
   for( int j=P.NgRa ; j<P.Nr-P.NgRb ; ++j ){
      double arho = 0.0, avol = 0.0;
      for( int k=P.NgZa ; k<P.Nz-P.NgZb ; ++k ){
         int a = P.ann0 + j + P.Nr*k;
         for( int bb=0 ; bb<ann_nblk[a] ; ++bb ){
            const double *p = part + (size_t)(ann_blk0[a]+bb)*RP_N;
            for( int m=0 ; m<RP_RHOMIN ; ++m ) tot[m] += p[m];
            if( p[RP_RHOMIN] < tot[RP_RHOMIN] ) tot[RP_RHOMIN] = p[RP_RHOMIN];
            arho += p[RP_ARHO]; avol += p[RP_AVOL];
         }
      }
      double rho_avg = arho/avol;
      const double rho0 = 1.0;
      if( rhoavg_min > rho_avg/rho0 ) rhoavg_min = rho_avg/rho0;
   }
   double Vol = tot[RP_VOL];
   double *o = out + (size_t)d*17;
   o[0] = S.t;
   o[1] = tot[RP_TORQUE]; o[2] = tot[RP_POWER]; o[3] = tot[RP_FR];
   o[4] = tot[RP_RHOMIN]; o[5] = rhoavg_min;
   o[6] = tot[RP_PSIR]; o[7] = tot[RP_PSII]; o[8] = tot[RP_MASS];
   o[9] = tot[RP_MDOT]/Vol; o[10] = tot[RP_SR]/tot[RP_S0];
   o[11] = tot[RP_L1RHO]/Vol; o[12] = tot[RP_L1ISEN]/Vol; o[13] = tot[RP_L1B]/Vol;
   o[14] = tot[RP_BR2];
   o[15] = tot[RP_BRBP]/tot[RP_PDV];             /* aM */
   o[16] = tot[RP_PDV]/tot[RP_B2];               /* bM */
}

/* ------------------------------------------------------------------ setup
 * setupCells (domain.c:319-383): initial(), prim2cons, cons2prim on real
 * cells (FP64); then main.c's boundary_trans for ghosts. */
template<int Q, int NC, class R>
__global__ void __launch_bounds__(CB) k_setup(ViewT<R> v, int bc){
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const int N = v.Ncell;
   int c = v.ann_off[a] + i;
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   int j = v.ann_j[a], k = v.ann_k[a];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   bool real = j >= P.NgRa && j < P.Nr - P.NgRb && k >= P.NgZa && k < P.Nz - P.NgZb;
   int err = 0;
   double piph = v.piph[c], dphi = v.dphi[c];
   double prim[Q], cons[Q];
   if( real ){
      double z = centroid_z(zk[k], zk[k-1]);
      double r = centroid_r(rj[j], rj[j-1]);
      double phim = piph - dphi;
      double dph = get_dp(piph, phim, P.Pmax, &err);
      double dV = dV_of(rj[j], rj[j-1], dph, zk[k], zk[k-1]);
      double x[3] = {r, piph - .5*dphi, z};
      initial<Q,NC>(P, prim, x);
      if( P.rotframe ) prim[UPP] -= P.RotOmega;
      if( P.atmos )                                   /* domain.c:193-200 */
         for( int p=0 ; p<P.npl ; ++p ) adjust_gas(v.ds[d].pl[p], x, prim, P.gam);
      if( P.noise_type && v.noise )                   /* domain.c:202-203 */
         add_noise(P.noise_type, P.noise_abs, P.noise_rel, prim, x, v.noise + 4*(size_t)c);
      double om = get_om(P, r);
      bool done = false;
      if constexpr ( NC == 8 && sizeof(R) == sizeof(double) ){
         if( P.gr ){                /* grmhd2 prim2cons / cons2prim at x (domain.c:205, 237) */
            const GRParams G = gr_params(P);
            Metric3 g;
            metric_at(G, x, g);
            gr_prim2cons(G, g, prim, cons, x, dV);
            gr_cons2prim(P, g, cons, prim, x, dV);
            done = true;
         }
      }
      if( !done ){
         prim2cons<Q,NC,double>(P, prim, cons, r, om, dV);
         /* with CT, cons2prim follows set_B_fields (domain.c:211-237): k_c2p */
         if( !v.ct ) cons2prim<Q,NC>(P, cons, prim, r, om, dV);
      }
      /* main.c's boundary pass: a horizon module re-initialises the
       * excised cells' prims (their cons stay set-up's) */
      {
         const bool ex = P.bc_horizon && cell_excised(P, P.bc_horizon, j, k, rj, zk, piph, dphi);
         if( ex ) fixed_ghost_init<Q,NC>(P, bc, j, k, rj, zk, piph, dphi, prim);
         if( v.xflag ) v.xflag[c] = ex ? 1 : 0;
      }
#pragma unroll
      for( int q=0 ; q<Q ; ++q ){ v.prim[q*N+c] = (R)prim[q]; v.cons[q*N+c] = cons[q]; }
   }else{
      if( fixed_ghost_init<Q,NC>(P, bc, j, k, rj, zk, piph, dphi, prim) ){
#pragma unroll
         for( int q=0 ; q<Q ; ++q ) v.prim[q*N+c] = (R)prim[q];
      }
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) v.cons[q*N+c] = 0.0;
   }
   if constexpr ( sizeof(R) != sizeof(double) ){
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) v.ccarry[q*N+c] = 0.0f;
   }
   if constexpr ( NC == 8 ){
      if( v.ct ){                        /* set_B_fields, bfields.c:22-42 */
         double x[3] = { centroid_r(rj[j], rj[j-1]), piph, centroid_z(zk[k], zk[k-1]) };
         double pb[Q];
         initial<Q,NC>(P, pb, x);
         double dA = (rj[j]-rj[j-1])*(zk[k]-zk[k-1]);
         v.Phi[c] = pb[BPP]*dA;
         for( int s=1 ; s<v.nfs ; ++s ) v.Phi[(size_t)s*N + c] = 0.0;
      }
   }
   raise_err(v, err);
}

/* setupCells after restart() (domain.c:139-240 with restart_flag set): the
 * checkpoint's prim, Phi and piph are in place (Doub2Cell, h5in.c:72-77).
 * calc_dp (misc.c:271-288), wiph = 0, and on real cells prim2cons then
 * cons2prim -- no initial(), subtract_omega or set_B_fields, so the stored
 * face fluxes stand; ghosts as after set-up (main.c:53-62): the fixed
 * boundary's values, cons zero (h5in.c leaves the ghosts' cons unset and
 * nothing reads them). */
template<int Q, int NC, class R>
__global__ void __launch_bounds__(CB) k_restart(ViewT<R> v, int bc){
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const int N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + i;
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   int j = v.ann_j[a], k = v.ann_k[a];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   bool real = j >= P.NgRa && j < P.Nr - P.NgRb && k >= P.NgZa && k < P.Nz - P.NgZb;
   int err = 0;
   double piph = v.piph[c];
   double dphi = get_dp(piph, v.piph[c0 + (i == 0 ? np-1 : i-1)], P.Pmax, &err);
   v.dphi[c] = dphi;
   v.wiph[c] = 0.0;
   double prim[Q], cons[Q];
   if( real ){
      double z = centroid_z(zk[k], zk[k-1]);
      double r = centroid_r(rj[j], rj[j-1]);
      double dph = get_dp(piph, piph - dphi, P.Pmax, &err);
      double dV = dV_of(rj[j], rj[j-1], dph, zk[k], zk[k-1]);
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) prim[q] = (double)v.prim[q*N+c];
      if( P.noise_type && v.noise ){                  /* domain.c:202-203, restart too */
         double x[3] = {r, piph - .5*dphi, z};
         add_noise(P.noise_type, P.noise_abs, P.noise_rel, prim, x, v.noise + 4*(size_t)c);
      }
      double om = get_om(P, r);
      bool done = false;
      if constexpr ( NC == 8 && sizeof(R) == sizeof(double) ){
         if( P.gr ){
            double x[3] = {r, piph - .5*dphi, z};
            const GRParams G = gr_params(P);
            Metric3 g;
            metric_at(G, x, g);
            gr_prim2cons(G, g, prim, cons, x, dV);
            gr_cons2prim(P, g, cons, prim, x, dV);
            done = true;
         }
      }
      if( !done ){
         prim2cons<Q,NC,double>(P, prim, cons, r, om, dV);
         cons2prim<Q,NC>(P, cons, prim, r, om, dV);
      }
      {
         const bool ex = P.bc_horizon && cell_excised(P, P.bc_horizon, j, k, rj, zk, piph, dphi);
         if( ex ) fixed_ghost_init<Q,NC>(P, bc, j, k, rj, zk, piph, dphi, prim);
         if( v.xflag ) v.xflag[c] = ex ? 1 : 0;     /* setupCells marks the real cells anew */
      }
#pragma unroll
      for( int q=0 ; q<Q ; ++q ){ v.prim[q*N+c] = (R)prim[q]; v.cons[q*N+c] = cons[q]; }
   }else{
      if( fixed_ghost_init<Q,NC>(P, bc, j, k, rj, zk, piph, dphi, prim) ){
#pragma unroll
         for( int q=0 ; q<Q ; ++q ) v.prim[q*N+c] = (R)prim[q];
      }
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) v.cons[q*N+c] = 0.0;
   }
   if constexpr ( sizeof(R) != sizeof(double) ){
#pragma unroll
      for( int q=0 ; q<Q ; ++q ) v.ccarry[q*N+c] = 0.0f;
   }
   raise_err(v, err);
}

/* prim2cons on real cells for an upload without cons (domain.c:349). */
template<int Q, int NC, class R>
__global__ void __launch_bounds__(CB) k_prim2cons(ViewT<R> v){
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const int N = v.Ncell;
   int c = v.ann_off[a] + i;
   const DiskParams &P = v.dp[v.ann_disk[a]];
   int j = v.ann_j[a], k = v.ann_k[a];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   int err = 0;
   double piph = v.piph[c], dphi = v.dphi[c];
   double r = centroid_r(rj[j], rj[j-1]);
   double dph = get_dp(piph, piph - dphi, P.Pmax, &err);
   double dV = dV_of(rj[j], rj[j-1], dph, zk[k], zk[k-1]);
   double prim[Q], cons[Q];
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) prim[q] = (double)v.prim[q*N+c];
   bool done = false;
   if constexpr ( NC == 8 && sizeof(R) == sizeof(double) ){
      if( P.gr ){                   /* calc_cons with grmhd2 at the centroid */
         double x[3] = {r, piph - .5*dphi, centroid_z(zk[k], zk[k-1])};
         const GRParams G = gr_params(P);
         Metric3 g;
         metric_at(G, x, g);
         gr_prim2cons(G, g, prim, cons, x, dV);
         done = true;
      }
   }
   if( !done ) prim2cons<Q,NC,double>(P, prim, cons, r, get_om(P, r), dV);
#pragma unroll
   for( int q=0 ; q<Q ; ++q ) v.cons[q*N+c] = cons[q];
   raise_err(v, err);
}

/* set_wcell alone (setupCells' last call, domain.c:385). */
template<int Q, class R>
__global__ void __launch_bounds__(CB) k_wcell(ViewT<R> v){
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const int N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + i;
   int cp = c0 + (i+1 == np ? 0 : i+1);
   const DiskParams &P = v.dp[v.ann_disk[a]];
   double w = 0.0;
   bool gr = false;
   if constexpr ( Q == 9 && sizeof(R) == sizeof(double) ) gr = P.gr;
   if( gr ){                        /* set_wcell with grmhd2's get_omega */
      if( P.mesh_motion ){
         int j = v.ann_j[a], k = v.ann_k[a];
         const double *rj = v.rj + P.rj0 + 1, *zk = v.zk + P.zk0 + 1;
         double x[3] = {centroid_r(rj[j], rj[j-1]), 0.0, centroid_z(zk[k], zk[k-1])};
         double pc[Q], pr[Q];
         for( int q=0 ; q<Q ; ++q ){ pc[q] = (double)v.prim[q*N + c]; pr[q] = (double)v.prim[q*N + cp]; }
         w = .5*(gr_omega_at(P, pc, x) + gr_omega_at(P, pr, x));
      }
   }else if( P.mesh_motion ) w = .5*((double)v.prim[UPP*N + c] + (double)v.prim[UPP*N + cp]);
   if( P.mesh_motion == 4 ){
      int j = v.ann_j[a];
      const double *rj = v.rj + P.rj0 + 1;
      w = mesh_om(P, centroid_r(rj[j], rj[j-1]));
   }
   v.wiph[c] = w;
}

/* Stand-alone getmindt (misc.c:39-84) into ds[d].dtmin. */
template<int Q, int NC, class R>
__global__ void __launch_bounds__(CB) k_mindt(ViewT<R> v){
   __shared__ unsigned long long s_dt[CB/32];
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   const int N = v.Ncell;
   int c0 = v.ann_off[a];
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   int j = v.ann_j[a], k = v.ann_k[a];
   bool real = j >= P.NgRa && j < P.Nr - P.NgRb && k >= P.NgZa && k < P.Nz - P.NgZb;
   double dtc = 1.0e300;
   int err = 0;
   bool excised = P.bc_horizon && i < np &&
                  (v.xflag ? v.xflag[c0 + i] != 0
                           : horizon_cut(P, P.bc_horizon, j, k, v.rj + P.rj0 + 1, v.zk + P.zk0 + 1));
   if( i < np && real && !excised ){
      int c = c0 + i;
      const double *rj = v.rj + P.rj0 + 1;
      const double *zk = v.zk + P.zk0 + 1;
      double rp = rj[j], rm = rj[j-1], zp = zk[k], zm = zk[k-1];
      double piph = v.piph[c], phim = piph - v.dphi[c];
      int cprev = c0 + (i == 0 ? np-1 : i-1);
      double w = .5*(v.wiph[cprev] + v.wiph[c]);
      double r = centroid_r(rp, rm);
      bool gr = false;
      if constexpr ( NC == 8 && sizeof(R) == sizeof(double) ) gr = P.gr;
      if( gr ){                     /* mindt of grmhd2, grmhd2.c:748-832 */
         double pc[Q];
         for( int q=0 ; q<Q ; ++q ) pc[q] = (double)v.prim[q*N+c];
         double xp[3] = {rp, piph, zp}, xm[3] = {rm, phim, zm};
         double dtg = gr_mindt(P, v.gr_ann[a].m, pc, w, xp, xm, &err);
         if( dtg == dtg ) dtc = dtg;
      }else{
         double vp = ((double)v.prim[UPP*N+c]-w)*r;
         double cs = sqrt(P.gam*(double)v.prim[PPP*N+c]/(double)v.prim[RHO*N+c]);
         if constexpr ( NC == 8 ){               /* mhd.c:452-486: fast speed */
            double Br = v.prim[BRR*N+c], Bp = v.prim[BPP*N+c], Bz = v.prim[BZZ*N+c];
            double b2 = (Br*Br+Bp*Bp+Bz*Bz)/(double)v.prim[RHO*N+c];
            cs = sqrt(cs*cs + b2);
         }
         double maxvr = cs + fabs((double)v.prim[URR*N+c]);
         double maxvp = cs + fabs(vp);
         double maxvz = cs + fabs((double)v.prim[UZZ*N+c]);
         double dtr = (rp-rm)/maxvr;
         double dtp = (.5*(rp+rm))*get_dp(piph, phim, P.Pmax, &err)/maxvp;
         double dtz = (zp-zm)/maxvz;
         double dtm = dtr;
         if( dtm > dtp ) dtm = dtp;
         if( dtm > dtz ) dtm = dtz;
         if( P.visc ){
            double pc[Q];
#pragma unroll
            for( int q=0 ; q<Q ; ++q ) pc[q] = (double)v.prim[q*N+c];
            dtm = visc_dt_limit(P, pc, r, dtm, rp, rm, zp, zm, get_dp(piph, phim, P.Pmax, &err));
         }
         if( dtm == dtm ) dtc = dtm;
      }
   }
   raise_err(v, err);
   unsigned long long bits = dbits(dtc);
   int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
   for( int o=16 ; o>0 ; o>>=1 ){
      unsigned long long ob = __shfl_down_sync(0xffffffffu, bits, o);
      bits = ob < bits ? ob : bits;
   }
   if( lane == 0 ) s_dt[wid] = bits;
   __syncthreads();
   if( threadIdx.x == 0 && real ){
      unsigned long long mb = s_dt[0];
      for( int w=1 ; w<CB/32 ; ++w ) mb = s_dt[w] < mb ? s_dt[w] : mb;
      atomicMin(&v.ds[d].dtmin, mb);
   }
}

template<class R>
__global__ void k_mindt_begin(ViewT<R> v, int ndisk){
   int d = blockIdx.x*blockDim.x + threadIdx.x;
   if( d >= ndisk ) return;
   const DiskParams &P = v.dp[d];
   double dt0 = P.maxDT / P.CFL;
   if( dt0 <= 0.0 ) dt0 = 1.0e100;
   v.ds[d].dtmin = dbits(dt0);
}
template<class R>
__global__ void k_mindt_end(ViewT<R> v, int ndisk){
   int d = blockIdx.x*blockDim.x + threadIdx.x;
   if( d >= ndisk ) return;
   double mn = __longlong_as_double((long long)v.ds[d].dtmin);
   v.ds[d].dt_next = mn*v.dp[d].CFL;
}

} // namespace disco
