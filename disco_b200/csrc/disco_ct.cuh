/*
 * Constrained transport of the in-plane field in 2D (in.par
 * Constrained_Transport 1 with CT_MODE 1; bfields.c, riemann.c:73-85 and
 * 175-187, onestep.c:140-185), FP64, as order-preserving per-cell and
 * per-face kernels.
 *
 * The reference keeps the magnetic flux of every r-face in one slot of the
 * cell that "owns" the face (the face ending at the cell's piph: LRtype 0
 * -> L->Phi[2], LRtype 1 -> R->Phi[1], get_phi_pointer, bfields.c:734-758),
 * and the flux through the cell's phi face at piph in Phi[0].  A cell owns
 * exactly one face of each r-track beside it; the face builder records it
 * (consL / consR), so every scatter of bfields.c becomes a gather:
 *
 *   k_update     phi faces' (Ez, Br) from flux_to_E (also on the ghost
 *                annuli next to the real ones, misc.c:382-397)
 *   k_flux_t     r faces' (Erz, Brz)
 *   k_ct_edges   the cell's four edge values E[0..3], B[0..3]: the phi
 *                faces' half values plus the r faces' (riemann.c:175-187),
 *                in face order
 *   k_ct_faces   avg_Efields (bfields.c:392-644: phi average, then the
 *                face's interpolation) and subtract_advective_B_fluxes
 *                (:646-690) for each face's owner edge, then E dl dt
 *   k_ct_update  update_B_fluxes (:313-382): each slot gets its own face's
 *                -E dl dt and the previous face's +E dl dt in the order the
 *                reference's track loop applies them; Phi[0] the owned
 *                faces' terms, inner track first; then move_cells
 *   k_ct_flag    check_flipped (:693-731) on the moved cells
 *   k_ct_flip    flip_fluxes (:760-814): one warp per track, flagged faces
 *                in order by one lane (LRtype toggles carry to later ones)
 *   ct_cons_B    B_faces_to_cells type 1 (:88-182) before calc_prim
 *
 * Values the reference leaves stale (edge fields of annuli outside the
 * phi_flux range) are zero here; they reach only slots of ghost cells that
 * no real cell reads.  The pole branches of avg_Efields (NgRa/NgRb = 0)
 * write edges that no face owns, so they are not evaluated.
 */
#pragma once
#include "disco_kernels.cuh"

namespace disco {

/* annuli whose phi faces phi_flux evaluates under CT (misc.c:382-397) */
__device__ __forceinline__ bool ct_phi_annulus(const DiskParams &P, int j, int k){
   int jmin = P.NgRa == 0 ? 0 : P.NgRa-1, jmax = P.NgRb == 0 ? P.Nr : P.Nr-P.NgRb+1;
   int kmin = P.NgZa == 0 ? 0 : P.NgZa-1, kmax = P.NgZb == 0 ? P.Nz : P.Nz-P.NgZb+1;
   return j >= jmin && j < jmax && k >= kmin && k < kmax;
}

/* the slot holding face f's flux under its current LRtype */
template<class R>
__device__ __forceinline__ double *ct_slot(const ViewT<R> &v, double *base, int f){
   return v.fLR[f] == 0 ? base + 2*(size_t)v.Ncell + v.fL[f] : base + (size_t)v.Ncell + v.fR[f];
}

template<class R>
__global__ void __launch_bounds__(CB) k_ct_edges(ViewT<R> v){
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const int N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + i;
   int cm = c0 + (i == 0 ? np-1 : i-1);
   const DiskParams &P = v.dp[v.ann_disk[a]];
   int j = v.ann_j[a], k = v.ann_k[a];
   double E[4] = {0.0, 0.0, 0.0, 0.0}, B[4] = {0.0, 0.0, 0.0, 0.0};
   if( ct_phi_annulus(P, j, k) ){
      /* riemann_phi: cL->E[0], E[1] and cR->E[2], E[3] = .5 Ez (riemann.c:73-85) */
      double eR = .5*v.pE[c], eL = .5*v.pE[cm];
      double bR = .5*v.pB[c], bL = .5*v.pB[cm];
      E[0] = eR; E[1] = eR; E[2] = eL; E[3] = eL;
      B[0] = bR; B[1] = bR; B[2] = bL; B[3] = bL;
      double dph = v.dphi[c];
      int I0 = v.I0[a];
      /* riemann_trans dim 1 (riemann.c:175-187): as R of the inner track,
       * E[0], E[2] += .5 Erz fracR; as L of the outer track, E[1], E[3] */
      if( j >= 1 ){
         int t = P.trr0 + (j-1) + (P.Nr-1)*k;
         if( v.tr_flux[t] ){
            Runs rn = cell_runs(v, v.consR, t, c0, np, i, I0);
            for( int pass=0 ; pass<2 ; ++pass ){
               int s = pass ? rn.s2 : rn.s1, e = pass ? rn.e2 : rn.e1;
               for( int f=s ; f<=e ; ++f ){
                  double fr = v.fdp[f] / dph;
                  double xe = .5*v.fEt[f]*fr, xb = .5*v.fBt[f]*fr;
                  E[0] += xe; E[2] += xe; B[0] += xb; B[2] += xb;
               }
            }
         }
      }
      if( j <= P.Nr-2 ){
         int t = P.trr0 + j + (P.Nr-1)*k;
         if( v.tr_flux[t] ){
            Runs rn = cell_runs(v, v.consL, t, c0, np, i, I0);
            for( int pass=0 ; pass<2 ; ++pass ){
               int s = pass ? rn.s2 : rn.s1, e = pass ? rn.e2 : rn.e1;
               for( int f=s ; f<=e ; ++f ){
                  double fr = v.fdp[f] / dph;
                  double xe = .5*v.fEt[f]*fr, xb = .5*v.fBt[f]*fr;
                  E[1] += xe; E[3] += xe; B[1] += xb; B[3] += xb;
               }
            }
         }
      }
   }
#pragma unroll
   for( int s=0 ; s<4 ; ++s ){ v.ctE[s*N + c] = E[s]; v.ctB[s*N + c] = B[s]; }
}

/* next / previous cell of annulus a (cyclic) */
template<class R>
__device__ __forceinline__ int ct_next(const ViewT<R> &v, int a, int c){
   int o = v.ann_off[a], n = v.ann_np[a];
   return c+1 == o+n ? o : c+1;
}
template<class R>
__device__ __forceinline__ int ct_prev(const ViewT<R> &v, int a, int c){
   int o = v.ann_off[a], n = v.ann_np[a];
   return c == o ? o+n-1 : c-1;
}

template<class R>
__global__ void __launch_bounds__(FB) k_ct_faces(ViewT<R> v){
   int2 b = v.fblk[blockIdx.x];
   int t = b.x;
   if( v.tr_dim[t] != 1 ) return;
   int f = v.tr_off[t] + b.y + threadIdx.x;
   if( f >= v.tr_off[t+1] ) return;
   const size_t N = v.Ncell;
   int A = v.tr_a[t], Bn = v.tr_b[t];
   int d = v.ann_disk[A];
   const DiskParams &P = v.dp[d];
   int err = 0;
   int L = v.fL[f], Rc = v.fR[f];
   int lr = v.fLR[f];
   int o = lr == 0 ? L : Rc, c2 = lr == 0 ? Rc : L;
   int ao = lr == 0 ? A : Bn, a2 = lr == 0 ? Bn : A;
   int on = ct_next(v, ao, o);
   int c2n = ct_next(v, a2, c2), c2p = ct_prev(v, a2, c2);
   const double *E = v.ctE, *B = v.ctB;
   /* the phi average of avg_Efields: edge s of cell c becomes
    * .5 (E[s](c) + E[s+2](c+1)) for s = 0, 1 and .5 (E[s-2](c-1) + E[s](c))
    * for s = 2, 3 (bfields.c:400-418) */
   double p1 = v.piph[o], p2 = v.piph[c2];
   double dp1 = get_dp(p2, p1, P.Pmax, &err);
   double dp2 = v.dphi[c2] - dp1;
   double Eo, Bo, Eav, Bav;
   if( lr == 0 ){
      Eo = .5*(E[1*N + o] + E[3*N + on]);
      Bo = .5*(B[1*N + o] + B[3*N + on]);
      double e0 = .5*(E[0*N + c2] + E[2*N + c2n]), e2 = .5*(E[0*N + c2p] + E[2*N + c2]);
      double b0 = .5*(B[0*N + c2] + B[2*N + c2n]), b2 = .5*(B[0*N + c2p] + B[2*N + c2]);
      Eav = ( dp2*e0 + dp1*e2 )/(dp1+dp2);
      Bav = ( dp2*b0 + dp1*b2 )/(dp1+dp2);
   }else{
      Eo = .5*(E[0*N + o] + E[2*N + on]);
      Bo = .5*(B[0*N + o] + B[2*N + on]);
      double e1 = .5*(E[1*N + c2] + E[3*N + c2n]), e3 = .5*(E[1*N + c2p] + E[3*N + c2]);
      double b1 = .5*(B[1*N + c2] + B[3*N + c2n]), b3 = .5*(B[1*N + c2p] + B[3*N + c2]);
      Eav = ( dp2*e1 + dp1*e3 )/(dp1+dp2);
      Bav = ( dp2*b1 + dp1*b3 )/(dp1+dp2);
   }
   double fE = .5*(Eo + Eav);
   double fB = .5*(Bo + Bav);
   /* subtract_advective_B_fluxes: the owner's edge sits at r_jph[j] of the
    * track (hR of L, hL of R) and moves with the owner's wiph */
   int j = v.tr_j[t], k = v.tr_k[t];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   double h = rj[j];
   double w = v.wiph[o];
   double Ef = fE - h*w*fB;
   double dl = zk[k]-zk[k-1];                           /* r-face dl = dz, faces_alt.c:26-27 */
   double dt = v.ds[d].dt*v.dtfac;
   v.fX[f] = Ef*dl*dt;
   raise_err(v, err);
}

/* update_B_fluxes on the slots of cell c, then (first substep) move_cells /
 * clean_pi / calc_dp as k_update does without CT */
template<class R>
__global__ void __launch_bounds__(CB) k_ct_update(ViewT<R> v, int first){
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const size_t N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + i;
   const DiskParams &P = v.dp[v.ann_disk[a]];
   int j = v.ann_j[a], k = v.ann_k[a];
   const double *X = v.fX;
   double P0 = v.Phi[c];
   if( j >= 1 ){                           /* inner track: the owned face has LRtype 1 */
      int t = P.trr0 + (j-1) + (P.Nr-1)*k;
      int f = v.consR[c], o = v.tr_off[t];
      int fm = f > o ? f-1 : v.tr_off[t+1]-1;
      P0 = P0 - X[f];
      double S = v.Phi[N + c];
      S = f > o ? (S + X[fm]) - X[f] : (S - X[f]) + X[fm];
      v.Phi[N + c] = S;
   }
   if( j <= P.Nr-2 ){                      /* outer track: LRtype 0 */
      int t = P.trr0 + j + (P.Nr-1)*k;
      int f = v.consL[c], o = v.tr_off[t];
      int fm = f > o ? f-1 : v.tr_off[t+1]-1;
      P0 = P0 + X[f];
      double S = v.Phi[2*N + c];
      S = f > o ? (S + X[fm]) - X[f] : (S - X[f]) + X[fm];
      v.Phi[2*N + c] = S;
   }
   v.Phi[c] = P0;
   if( first ){
      int err = 0;
      int cprev = c0 + (i == 0 ? np-1 : i-1);
      double piph = v.piph_new[c];
      v.dphi[c] = get_dp(piph, v.piph_new[cprev], P.Pmax, &err);
      v.piph[c] = piph;
      raise_err(v, err);
   }
}

/* check_flipped: face g is flagged when its owner's piph now lies before
 * the previous face's owner's */
template<class R>
__global__ void __launch_bounds__(FB) k_ct_flag(ViewT<R> v){
   int2 b = v.fblk[blockIdx.x];
   int t = b.x;
   if( v.tr_dim[t] != 1 ) return;
   int f = v.tr_off[t] + b.y + threadIdx.x;
   if( f >= v.tr_off[t+1] ) return;
   const DiskParams &P = v.dp[v.ann_disk[v.tr_a[t]]];
   int err = 0;
   int fm = f > v.tr_off[t] ? f-1 : v.tr_off[t+1]-1;
   int own = v.fLR[f] == 0 ? v.fL[f] : v.fR[f];
   int ownm = v.fLR[fm] == 0 ? v.fL[fm] : v.fR[fm];
   double dp = get_signed_dp(v.piph[own], v.piph[ownm], P.Pmax, &err);
   v.fFlip[f] = dp < 0. ? 1 : 0;
   raise_err(v, err);
}

/* flip_fluxes, one warp per track */
template<class R>
__global__ void k_ct_flip(ViewT<R> v){
   int t = (blockIdx.x*blockDim.x + threadIdx.x) >> 5;
   int lane = threadIdx.x & 31;
   if( t >= v.Ntr || v.tr_dim[t] != 1 ) return;
   int o = v.tr_off[t], n = v.tr_off[t+1] - o;
   for( int base=0 ; base<n ; base+=32 ){
      bool fl = base + lane < n && v.fFlip[o + base + lane];
      unsigned m = __ballot_sync(0xffffffffu, fl);
      if( lane == 0 ){
         while( m ){
            int f = o + base + __ffs(m) - 1;
            m &= m - 1;
            int fm = f > o ? f-1 : o+n-1;
            int fp = f < o+n-1 ? f+1 : o;
            double *Pf = ct_slot(v, v.Phi, f), *Rf = ct_slot(v, v.RKPhi, f);
            double *Pm = ct_slot(v, v.Phi, fm), *Rm = ct_slot(v, v.RKPhi, fm);
            double *Pp = ct_slot(v, v.Phi, fp), *Rp = ct_slot(v, v.RKPhi, fp);
            double ph = *Pf, rk = *Rf;
            *Pf = *Pm + ph;
            *Rf = *Rm + rk;
            *Pm = -ph;
            *Rm = -rk;
            *Pp = *Pp + ph;
            *Rp = *Rp + rk;
            v.fLR[f] ^= 1;
            v.fLR[fm] ^= 1;
         }
      }
      __syncwarp();
   }
}

/* B_faces_to_cells type 1 for a real cell (bfields.c:114-182): cons[BRR] from
 * the fluxes of the cell's r faces (inner track first, each in face order,
 * slots by the current LRtype) over their area, cons[BPP] from the two phi
 * faces, with the moved cell's volume */
template<class R>
__device__ void ct_cons_B(const ViewT<R> &v, const DiskParams &P, int a, int c0, int np, int i,
                          int j, int k, double rp, double rm, double zp, double zm, double *cons,
                          int *err){
   const size_t N = v.Ncell;
   int c = c0 + i, cm = c0 + (i == 0 ? np-1 : i-1);
   double S = 0.0, T = 0.0;
   int I0 = v.I0[a];
   if( j >= 1 ){
      Runs rn = cell_runs(v, v.consR, P.trr0 + (j-1) + (P.Nr-1)*k, c0, np, i, I0);
      for( int pass=0 ; pass<2 ; ++pass ){
         int s = pass ? rn.s2 : rn.s1, e = pass ? rn.e2 : rn.e1;
         for( int f=s ; f<=e ; ++f ){
            S += v.fLR[f] == 0 ? v.Phi[2*N + v.fL[f]] : v.Phi[N + v.fR[f]];
            T += v.fdA[f];
         }
      }
   }
   if( j <= P.Nr-2 ){
      Runs rn = cell_runs(v, v.consL, P.trr0 + j + (P.Nr-1)*k, c0, np, i, I0);
      for( int pass=0 ; pass<2 ; ++pass ){
         int s = pass ? rn.s2 : rn.s1, e = pass ? rn.e2 : rn.e1;
         for( int f=s ; f<=e ; ++f ){
            S += v.fLR[f] == 0 ? v.Phi[2*N + v.fL[f]] : v.Phi[N + v.fR[f]];
            T += v.fdA[f];
         }
      }
   }
   double x0 = centroid_r(rp, rm);
   double dph = get_dp(v.piph[c], v.piph[cm], P.Pmax, err);
   double dV = dV_of(rp, rm, dph, zp, zm);
   double dA = (rp-rm)*(zp-zm);
   double rfac = 1.0/x0;                                /* bfield_scale_factor(x0, 0) */
   double hr = 1.0, hp = x0;
   cons[BRR] = S * (dV*rfac/(T * hr));
   cons[BPP] = .5*(v.Phi[c]+v.Phi[cm])*dV/(dA * hp);
}

/* set_B_fields (bfields.c:49-61): each r face's flux prim[BRR] dA at its
 * centre, into its owner's slot */
template<int Q, int NC, class R>
__global__ void __launch_bounds__(FB) k_ct_face_init(ViewT<R> v){
   int2 b = v.fblk[blockIdx.x];
   int t = b.x;
   if( v.tr_dim[t] != 1 ) return;
   int f = v.tr_off[t] + b.y + threadIdx.x;
   if( f >= v.tr_off[t+1] ) return;
   const DiskParams &P = v.dp[v.ann_disk[v.tr_a[t]]];
   int j = v.tr_j[t], k = v.tr_k[t];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   double x[3] = { .5*(rj[j]+rj[j]), v.fphic[f], 0.5*(zk[k]+zk[k-1]) };
   double prim[Q];
   initial<Q,NC>(P, prim, x);
   *ct_slot(v, v.Phi, f) = prim[BRR]*v.fdA[f];
}

}  // namespace disco
