/*
 * Constrained transport (in.par Constrained_Transport 1; bfields.c,
 * riemann.c:73-110 and 175-213, onestep.c:140-185) as order-preserving
 * per-cell and per-face kernels.  CT_MODE 1 (2D: the in-plane field) and
 * CT_MODE 2 (3D: also the z faces, the E_phi edges and make_edge_adjust).
 * The edge arithmetic runs in the bulk real type R (FP32 in the mixed form);
 * the face fluxes Phi and their updates E dl dt stay FP64, so CT keeps the
 * discrete div B in both forms.
 *
 * The reference keeps the magnetic flux of every r- or z-face in one slot of
 * the cell that "owns" the face (the face ending at the cell's piph: r faces
 * LRtype 0 -> L->Phi[2], 1 -> R->Phi[1]; z faces L->Phi[4], R->Phi[3];
 * get_phi_pointer, bfields.c:734-758) and the flux through the cell's phi
 * face at piph in Phi[0].  A cell owns exactly one face of each track beside
 * it; the face builder records it (consL / consR, consZL / consZR), so every
 * scatter of bfields.c becomes a gather:
 *
 *   k_update     phi faces' (Ez, Br, Er, Bz) from flux_to_E (also on the
 *                ghost annuli next to the real ones, misc.c:382-397)
 *   k_flux_t     r and z faces' (Erz, Brz, E_phi)
 *   k_ct_edges   each cell's edge values E[0..7], B[0..7]: the phi faces'
 *                half values plus the r and z faces' fractions, in face order
 *   k_ct_faces   avg_Efields (bfields.c:392-644: phi average, then the
 *                face's interpolation) and subtract_advective_B_fluxes
 *                (:646-690) for each face's owner edge, then E dl dt
 *   k_ct_line    make_edge_adjust's 4-way merge (bfields.c:888-1127) as a
 *                merge path: each cell finds its step in the merge of every
 *                edge line it borders (from the face lists of the two tracks
 *                it shares with the line and one binary search for the
 *                diagonal annulus), re-evaluates get_which4 there and writes
 *                that step's E_phi dl dt
 *   k_ct_update  update_B_fluxes (:313-382) and make_edge_adjust on each
 *                cell's slots: a slot gets its own face's term and the
 *                previous face's, in the order the track loop applies them,
 *                then the edge steps of its two lines, in line order; Phi[0]
 *                the owned faces' terms; then move_cells
 *   k_ct_flag    check_flipped (:693-731) on the moved cells
 *   k_ct_flip    flip_fluxes (:760-814): one warp per track, flagged faces
 *                in order by one lane (LRtype toggles carry to later ones)
 *   ct_cons_B    B_faces_to_cells type 1 (:88-309) before calc_prim
 *
 * Values the reference leaves stale (edge fields and E_phi of annuli and
 * faces outside the CT flux ranges) are zero here; they reach only slots of
 * ghost cells' faces that no real cell reads.  The r-pole branches of
 * avg_Efields (NgRa/NgRb = 0) write edges that no face owns, so they are not
 * evaluated; the z-pole branches (NgZa/NgZb = 0 in 3D) reach the z faces the
 * bottom layer's cells own above them and the top layer's own below them:
 * k_ct_faces keeps those faces' E per owner and k_ct_zpole writes their X
 * from the annulus mean.
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

/* the slot holding face f's flux under its current LRtype (z: zf) */
template<class R>
__device__ __forceinline__ double *ct_slot(const ViewT<R> &v, double *base, int f, bool zf){
   size_t N = v.Ncell;
   if( zf ) return v.fLR[f] == 0 ? base + 4*N + v.fL[f] : base + 3*N + v.fR[f];
   return v.fLR[f] == 0 ? base + 2*N + v.fL[f] : base + N + v.fR[f];
}

/* fn(f) for each face of cell i's runs in track t, in face order */
template<class R, class F>
__device__ __forceinline__ void ct_over_runs(const ViewT<R> &v, const int *cons, int t, int c0,
                                             int np, int i, int I0, F fn){
   Runs rn = cell_runs(v, cons, t, c0, np, i, I0);
   for( int f=rn.s1 ; f<=rn.e1 ; ++f ) fn(f);
   for( int f=rn.s2 ; f<=rn.e2 ; ++f ) fn(f);
}

template<class R>
__global__ void __launch_bounds__(CB) k_ct_edges(ViewT<R> v){
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const size_t N = v.Ncell;
   int c0 = v.ann_off[a], c = c0 + i;
   int cm = c0 + (i == 0 ? np-1 : i-1);
   const DiskParams &P = v.dp[v.ann_disk[a]];
   int j = v.ann_j[a], k = v.ann_k[a];
   const int ne = v.ct == 2 ? 8 : 4;
   R E[8] = {0,0,0,0,0,0,0,0}, B[8] = {0,0,0,0,0,0,0,0};
   if( ct_phi_annulus(P, j, k) ){
      /* riemann_phi: cL->E[0], E[1] (E[4], E[5]) and cR->E[2], E[3] (E[6],
       * E[7]) = .5 Ez (.5 Er), riemann.c:73-110 */
      R eR = R(.5)*v.pE[c], eL = R(.5)*v.pE[cm];
      R bR = R(.5)*v.pB[c], bL = R(.5)*v.pB[cm];
      E[0] = eR; E[1] = eR; E[2] = eL; E[3] = eL;
      B[0] = bR; B[1] = bR; B[2] = bL; B[3] = bL;
      if( v.ct == 2 ){
         R zR = R(.5)*v.pEr[c], zL = R(.5)*v.pEr[cm];
         R wR = R(.5)*v.pBz[c], wL = R(.5)*v.pBz[cm];
         E[4] = zR; E[5] = zR; E[6] = zL; E[7] = zL;
         B[4] = wR; B[5] = wR; B[6] = wL; B[7] = wL;
      }
      R dph = (R)v.dphi[c];
      int I0 = v.I0[a];
      /* riemann_trans (riemann.c:175-205): as R of the inner (lower) track
       * E[0], E[2] (E[4], E[6]) += .5 Erz fracR; as L of the outer (upper)
       * track E[1], E[3] (E[5], E[7]) += .5 Erz fracL */
      auto add = [&](int lo, int hi) {
         return [&, lo, hi](int f) {
            R fr = (R)v.fdp[f] / dph;
            R xe = R(.5)*v.fEt[f]*fr, xb = R(.5)*v.fBt[f]*fr;
            E[lo] += xe; E[hi] += xe; B[lo] += xb; B[hi] += xb;
         };
      };
      if( j >= 1 ){
         int t = P.trr0 + (j-1) + (P.Nr-1)*k;
         if( v.tr_flux[t] ) ct_over_runs(v, v.consR, t, c0, np, i, I0, add(0, 2));
      }
      if( j <= P.Nr-2 ){
         int t = P.trr0 + j + (P.Nr-1)*k;
         if( v.tr_flux[t] ) ct_over_runs(v, v.consL, t, c0, np, i, I0, add(1, 3));
      }
      if( v.ct == 2 && P.Nz > 1 ){
         if( k >= 1 ){
            int t = P.trz0 + j + P.Nr*(k-1);
            if( v.tr_flux[t] ) ct_over_runs(v, v.consZR, t, c0, np, i, I0, add(4, 6));
         }
         if( k <= P.Nz-2 ){
            int t = P.trz0 + j + P.Nr*k;
            if( v.tr_flux[t] ) ct_over_runs(v, v.consZL, t, c0, np, i, I0, add(5, 7));
         }
      }
   }
#pragma unroll
   for( int s=0 ; s<8 ; ++s ) if( s < ne ){ v.ctE[s*N + c] = E[s]; v.ctB[s*N + c] = B[s]; }
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
   bool zf = v.tr_dim[t] == 2;
   if( zf && v.ct != 2 ) return;
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
   const R *E = v.ctE, *B = v.ctB;
   const size_t s0 = zf ? 4 : 0;          /* r faces use edges 0-3, z faces 4-7 */
   /* the phi average of avg_Efields: edge s of cell c becomes
    * .5 (E[s](c) + E[s+2](c+1)) for the right edges s = 0, 1 and
    * .5 (E[s-2](c-1) + E[s](c)) for the left ones (bfields.c:400-442) */
   double p1 = v.piph[o], p2 = v.piph[c2];
   double dp1 = get_dp(p2, p1, P.Pmax, &err);
   double dp2 = v.dphi[c2] - dp1;
   const R w1 = (R)dp1, w2 = (R)dp2;
   /* owner edge s_o (and its left twin s_o+2); c2's edges s_c, s_c+2 */
   size_t so = lr == 0 ? s0+1 : s0, sc = lr == 0 ? s0 : s0+1;
   R Eo = R(.5)*(E[so*N + o] + E[(so+2)*N + on]);
   R Bo = R(.5)*(B[so*N + o] + B[(so+2)*N + on]);
   R ea = R(.5)*(E[sc*N + c2] + E[(sc+2)*N + c2n]), eb = R(.5)*(E[sc*N + c2p] + E[(sc+2)*N + c2]);
   R ba = R(.5)*(B[sc*N + c2] + B[(sc+2)*N + c2n]), bb = R(.5)*(B[sc*N + c2p] + B[(sc+2)*N + c2]);
   R Eav = ( w2*ea + w1*eb )/(w1+w2);
   R Bav = ( w2*ba + w1*bb )/(w1+w2);
   R fE = R(.5)*(Eo + Eav);
   R fB = R(.5)*(Bo + Bav);
   /* subtract_advective_B_fluxes: the owner's edge moves with its wiph; an
    * r face's edge sits at r_jph[j] (E -= h w B), a z face's at the
    * annulus centroid (E += h w B) */
   int j = v.tr_j[t], k = v.tr_k[t];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   double w = v.wiph[o];
   R Ef;
   double dl;
   if( !zf ){
      double h = rj[j];
      Ef = fE - (R)(h*w)*fB;
      dl = zk[k]-zk[k-1];                         /* r-face dl = dz, faces_alt.c:26-27 */
   }else{
      double h = v.tr_r[t];                        /* centroid_r(r_j, r_j-1) */
      Ef = fE + (R)(h*w)*fB;
      dl = rj[j]-rj[j-1];                         /* z-face dl = dr */
   }
   double dt = v.ds[d].dt*v.dtfac;
   /* avg_Efields' z-pole branch (bfields.c:580-617): without z ghosts the
    * bottom layer's E[5] and the top layer's E[4] become their annulus's
    * mean and B 0 -- the owner's value is kept for k_ct_zpole, which writes
    * these faces' X */
   if( zf && v.ctPole && ((lr == 0 && k == 0 && P.NgZa == 0) ||
                          (lr == 1 && k+1 == P.Nz-1 && P.NgZb == 0)) ){
      v.ctPole[o] = (double)fE;
   }else{
      v.fX[f] = (double)Ef*dl*dt;
   }
   raise_err(v, err);
}

/* The z-pole average (bfields.c:580-617) of pole annulus pl[blockIdx.x]
 * (x: annulus, y: 0 the bottom layer, its cells' upper faces; 1 the top
 * layer, their lower faces): E = the sum of the cells' owned-face E in cell
 * order over Np, B = 0, so the advective term vanishes and each owned face
 * takes X = E dl dt. */
template<class R>
__global__ void __launch_bounds__(CB) k_ct_zpole(ViewT<R> v, const int2 *pl){
   __shared__ double s_E;
   const int2 pa = pl[blockIdx.x];
   const int a = pa.x, top = pa.y;
   const int np = v.ann_np[a], c0 = v.ann_off[a];
   const int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   if( threadIdx.x == 0 ){
      double E = 0.0;
      for( int i=0 ; i<np ; ++i ) E += v.ctPole[c0 + i];
      s_E = E/np;
   }
   __syncthreads();
   const int j = v.ann_j[a];
   const double *rj = v.rj + P.rj0 + 1;
   const double dl = rj[j]-rj[j-1];                   /* z-face dl = dr */
   const double dt = v.ds[d].dt*v.dtfac;
   const R E = (R)s_E;
   const int *own = top ? v.consZR : v.consZL;
   for( int i=threadIdx.x ; i<np ; i+=blockDim.x ) v.fX[own[c0 + i]] = (double)E*dl*dt;
}

/* get_which4 (bfields.c:834-885): which of four phi edges is smallest (mode
 * 0) or largest (mode 1), comparing pairs with the periodic wrap of
 * phi_switch (:818-832), and the toggles of the two pairs not chosen */
__device__ __forceinline__ int ct_phi_switch(double dphi, double Pmax, int mode, int *err){
   int n = 0;
   while( dphi > .5*Pmax ){ dphi -= Pmax; if( ++n > WRAP_CAP ){ *err |= ERRF_WRAP; break; } }
   while( dphi <-.5*Pmax ){ dphi += Pmax; if( ++n > WRAP_CAP ){ *err |= ERRF_WRAP; break; } }
   if( mode == 1 ) dphi = -dphi;
   return dphi > 0. ? 1 : 0;
}
__device__ __forceinline__ int ct_which4(double phi, double phiR, double phiU, double phiUR,
                                         int *LR_alt, int *UD_alt, int mode, double Pmax, int *err){
   int LR_D = ct_phi_switch(phi - phiR, Pmax, mode, err);
   int LR_U = ct_phi_switch(phiU - phiUR, Pmax, mode, err);
   double phi1 = LR_D ? phiR : phi;
   double phi2 = LR_U ? phiUR : phiU;
   int UD = ct_phi_switch(phi1 - phi2, Pmax, mode, err);
   int which4 = UD == 0 ? (LR_D == 0 ? 0 : 1) : (LR_U == 0 ? 2 : 3);
   if( mode == 0 ){
      *LR_alt = (which4 == 0 || which4 == 1) ? LR_U : LR_D;
      if( which4 == 0 || which4 == 2 ) *UD_alt = ct_phi_switch(phiR - phiUR, Pmax, mode, err);
      else                             *UD_alt = ct_phi_switch(phi - phiU, Pmax, mode, err);
   }
   return which4;
}

/* E_phi of the face cell c owns on side s (0 inner r, 1 outer r, 2 lower z,
 * 3 upper z), as riemann_trans left it (riemann.c:188-212); cell (jc, kc) */
template<class R>
__device__ __forceinline__ R ct_ephi(const ViewT<R> &v, const DiskParams &P, int c, int jc,
                                     int kc, int s){
   int t, f;
   if( s == 0 ){ t = P.trr0 + (jc-1) + (P.Nr-1)*kc; f = v.consR[c]; }
   else if( s == 1 ){ t = P.trr0 + jc + (P.Nr-1)*kc; f = v.consL[c]; }
   else if( s == 2 ){ t = P.trz0 + jc + P.Nr*(kc-1); f = v.consZR[c]; }
   else { t = P.trz0 + jc + P.Nr*kc; f = v.consZL[c]; }
   return v.tr_flux[t] ? v.fEphi[f] : R(0.0);
}

/* make_edge_adjust, one thread per (cell, list): the line (jl, kl) is the
 * r_jph[jl], z_kph[kl] edge; its lists are the annuli (jl,kl) [c],
 * (jl+1,kl) [cR], (jl,kl+1) [cU], (jl+1,kl+1) [cUR], each from its I0, and
 * the reference merges them by repeated get_which4, ties to the lower list
 * index.  A cell of list m at position t is consumed at step
 * e = t + (cells of each other list before it): two of those counts are the
 * cell's position in the face list of the track it shares with that list
 * minus t, the third (the diagonal annulus) a binary search. */
template<class R>
__global__ void __launch_bounds__(CB) k_ct_line(ViewT<R> v){
   int2 b = v.cblk[blockIdx.x];
   int a = b.x, i = b.y + threadIdx.x;
   int np = v.ann_np[a];
   if( i >= np ) return;
   const size_t N = v.Ncell;
   int c = v.ann_off[a] + i;
   int d = v.ann_disk[a];
   const DiskParams &P = v.dp[d];
   if( P.Nz < 2 ) return;
   int j = v.ann_j[a], k = v.ann_k[a];
   const double *rj = v.rj + P.rj0 + 1;
   const double Pmax = P.Pmax;
   const double dt = v.ds[d].dt*v.dtfac;
   int err = 0;
   int t = i - v.I0[a];
   if( t < 0 ) t += np;
   double ux = v.piph[c];
   for( int m=0 ; m<4 ; ++m ){
      int jl = j - (m & 1), kl = k - (m >> 1);
      if( jl < 0 || jl > P.Nr-2 || kl < 0 || kl > P.Nz-2 ) continue;
      int an[4], cnt[4];
      for( int n=0 ; n<4 ; ++n ) an[n] = P.ann0 + (jl + (n & 1)) + P.Nr*(kl + (n >> 1));
      cnt[m] = t;
      for( int n=0 ; n<4 ; ++n ){
         if( n == m ) continue;
         int x = n ^ m;
         if( x == 1 ){                /* same layer: the r-track of that layer */
            int tr = P.trr0 + jl + (P.Nr-1)*(kl + (m >> 1));
            int f = (m & 1) ? v.consR[c] : v.consL[c];
            cnt[n] = f - v.tr_off[tr] - t;
         }else if( x == 2 ){          /* same column: the z-track of that column */
            int tz = P.trz0 + (jl + (m & 1)) + P.Nr*kl;
            int f = (m >> 1) ? v.consZR[c] : v.consZL[c];
            cnt[n] = f - v.tr_off[tz] - t;
         }else{                       /* diagonal: cells of list n before this one */
            int o = v.ann_off[an[n]], nn = v.ann_np[an[n]], I0n = v.I0[an[n]];
            /* both lists unrolled from I0: the count is near t nn / np */
            cnt[n] = gallop_lb(0, nn, __float2int_rz(__fdividef((float)t*(float)nn, (float)np)), [&](int mid){
               int s = I0n + mid; if( s >= nn ) s -= nn;
               double uy = v.piph[o + s];
               return !(n < m ? uy <= ux : uy < ux);
            });
         }
      }
      int e = cnt[0] + cnt[1] + cnt[2] + cnt[3];
      int line = P.ln0 + jl + (P.Nr-1)*kl;
      if( e < 0 || e >= v.line_off[line+1] - v.line_off[line] ){ err |= ERRF_INTERNAL; continue; }
      v.rk[m*N + c] = e;
      /* the reference's state at step e */
      int cur[4];
      bool bad = false;
      for( int n=0 ; n<4 ; ++n ){
         int o = v.ann_off[an[n]], nn = v.ann_np[an[n]];
         int s = v.I0[an[n]] + cnt[n];          /* I0 < nn, 0 <= cnt <= nn */
         if( s >= nn ) s -= nn;
         if( s < 0 || s >= nn ){ bad = true; s = 0; }
         cur[n] = o + s;
      }
      if( bad ){ err |= ERRF_INTERNAL; continue; }
      int LR_alt = 0, UD_alt = 0;
      int w4 = ct_which4(v.piph[cur[0]], v.piph[cur[1]], v.piph[cur[2]], v.piph[cur[3]],
                         &LR_alt, &UD_alt, 0, Pmax, &err);
      int w4b = ct_which4(v.piph[cur[0]] - v.dphi[cur[0]], v.piph[cur[1]] - v.dphi[cur[1]],
                          v.piph[cur[2]] - v.dphi[cur[2]], v.piph[cur[3]] - v.dphi[cur[3]],
                          NULL, NULL, 1, Pmax, &err);
      if( w4 != m ) err |= ERRF_INTERNAL;
      /* E_phi of the cells' owned faces: c [3],[1]; cR [3],[0]; cU [1],[2]; cUR [0],[2] */
      auto eph = [&](int n, int s){ return ct_ephi(v, P, cur[n], jl + (n & 1), kl + (n >> 1), s); };
      const R q4 = R(.25);
      R E;
      if( w4 == 0 ){
         E = q4*( eph(0,3) + eph(0,1) );
         if( LR_alt == 0 ) E += q4*eph(2,1); else E += q4*eph(3,0);
         if( UD_alt == 0 ) E += q4*eph(1,3); else E += q4*eph(3,2);
      }else if( w4 == 1 ){
         E = q4*( eph(1,3) + eph(1,0) );
         if( LR_alt == 0 ) E += q4*eph(2,1); else E += q4*eph(3,0);
         if( UD_alt == 0 ) E += q4*eph(0,3); else E += q4*eph(2,2);
      }else if( w4 == 2 ){
         E = q4*( eph(2,2) + eph(2,1) );
         if( LR_alt == 0 ) E += q4*eph(0,1); else E += q4*eph(1,0);
         if( UD_alt == 0 ) E += q4*eph(1,3); else E += q4*eph(3,2);
      }else{
         E = q4*( eph(3,2) + eph(3,0) );
         if( LR_alt == 0 ) E += q4*eph(0,1); else E += q4*eph(1,0);
         if( UD_alt == 0 ) E += q4*eph(0,3); else E += q4*eph(2,2);
      }
      double xp1 = v.piph[cur[w4]];
      double xm1 = v.piph[cur[w4b]] - v.dphi[cur[w4b]];
      double dl = (.5*(rj[jl]+rj[jl]))*get_dp(xp1, xm1, Pmax, &err);   /* get_dL(.,.,0) */
      v.lineX[v.line_off[line] + e] = (double)E*dl*dt;
   }
   raise_err(v, err);
}

/* The edge steps of line l that fall on face f of a track whose two cells'
 * lists in that line are mA (first / inner-lower annulus) and mB: the steps
 * whose pointer sum over the pair equals the face's index d, i.e. after the
 * element that ends face d-1 up to the one that ends face d; face 0 also
 * takes the steps after the pair's last element (the pair has wrapped).
 * Applied in step order as S += sign X. */
template<class R>
__device__ __forceinline__ double ct_line_terms(const ViewT<R> &v, double S, int line, int tr,
                                                int f, int mA, int mB, double sign){
   const size_t N = v.Ncell;
   const double *X = v.lineX + v.line_off[line];
   int f0 = v.tr_off[tr], f1 = v.tr_off[tr+1];
   auto rank = [&](int g){
      return v.fLR[g] == 0 ? v.rk[mA*N + v.fL[g]] : v.rk[mB*N + v.fR[g]];
   };
   int hi = rank(f);
   int lo = f == f0 ? 0 : rank(f-1) + 1;
   for( int e=lo ; e<=hi ; ++e ) S += sign*X[e];
   if( f == f0 ){
      int ne = v.line_off[line+1] - v.line_off[line];
      for( int e=rank(f1-1)+1 ; e<ne ; ++e ) S += sign*X[e];
   }
   return S;
}

/* update_B_fluxes on the slots of cell c (r part, then z part, then
 * make_edge_adjust), then (first substep) move_cells / clean_pi / calc_dp
 * as k_update does without CT */
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
   const bool z3 = v.ct == 2 && P.Nz > 1;
   /* own face f (the track's first face o) and the face before it */
   auto fm_of = [&](int f, int tr){ return f > v.tr_off[tr] ? f-1 : v.tr_off[tr+1]-1; };
   double P0 = v.Phi[c];
   double S1 = v.Phi[N + c], S2 = v.Phi[2*N + c], S3 = 0.0, S4 = 0.0;
   int f1 = -1, f2 = -1, f3 = -1, f4 = -1, t1 = 0, t2 = 0, t3 = 0, t4 = 0;
   if( j >= 1 ){                           /* inner r face: owned with LRtype 1 */
      t1 = P.trr0 + (j-1) + (P.Nr-1)*k;
      f1 = v.consR[c];
      int fm = fm_of(f1, t1);
      P0 = P0 - X[f1];
      S1 = f1 > v.tr_off[t1] ? (S1 + X[fm]) - X[f1] : (S1 - X[f1]) + X[fm];
   }
   if( j <= P.Nr-2 ){                      /* outer r face: LRtype 0 */
      t2 = P.trr0 + j + (P.Nr-1)*k;
      f2 = v.consL[c];
      int fm = fm_of(f2, t2);
      P0 = P0 + X[f2];
      S2 = f2 > v.tr_off[t2] ? (S2 + X[fm]) - X[f2] : (S2 - X[f2]) + X[fm];
   }
   if( z3 ){
      S3 = v.Phi[3*N + c]; S4 = v.Phi[4*N + c];
      if( k >= 1 ){                        /* lower z face: LRtype 1, R->Phi[3] += X */
         t3 = P.trz0 + j + P.Nr*(k-1);
         f3 = v.consZR[c];
         int fm = fm_of(f3, t3);
         P0 = P0 + X[f3];
         S3 = f3 > v.tr_off[t3] ? (S3 - X[fm]) + X[f3] : (S3 + X[f3]) - X[fm];
      }
      if( k <= P.Nz-2 ){                   /* upper z face: LRtype 0, L->Phi[4] += X */
         t4 = P.trz0 + j + P.Nr*k;
         f4 = v.consZL[c];
         int fm = fm_of(f4, t4);
         P0 = P0 - X[f4];
         S4 = f4 > v.tr_off[t4] ? (S4 - X[fm]) + X[f4] : (S4 + X[f4]) - X[fm];
      }
      /* make_edge_adjust: lines in (k, j) order; add_E_phi takes L -, R +,
       * U -, D + (bfields.c:384-389) */
      const int ln = P.ln0;
      const int W = P.Nr-1;
      if( f2 >= 0 ){                       /* r face (j, j+1) at layer k */
         if( k >= 1 )      S2 = ct_line_terms(v, S2, ln + j + W*(k-1), t2, f2, 2, 3, -1.0);
         if( k <= P.Nz-2 ) S2 = ct_line_terms(v, S2, ln + j + W*k, t2, f2, 0, 1, 1.0);
      }
      if( f1 >= 0 ){                       /* r face (j-1, j) at layer k */
         if( k >= 1 )      S1 = ct_line_terms(v, S1, ln + (j-1) + W*(k-1), t1, f1, 2, 3, -1.0);
         if( k <= P.Nz-2 ) S1 = ct_line_terms(v, S1, ln + (j-1) + W*k, t1, f1, 0, 1, 1.0);
      }
      if( f4 >= 0 ){                       /* z face (k, k+1) of column j */
         if( j >= 1 )      S4 = ct_line_terms(v, S4, ln + (j-1) + W*k, t4, f4, 1, 3, 1.0);
         if( j <= P.Nr-2 ) S4 = ct_line_terms(v, S4, ln + j + W*k, t4, f4, 0, 2, -1.0);
      }
      if( f3 >= 0 ){                       /* z face (k-1, k) of column j */
         if( j >= 1 )      S3 = ct_line_terms(v, S3, ln + (j-1) + W*(k-1), t3, f3, 1, 3, 1.0);
         if( j <= P.Nr-2 ) S3 = ct_line_terms(v, S3, ln + j + W*(k-1), t3, f3, 0, 2, -1.0);
      }
      v.Phi[3*N + c] = S3;
      v.Phi[4*N + c] = S4;
   }
   v.Phi[N + c] = S1;
   v.Phi[2*N + c] = S2;
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
 * the previous face's owner's (r and z tracks) */
template<class R>
__global__ void __launch_bounds__(FB) k_ct_flag(ViewT<R> v){
   int2 b = v.fblk[blockIdx.x];
   int t = b.x;
   if( v.tr_dim[t] == 2 && v.ct != 2 ) return;
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
   if( t >= v.Ntr ) return;
   bool zf = v.tr_dim[t] == 2;
   if( zf && v.ct != 2 ) return;
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
            double *Pf = ct_slot(v, v.Phi, f, zf), *Rf = ct_slot(v, v.RKPhi, f, zf);
            double *Pm = ct_slot(v, v.Phi, fm, zf), *Rm = ct_slot(v, v.RKPhi, fm, zf);
            double *Pp = ct_slot(v, v.Phi, fp, zf), *Rp = ct_slot(v, v.RKPhi, fp, zf);
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

/* B_faces_to_cells type 1 for a real cell (bfields.c:88-309): cons[BRR]
 * (cons[BZZ]) from the fluxes of the cell's r (z) faces -- inner / lower
 * track first, each in face order, slots by the current LRtype -- over their
 * area, cons[BPP] from the two phi faces, with the moved cell's volume */
template<class R>
__device__ void ct_cons_B(const ViewT<R> &v, const DiskParams &P, int a, int c0, int np, int i,
                          int j, int k, double rp, double rm, double zp, double zm, double *cons,
                          int *err){
   const size_t N = v.Ncell;
   int c = c0 + i, cm = c0 + (i == 0 ? np-1 : i-1);
   int I0 = v.I0[a];
   double S = 0.0, T = 0.0;
   /* every face of the cell's run in its inner (lower) track has the cell as
    * R, in its outer (upper) track as L; the other side's cell is read only
    * when that one owns the face */
   auto sum_rin = [&](int f){
      S += v.fLR[f] == 0 ? v.Phi[2*N + v.fL[f]] : v.Phi[N + c];
      T += v.fdA[f];
   };
   auto sum_rout = [&](int f){
      S += v.fLR[f] == 0 ? v.Phi[2*N + c] : v.Phi[N + v.fR[f]];
      T += v.fdA[f];
   };
   if( j >= 1 )      ct_over_runs(v, v.consR, P.trr0 + (j-1) + (P.Nr-1)*k, c0, np, i, I0, sum_rin);
   if( j <= P.Nr-2 ) ct_over_runs(v, v.consL, P.trr0 + j + (P.Nr-1)*k, c0, np, i, I0, sum_rout);
   double x0 = v.ann_rc[a];                          /* centroid_r(rp, rm) */
   double dph = get_dp(v.piph[c], v.piph[cm], P.Pmax, err);
   double dV = dV_of(rp, rm, dph, zp, zm);
   double dA = (rp-rm)*(zp-zm);
   double rfac = 1.0/x0;                                /* bfield_scale_factor(x0, 0) */
   double hr = 1.0, hp = x0;
   cons[BRR] = S * (dV*rfac/(T * hr));
   cons[BPP] = .5*(v.Phi[c]+v.Phi[cm])*dV/(dA * hp);
   if( v.ct == 2 && P.Nz > 1 ){
      double Sz = 0.0, Tz = 0.0;
      auto sum_zin = [&](int f){
         Sz += v.fLR[f] == 0 ? v.Phi[4*N + v.fL[f]] : v.Phi[3*N + c];
         Tz += v.fdA[f];
      };
      auto sum_zout = [&](int f){
         Sz += v.fLR[f] == 0 ? v.Phi[4*N + c] : v.Phi[3*N + v.fR[f]];
         Tz += v.fdA[f];
      };
      if( k >= 1 )      ct_over_runs(v, v.consZR, P.trz0 + j + P.Nr*(k-1), c0, np, i, I0, sum_zin);
      if( k <= P.Nz-2 ) ct_over_runs(v, v.consZL, P.trz0 + j + P.Nr*k, c0, np, i, I0, sum_zout);
      double zfac = 1.0, hz = 1.0;                      /* bfield_scale_factor(x2, 2) */
      cons[BZZ] = Sz * (dV*zfac/(Tz * hz));
   }
}

/* set_B_fields (bfields.c:44-80): each r (z) face's flux prim[BRR] dA
 * (prim[BZZ] dA) at its centre, into its owner's slot */
template<int Q, int NC, class R>
__global__ void __launch_bounds__(FB) k_ct_face_init(ViewT<R> v){
   int2 b = v.fblk[blockIdx.x];
   int t = b.x;
   bool zf = v.tr_dim[t] == 2;
   if( zf && v.ct != 2 ) return;
   int f = v.tr_off[t] + b.y + threadIdx.x;
   if( f >= v.tr_off[t+1] ) return;
   const DiskParams &P = v.dp[v.ann_disk[v.tr_a[t]]];
   int j = v.tr_j[t], k = v.tr_k[t];
   const double *rj = v.rj + P.rj0 + 1;
   const double *zk = v.zk + P.zk0 + 1;
   double prim[Q];
   if( !zf ){
      double x[3] = { .5*(rj[j]+rj[j]), v.fphic[f], 0.5*(zk[k]+zk[k-1]) };
      initial<Q,NC>(P, prim, x);
      *ct_slot(v, v.Phi, f, false) = prim[BRR]*v.fdA[f];
   }else{
      double x[3] = { centroid_r(rj[j], rj[j-1]), v.fphic[f], .5*(zk[k]+zk[k]) };
      initial<Q,NC>(P, prim, x);
      *ct_slot(v, v.Phi, f, true) = prim[BZZ]*v.fdA[f];
   }
}

}  // namespace disco
