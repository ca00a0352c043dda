/*
 * One RK2 timestep of a whole batch as ONE persistent launch (the RK
 * substeps' six kernel passes and the per-disk bookkeeping of
 * disco_batch_impl.cuh's launch_step_qt, fused by a dataflow schedule).
 *
 * The work is the same blocks the multi-kernel path launches -- k_begin's,
 * k_I0's, k_faces', k_grad's, k_flux_t's, k_update's and k_c2p's block
 * tables for both substeps, plus per-disk items for timestep()'s start, the
 * planet update between the substeps (onestep.c:163-166) and the end
 * (dt of the next step) -- and the same device bodies run them
 * (disco_kernels.cuh), so the arithmetic, and with it every result, is the
 * multi-kernel path's bit for bit.  What changes is when a block may run:
 * instead of a kernel boundary after each pass, a block waits only for the
 * blocks it reads from, through completion counters per annulus and per
 * track (per substep), e.g. the faces of track (A, B) once k_begin's blocks
 * of annuli A and B and their I0 are done; the gradients of annulus a once
 * the faces of its two tracks are; the update of a once the fluxes of its
 * two tracks are.  Every block's inputs are thus complete and no block
 * overwrites what a block that has not run yet still reads (the write-after-
 * read cases are closed by the same chains: e.g. k_c2p moves annulus a only
 * after its update, which waited for the fluxes of both its tracks, which
 * waited for both gradients, ...).
 *
 * Schedule.  The host sorts the items into one list in which every item's
 * dependencies come earlier: a wavefront in r over all disks at once (each
 * disk's radius normalised by its Nr), cut into tiles of about 8 grids'
 * worth of items, and inside a tile by substep and stage, so that what a
 * stage writes is read by the next stage about one grid's worth of items
 * later, while it is still in L2.  CTA g of the grid runs items g, g+G,
 * g+2G, ... in that order.  The
 * launch is cooperative, so all G CTAs are resident: the smallest item not
 * yet done always has its dependencies done and its CTA free to run it, so
 * the schedule cannot deadlock.  Every wait is bounded (PERSIST_SPIN_CAP
 * polls); a wait that runs out sets ERRF_TIMEOUT and a global abort word
 * that makes every other CTA leave at its next wait.
 *
 * Scope: hydro and MHD without constrained transport, 2D disks (Nz = 1),
 * RK2, fixed / polar or no boundaries, no Mesh_Motion 3, no viscosity; the
 * host falls back to the multi-kernel path otherwise.
 */
#pragma once
#include "disco_kernels.cuh"

namespace disco {

enum { PS_DBEGIN = 0, PS_BEGIN, PS_I0, PS_FACES, PS_GRAD, PS_FLUX, PS_UPDATE, PS_C2P,
       PS_DMID, PS_DIAGFIN, PS_DTAIL };

/* polls of a completion counter before a wait gives up (each poll sleeps
 * about 100 ns, so about 1.7 s; a step takes milliseconds) */
#define PERSIST_SPIN_CAP (1 << 24)

struct PersistArgs {
   const int4 *items;     /* .x stage | substep << 4, .y block index (or first annulus / disk), .z count */
   int nitems;
   int *cnt;              /* completion counters, zeroed before each launch */
   int *ctl;              /* ctl[0] abort word, ctl[1] CTAs that have left (zeroed with cnt) */
   /* offsets into cnt, per substep: per annulus (begin, I0, grad, update,
    * c2p), per track (faces, flux), per disk (c2p blocks done) */
   int o_begin[2], o_I0[2], o_faces[2], o_grad[2], o_flux[2], o_upd[2], o_c2p[2], o_c2pd[2];
   int o_d0, o_d1;        /* per disk: timestep() start done, planet update after substep 1 done */
   const int *nc;         /* per annulus: k_begin / k_grad / k_c2p blocks (cblk) */
   const int *nu;         /* per annulus: k_update blocks (ublk) */
   const int *nf;         /* per track: k_faces / k_flux_t blocks (fblk) */
   const int *ndc;        /* per disk: cblk blocks */
   double *Qrz;
   const int *ann_blk0, *ann_nblk;
   int bc, diag, use_next;
};

__device__ __forceinline__ int ld_acquire(const int *p){
   int x;
   asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
   return x;
}

__device__ __forceinline__ int ld_relaxed(const int *p){
   int x;
   asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(x) : "l"(p) : "memory");
   return x;
}

/* Bounded wait until *p >= target; false on time-out or abort. */
__device__ __forceinline__ bool wait_ge(const int *p, int target, const int *abortp){
   if( ld_acquire(p) >= target ) return true;
   for( int it=0 ; it<PERSIST_SPIN_CAP ; ++it ){
      __nanosleep(100);
      if( ld_acquire(p) >= target ) return true;
      if( (it & 63) == 63 && ld_acquire(abortp) ) return false;
   }
   return false;
}

/* Up to four counters at once: one round of independent loads first (the
 * usual case, every input already done), the bounded waits only for what is
 * not; then an acquire fence for the reads that follow. */
__device__ __forceinline__ bool wait4(const int *const *p, const int *t, int n, const int *abortp){
   int x[4];
#pragma unroll
   for( int m=0 ; m<4 ; ++m ) x[m] = m < n ? ld_relaxed(p[m]) : 0;
   bool ok = true;
#pragma unroll
   for( int m=0 ; m<4 ; ++m ) if( m < n && x[m] < t[m] ) ok = false;
   if( !ok ){
      for( int m=0 ; m<n ; ++m ) if( !wait_ge(p[m], t[m], abortp) ) return false;
   }
   asm volatile("fence.acq_rel.gpu;" ::: "memory");
   return true;
}

/* counter += 1 with release semantics (orders the CTA's prior writes, made
 * visible to thread 0 by the barrier before it) */
__device__ __forceinline__ void red_release(int *p){
   asm volatile("red.release.gpu.global.add.s32 [%0], 1;" :: "l"(p) : "memory");
}

/* the r-tracks inside / outside annulus a (-1: none) */
template<class R>
__device__ __forceinline__ int track_in(const ViewT<R> &v, int a){
   const DiskParams &P = v.dp[v.ann_disk[a]];
   int j = v.ann_j[a], k = v.ann_k[a];
   return j >= 1 ? P.trr0 + (j-1) + (P.Nr-1)*k : -1;
}
template<class R>
__device__ __forceinline__ int track_out(const ViewT<R> &v, int a){
   const DiskParams &P = v.dp[v.ann_disk[a]];
   int j = v.ann_j[a], k = v.ann_k[a];
   return j <= P.Nr-2 ? P.trr0 + j + (P.Nr-1)*k : -1;
}

/* Thread 0: wait for the item's inputs. */
template<class R>
__device__ bool persist_wait(const ViewT<R> &v, const PersistArgs &pa, int stage, int sub, int x, int n){
   const int *ab = pa.ctl;
   const int *C = pa.cnt;
   const int *p[4];
   int t[4], m = 0;
   auto need = [&](int off, int idx, int target){ p[m] = C + off + idx; t[m] = target; ++m; };
   switch( stage ){
   case PS_BEGIN: {
      int a = v.cblk[x].x, d = v.ann_disk[a];
      if( sub == 0 ) need(pa.o_d0, d, 1);
      else { need(pa.o_c2p[0], a, pa.nc[a]); need(pa.o_d1, d, 1); }
      break;
   }
   case PS_I0:
      if( sub == 0 ) return true;
      for( int a=x ; a<x+n ; ++a ) need(pa.o_c2p[0], a, pa.nc[a]);
      break;
   case PS_FACES: {
      int tr = v.fblk[x].x, A = v.tr_a[tr], B = v.tr_b[tr];
      need(pa.o_begin[sub], A, pa.nc[A]); need(pa.o_begin[sub], B, pa.nc[B]);
      need(pa.o_I0[sub], A, 1); need(pa.o_I0[sub], B, 1);
      break;
   }
   case PS_GRAD: {
      int a = v.cblk[x].x, ti = track_in(v, a), to = track_out(v, a);
      if( ti >= 0 ) need(pa.o_faces[sub], ti, pa.nf[ti]);
      if( to >= 0 ) need(pa.o_faces[sub], to, pa.nf[to]);
      break;
   }
   case PS_FLUX: {
      int tr = v.fblk[x].x, A = v.tr_a[tr], B = v.tr_b[tr];
      need(pa.o_grad[sub], A, pa.nc[A]); need(pa.o_grad[sub], B, pa.nc[B]);
      break;
   }
   case PS_UPDATE: {
      int a = v.ublk[x].x, ti = track_in(v, a), to = track_out(v, a);
      if( ti >= 0 ) need(pa.o_flux[sub], ti, pa.nf[ti]);
      if( to >= 0 ) need(pa.o_flux[sub], to, pa.nf[to]);
      break;
   }
   case PS_C2P: {
      int a = v.cblk[x].x;
      need(pa.o_upd[sub], a, pa.nu[a]);
      break;
   }
   case PS_DMID:
      need(pa.o_c2pd[0], x, pa.ndc[x]);
      break;
   case PS_DIAGFIN:
      for( int a=x ; a<x+n ; ++a ) if( !wait_ge(C + pa.o_c2p[1] + a, pa.nc[a], ab) ) return false;
      asm volatile("fence.acq_rel.gpu;" ::: "memory");
      return true;
   case PS_DTAIL:
      need(pa.o_c2pd[1], x, pa.ndc[x]);
      break;
   default:
      return true;
   }
   return m == 0 || wait4(p, t, m, ab);
}

/* Thread 0, after the block's barrier: mark the item done (release). */
template<class R>
__device__ void persist_signal(const ViewT<R> &v, const PersistArgs &pa, int stage, int sub, int x, int n){
   int *C = pa.cnt;
   switch( stage ){
   case PS_DBEGIN: red_release(C + pa.o_d0 + x); break;
   case PS_BEGIN:  red_release(C + pa.o_begin[sub] + v.cblk[x].x); break;
   case PS_I0:     for( int a=x ; a<x+n ; ++a ) red_release(C + pa.o_I0[sub] + a); break;
   case PS_FACES:  red_release(C + pa.o_faces[sub] + v.fblk[x].x); break;
   case PS_GRAD:   red_release(C + pa.o_grad[sub] + v.cblk[x].x); break;
   case PS_FLUX:   red_release(C + pa.o_flux[sub] + v.fblk[x].x); break;
   case PS_UPDATE: red_release(C + pa.o_upd[sub] + v.ublk[x].x); break;
   case PS_C2P: {
      int a = v.cblk[x].x;
      red_release(C + pa.o_c2p[sub] + a);
      red_release(C + pa.o_c2pd[sub] + v.ann_disk[a]);
      break;
   }
   case PS_DMID:   red_release(C + pa.o_d1 + x); break;
   default: break;
   }
}

/* All threads: run the item (the multi-kernel path's block bodies, with the
 * substep's flags: RK2, the first substep keeping the face topology, the
 * move in k_c2p). */
template<int Q, int NC, class R, int NQD>
__device__ __forceinline__ void persist_run(const ViewT<R> &v, const PersistArgs &pa, int stage, int sub,
                                            int x, int n){
   const int tid = threadIdx.x;
   const double dtfac = sub ? 0.5 : 1.0;
   switch( stage ){
   case PS_DBEGIN:  if( tid == 0 ) disk_begin_body<R>(v, x, pa.use_next); break;
   case PS_BEGIN:   begin_body<Q,NC,R>(v, sub ? 0.5 : 0.0, !sub, x); break;
   case PS_I0:      if( (tid >> 5) < n ) I0_body<R>(v, !sub, x + (tid >> 5), tid & 31); break;
   case PS_FACES:   faces_body<Q,R>(v, 1, !sub, x); break;
   case PS_GRAD:    grad_body<Q,1,R>(v, x); break;
   case PS_FLUX:    flux_body<Q,NC,1,R,false>(v, dtfac, x); break;
   case PS_UPDATE:  update_body<Q,NC,R,false>(v, !sub, dtfac, x); break;
   case PS_C2P:     c2p_body<Q,NC,R,NQD,false>(v, sub, pa.bc, pa.diag, !sub, 0, x); break;
   case PS_DMID:    if( tid == 0 ) disk_mid_body<R>(v, x, 0.0, 1, 1); break;
   case PS_DIAGFIN: if( tid < n ) diag_finish_body<R>(v, pa.Qrz, pa.ann_blk0, pa.ann_nblk, x + tid); break;
   case PS_DTAIL:
      if( tid == 0 ){ disk_mid_body<R>(v, x, 0.5, 0, 0); disk_end_body<R>(v, x); }
      break;
   default: break;
   }
}

#ifndef MB_PERSIST
#define MB_PERSIST 8
#endif

template<int Q, int NC, class R, int NQD>
__global__ void __launch_bounds__(CB, Q > 6 ? MB_MHD : MB_PERSIST) k_step(ViewT<R> v, PersistArgs pa){
   __shared__ int s_go;
   const int tid = threadIdx.x;
   for( int it=blockIdx.x ; it<pa.nitems ; it+=gridDim.x ){
      const int4 w = pa.items[it];
      const int stage = w.x & 15, sub = w.x >> 4;
      if( tid == 0 ){
         int ok = persist_wait<R>(v, pa, stage, sub, w.y, w.z) ? 1 : 0;
         if( !ok ){
            atomicExch(pa.ctl, 1);
            atomicOr(v.err, ERRF_TIMEOUT);
         }
         s_go = ok;
      }
      __syncthreads();
      if( !s_go ) break;
      persist_run<Q,NC,R,NQD>(v, pa, stage, sub, w.y, w.z);
      __syncthreads();
      if( tid == 0 ){
         __threadfence();        /* the block's writes, ordered by the barrier, before the counter */
         persist_signal<R>(v, pa, stage, sub, w.y, w.z);
      }
   }
   /* the last CTA out marks the face lists as built from the current piph
    * (the second substep rebuilt them), as k_c2p's topo_set does */
   if( tid == 0 ){
      __threadfence();
      if( atomicAdd(pa.ctl + 1, 1) == (int)gridDim.x - 1 && ld_acquire(pa.ctl) == 0 ) *v.topo = 1;
   }
}

} /* namespace disco */
