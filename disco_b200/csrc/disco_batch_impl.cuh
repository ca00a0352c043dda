/*
 * Internal to the disco_b200 library (not part of the C ABI): the batch
 * object and the templated launch sequences, shared by disco_batch.cu (FP64,
 * built with --fmad=false so it rounds as the reference) and
 * disco_batch_mixed.cu (the FP32 mixed form, built with FMA contraction).
 */
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "disco_b200.h"
#include "disco_kernels.cuh"

using namespace disco;

struct disco_batch {
   int device;
   disco_modules mods;
   int prec;
   int ndisk, Q, NC;
   int timestep_mode;        /* 0 = RK2, 1 = forward Euler */
   int bc_fixed;
   int any_mm3;
   int nq;
   std::vector<disco_params> params;
   /* topology (host) */
   std::vector<int> ann_off, ann_np, ann_disk, ann_j, ann_k;
   std::vector<int> tr_a, tr_b, tr_off, tr_flux, tr_j, tr_k;
   std::vector<double> tr_dxL, tr_dxR;
   std::vector<int2> cblk, fblk;
   std::vector<int> ann_blk0, ann_nblk;
   std::vector<double> rj, zk;
   std::vector<DiskParams> dparams;
   std::vector<int> disk_Nr, disk_Nz, disk_nreal;
   int64_t ncell, nreal;
   /* device: one set of allocations, seen through the view of the precision */
   ViewT<double> vd;
   ViewT<float> vf;
   std::vector<void *> allocs;
   int *d_ann_blk0, *d_ann_nblk;
   double *d_Qrz;
   int *d_err;
   cudaStream_t stream;
   cudaStream_t own_stream;
   std::vector<cudaEvent_t> *tape;       /* non-NULL: record an event after each launch */
   std::vector<const char *> *tape_names;
   cudaGraphExec_t graph;
   int have_cells;
};

static inline unsigned nblk(size_t n, unsigned t){ return (unsigned)((n + t - 1)/t); }

/* after a launch: in kernel-timing mode, an event closing that launch */
static inline void mark(disco_batch *b, const char *name){
   if( !b->tape ) return;
   cudaEvent_t e;
   cudaEventCreate(&e);
   cudaEventRecord(e, b->stream);
   b->tape->push_back(e);
   b->tape_names->push_back(name);
}

template<int Q, int NC, class R>
static void launch_mindt_qt(disco_batch *b, const ViewT<R> &v){
   unsigned nd = nblk(b->ndisk, 64);
   k_mindt_begin<R><<<nd, 64, 0, b->stream>>>(v, b->ndisk);
   k_mindt<Q,NC,R><<<(unsigned)b->cblk.size(), CB, 0, b->stream>>>(v);
   k_mindt_end<R><<<nd, 64, 0, b->stream>>>(v, b->ndisk);
}
template<int Q, int NC, class R>
static void launch_setup_qt(disco_batch *b, const ViewT<R> &v){
   unsigned ncb = (unsigned)b->cblk.size();
   k_setup<Q,NC,R><<<ncb, CB, 0, b->stream>>>(v, b->bc_fixed);
   k_wcell<Q,R><<<ncb, CB, 0, b->stream>>>(v);
   if( b->any_mm3 ) k_wmean_nomove<R><<<nblk(v.Nann, 128), 128, 0, b->stream>>>(v);
}

/* One substep of onestep() (onestep.c:84-229). */
template<int Q, int NC, class R>
static void launch_substep(disco_batch *b, ViewT<R> v, double RK, int first, int last, double dtfac){
   v.dtfac = dtfac;
   cudaStream_t s = b->stream;
   unsigned ncb = (unsigned)b->cblk.size(), nfb = (unsigned)b->fblk.size();
   k_begin<Q,NC,R><<<ncb, CB, 0, s>>>(v, RK, first);                  mark(b, "k_begin");
   if( first && b->any_mm3 ){ k_wmean<R><<<nblk(v.Nann, 128), 128, 0, s>>>(v); mark(b, "k_wmean"); }
   k_I0<R><<<nblk((size_t)v.Nann*32, 128), 128, 0, s>>>(v);           mark(b, "k_I0");
   k_faces<Q,R><<<nfb, FB, 0, s>>>(v, 1);                             mark(b, "k_faces");
   k_gradr<Q,R><<<ncb, CB, 0, s>>>(v);                                mark(b, "k_gradr");
   k_flux_r<Q,NC,R><<<nfb, FB, 0, s>>>(v);                            mark(b, "k_flux_r");
   k_flux_p<Q,NC,R><<<ncb, CB, 0, s>>>(v);                            mark(b, "k_flux_p");
   k_update<Q,NC,R><<<ncb, CB, 0, s>>>(v, first);                     mark(b, "k_update");
   k_c2p<Q,NC,R><<<ncb, CB, 0, s>>>(v, last, b->bc_fixed);            mark(b, "k_c2p");
}

/* timestep() (timestep.c:7-45). */
template<int Q, int NC, class R>
static void launch_step_qt(disco_batch *b, const ViewT<R> &v, int use_next){
   cudaStream_t s = b->stream;
   unsigned nd = nblk(b->ndisk, 64);
   k_disk_begin<R><<<nd, 64, 0, s>>>(v, b->ndisk, use_next);          mark(b, "k_disk_begin");
   if( b->timestep_mode == 1 ){
      launch_substep<Q,NC,R>(b, v, 0.0, 1, 1, 1.0);
      k_disk_mid<R><<<nd, 64, 0, s>>>(v, b->ndisk, 0.0, 1, 1);       mark(b, "k_disk_mid");
   }else{
      launch_substep<Q,NC,R>(b, v, 0.0, 1, 0, 1.0);
      k_disk_mid<R><<<nd, 64, 0, s>>>(v, b->ndisk, 0.0, 1, 1);       mark(b, "k_disk_mid");
      launch_substep<Q,NC,R>(b, v, 0.5, 0, 1, 0.5);
      k_disk_mid<R><<<nd, 64, 0, s>>>(v, b->ndisk, 0.5, 0, 0);       mark(b, "k_disk_mid");
   }
   if( b->nq ){
      k_diag_finish<R><<<nblk(v.Nann, 128), 128, 0, s>>>(v, b->d_Qrz, b->d_ann_blk0, b->d_ann_nblk);
      mark(b, "k_diag_finish");
   }
   k_disk_end<R><<<nd, 64, 0, s>>>(v, b->ndisk);                      mark(b, "k_disk_end");
}

/* Dispatch on the Hydro module: NUM_C 5 (euler) or 8 (mhd), NUM_N 1. */
template<class R>
static void launch_mindt_t(disco_batch *b, const ViewT<R> &v){
   if( b->NC == 8 ) launch_mindt_qt<9,8,R>(b, v); else launch_mindt_qt<6,5,R>(b, v);
}
template<class R>
static void launch_setup_t(disco_batch *b, const ViewT<R> &v){
   if( b->NC == 8 ) launch_setup_qt<9,8,R>(b, v); else launch_setup_qt<6,5,R>(b, v);
}
template<class R>
static void launch_step_t(disco_batch *b, const ViewT<R> &v, int use_next){
   if( b->NC == 8 ) launch_step_qt<9,8,R>(b, v, use_next); else launch_step_qt<6,5,R>(b, v, use_next);
}
template<class R>
static void launch_prim2cons_t(disco_batch *b, const ViewT<R> &v){
   unsigned ncb = (unsigned)b->cblk.size();
   if( b->NC == 8 ) k_prim2cons<9,8,R><<<ncb, CB, 0, b->stream>>>(v);
   else k_prim2cons<6,5,R><<<ncb, CB, 0, b->stream>>>(v);
}

/* FP32 mixed-form launches, defined in disco_batch_mixed.cu */
void mixed_launch_mindt(disco_batch *b);
void mixed_launch_setup(disco_batch *b);
void mixed_launch_step(disco_batch *b, int use_next);
void mixed_launch_prim2cons(disco_batch *b);
void mixed_launch_faces(disco_batch *b);
