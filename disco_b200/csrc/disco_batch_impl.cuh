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
#include "disco_ct.cuh"
#include "disco_step_persist.cuh"

using namespace disco;

struct disco_batch {
   int device;
   disco_modules mods;
   int prec;
   int ndisk, Q, NC;
   int timestep_mode;        /* 0 = RK2, 1 = forward Euler */
   int bc_fixed;             /* 0 none / zerograd, 1 fixed, 2 fixed3d, 3 polar */
   int any_mm3;
   int any_3d;               /* some disk has Nz > 1: z faces, gradz, z fluxes */
   int bc_zerograd;          /* Boundary/zerograd.c */
   std::vector<int2> zg_pairs;          /* (ghost annulus, source annulus), by layer */
   std::vector<unsigned char> zg_side;  /* per pair: 0 inner r, 1 outer r, 2 lower z, 3 upper z */
   unsigned char *d_zg_side;
   int zg_diode, zg_omk;                /* outflow diode; Omega from initial() in r ghosts */
   int any_visc;                        /* some disk has Use_Viscosity (Euler) */
   int gr;                              /* HYDRO = grmhd2 (FP64, no constrained transport) */
   std::vector<int> zg_off;             /* layer groups: r layers, a window layer, then z layers */
   int2 *d_zg_pairs;
   size_t zg_smem;                      /* dynamic shared memory of k_zerograd */
   std::vector<int2> zpole;             /* 3D CT z-pole annuli (annulus, 0 bottom / 1 top) */
   int2 *d_zpole;
   int nq;
   std::vector<disco_params> params;
   /* topology (host) */
   std::vector<int> ann_off, ann_np, ann_disk, ann_j, ann_k;
   std::vector<int> tr_a, tr_b, tr_off, tr_flux, tr_j, tr_k;
   std::vector<unsigned char> tr_dim;
   std::vector<double> tr_dxL, tr_dxR;
   std::vector<double> tr_r, tr_irf;    /* face centre radius per track, 1/(1/r) */
   std::vector<double> ann_rc;          /* centroid radius per annulus */
   std::vector<int2> cblk, fblk;
   /* the same face blocks in k_faces' order (per layer, the r and z tracks of
    * each annulus together) and the blocks k_flux_t solves per direction */
   std::vector<int2> fblk_rz, fblk_fl[2];
   int2 *d_fblk_rz, *d_fblk_fl[2];
   std::vector<int2> ublk;              /* k_update's blocks: chunks of CB-1 cells */
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
   double *d_stage;          /* Q x ncell FP64, set/get_cells staging (lazy) */
   double *d_rpart, *d_rout; /* report partials per cell block, lines per disk (lazy) */
   double *d_noise;          /* addNoise draws, 4 per cell (lazy) */
   int *d_err;
   cudaStream_t stream;
   cudaStream_t own_stream;
   std::vector<cudaEvent_t> *tape;       /* non-NULL: record an event after each launch */
   std::vector<const char *> *tape_names;
   cudaGraphExec_t graph;
   int have_cells;
   int ct;                   /* constrained transport: the CT_MODE (1, 2) or 0 (FP64 view only) */
   int nfs;                  /* face-flux slots per cell (NUM_FACES: 3 or 5) */
   std::vector<int> line_off;           /* edge lines of 3D CT, offsets into lineX */
   int line_ne;
   /* the one-launch step (disco_step_persist.cuh): schedule in use, whether
    * the batch's modules allow it, its sorted work list, completion
    * counters (zeroed before each launch) and resident grid */
   int sched;
   int persist_ok;
   int4 *d_pitems;
   int pnitems;
   int *d_pcnt;
   size_t pcnt_bytes;
   int pgrid;
   PersistArgs pargs;
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

/* boundary_trans of Boundary/zerograd.c (r layers, then z layers, each
 * layer from the real cells outwards), onestep.c:196-222 and main.c:53-62 */
template<int Q, class R>
static void launch_zerograd(disco_batch *b, const ViewT<R> &v){
   if( !b->bc_zerograd ) return;
   for( size_t g=0 ; g+1<b->zg_off.size() ; ++g ){
      int n = b->zg_off[g+1] - b->zg_off[g];
      if( n > 0 ) k_zerograd<Q,R><<<n, 128, b->zg_smem, b->stream>>>(v, b->d_zg_pairs + b->zg_off[g],
                                                                     b->d_zg_side + b->zg_off[g],
                                                                     b->zg_diode, b->zg_omk);
   }
   mark(b, "k_zerograd");
}
template<int Q, class R>
static int prepare_zerograd(disco_batch *b){
   if( !b->bc_zerograd ) return 0;
   return cudaFuncSetAttribute(k_zerograd<Q,R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)b->zg_smem) != cudaSuccess;
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
   if constexpr ( NC == 8 ){
      if( b->ct ){                  /* set_B_fields (bfields.c:12-86), then cons2prim */
         unsigned nfb = (unsigned)b->fblk.size();
         k_I0<R><<<nblk((size_t)v.Nann*32, 128), 128, 0, b->stream>>>(v);
         k_faces<Q,R><<<nfb, FB, 0, b->stream>>>(v, 0);
         k_ct_face_init<Q,NC,R><<<nfb, FB, 0, b->stream>>>(v);
         k_c2p<Q,NC,R,5,false,false,0><<<ncb, CB, 0, b->stream>>>(v, b->bc_fixed, 0);
      }
   }
   k_wcell<Q,R><<<ncb, CB, 0, b->stream>>>(v);
   if( b->any_mm3 ) k_wmean<R><<<nblk(v.Nann, WM_WARPS), 32*WM_WARPS, 0, b->stream>>>(v, 0);
   launch_zerograd<Q,R>(b, v);                   /* main.c:53-62 */
}

/* setupCells with restart_flag set, then main.c's boundaries (main.c:53-62) */
template<int Q, int NC, class R>
static void launch_restart_qt(disco_batch *b, const ViewT<R> &v){
   unsigned ncb = (unsigned)b->cblk.size();
   k_restart<Q,NC,R><<<ncb, CB, 0, b->stream>>>(v, b->bc_fixed);
   k_wcell<Q,R><<<ncb, CB, 0, b->stream>>>(v);
   if( b->any_mm3 ) k_wmean<R><<<nblk(v.Nann, WM_WARPS), 32*WM_WARPS, 0, b->stream>>>(v, 0);
   launch_zerograd<Q,R>(b, v);
}

/* k_c2p with the Analysis module's number of diagnostics (diag_disk2d 5,
 * diag_euler 8) and, for Euler, the viscous dt limit compiled in only when a
 * disk is viscous */
template<int Q, int NC, class R, int NQD, bool GR>
static void launch_c2p_nq(disco_batch *b, const ViewT<R> &v, int last, int diag){
   unsigned ncb = (unsigned)b->cblk.size();
   if constexpr ( NC == 5 ){
      if( b->any_visc ){
         if( last ) k_c2p<Q,NC,R,NQD,true,false,1><<<ncb, CB, 0, b->stream>>>(v, b->bc_fixed, diag);
         else       k_c2p<Q,NC,R,NQD,true,false,0><<<ncb, CB, 0, b->stream>>>(v, b->bc_fixed, diag);
         return;
      }
   }
   if( last ) k_c2p<Q,NC,R,NQD,false,GR,1><<<ncb, CB, 0, b->stream>>>(v, b->bc_fixed, diag);
   else       k_c2p<Q,NC,R,NQD,false,GR,0><<<ncb, CB, 0, b->stream>>>(v, b->bc_fixed, diag);
}
template<int Q, int NC, class R, bool GR = false>
static void launch_c2p(disco_batch *b, const ViewT<R> &v, int last, int diag){
   if constexpr ( NC == 8 && !GR ){
      if( b->nq == 18 ){ launch_c2p_nq<Q,NC,R,18,false>(b, v, last, diag); return; }
   }
   if( b->nq == 8 ) launch_c2p_nq<Q,NC,R,8,GR>(b, v, last, diag);
   else launch_c2p_nq<Q,NC,R,5,GR>(b, v, last, diag);
}
template<int Q, int NC, int DIM, class R, bool GR = false>
static void launch_flux_t(disco_batch *b, const ViewT<R> &v0){
   /* only the blocks of this direction's tracks with trans_flux faces */
   unsigned nfb = (unsigned)b->fblk_fl[DIM-1].size();
   if( nfb == 0 ) return;
   ViewT<R> v = v0; v.fblk = b->d_fblk_fl[DIM-1];
   if constexpr ( NC == 5 ){
      if( b->any_visc ){ k_flux_t<Q,NC,DIM,R,true><<<nfb, FB, 0, b->stream>>>(v); return; }
   }
   k_flux_t<Q,NC,DIM,R,false,GR><<<nfb, FB, 0, b->stream>>>(v);
}

/* One substep of onestep() (onestep.c:84-229); GR: the grmhd2 module. */
template<int Q, int NC, class R, bool GR = false>
static void launch_substep(disco_batch *b, ViewT<R> v, double RK, int first, int last, double dtfac){
   v.dtfac = dtfac;
   /* RK2: the first substep keeps the faces the previous step's second
    * substep built from the same piph; that substep marks them valid */
   v.topo_reuse = first && b->timestep_mode == 0;
   v.topo_set = !first;
   v.move_c2p = first && !b->ct;
   cudaStream_t s = b->stream;
   unsigned ncb = (unsigned)b->cblk.size(), nfb = (unsigned)b->fblk.size();
   k_begin<Q,NC,R,GR><<<ncb, CB, 0, s>>>(v, RK, first);               mark(b, "k_begin");
   if( first && b->any_mm3 ){ k_wmean<R><<<nblk(v.Nann, WM_WARPS), 32*WM_WARPS, 0, s>>>(v, 1); mark(b, "k_wmean"); }
   k_I0<R><<<nblk((size_t)v.Nann*32, 128), 128, 0, s>>>(v);           mark(b, "k_I0");
   {  /* the same blocks in the order that keeps an annulus's three tracks together */
      ViewT<R> vf = v; vf.fblk = b->d_fblk_rz;
      k_faces<Q,R><<<nfb, FB, 0, s>>>(vf, 1);                          mark(b, "k_faces");
   }
   if( b->any_3d ){ k_grad_rz<Q,R><<<ncb, CB, 0, s>>>(v);             mark(b, "k_grad"); }
   else{ k_grad<Q,1,R><<<ncb, CB, 0, s>>>(v);                         mark(b, "k_gradr"); }
   launch_flux_t<Q,NC,1,R,GR>(b, v);                                  mark(b, "k_flux_r");
   if( b->any_3d ){ launch_flux_t<Q,NC,2,R,GR>(b, v);                 mark(b, "k_flux_z"); }
   bool upd_visc = false;
   if constexpr ( NC == 5 ) upd_visc = b->any_visc;
   if( upd_visc ){
      if constexpr ( NC == 5 ) k_update<Q,NC,R,true><<<(unsigned)b->ublk.size(), CB, 0, s>>>(v, first);
   }else{
      k_update<Q,NC,R,false,GR><<<(unsigned)b->ublk.size(), CB, 0, s>>>(v, first);
   }
   mark(b, "k_update");
   if constexpr ( NC == 8 ){
      if( b->ct ){                  /* onestep.c:140-146 and 160-167 */
         k_ct_edges<R><<<ncb, CB, 0, s>>>(v);                           mark(b, "k_ct_edges");
         ViewT<R> vrz = v; vrz.fblk = b->d_fblk_rz;      /* per-face kernels, k_faces' order */
         k_ct_faces<R><<<nfb, FB, 0, s>>>(vrz);                         mark(b, "k_ct_faces");
         if( !b->zpole.empty() ){
            k_ct_zpole<R><<<(unsigned)b->zpole.size(), CB, 0, s>>>(v, b->d_zpole); mark(b, "k_ct_zpole");
         }
         if( b->ct == 2 && b->any_3d ){
            k_ct_line<R><<<ncb, CB, 0, s>>>(v);                         mark(b, "k_ct_line");
         }
         k_ct_update<R><<<ncb, CB, 0, s>>>(v, first);                   mark(b, "k_ct_update");
         if( first ){
            k_ct_flag<R><<<nfb, FB, 0, s>>>(vrz);                       mark(b, "k_ct_flag");
            k_ct_flip<R><<<nblk((size_t)v.Ntr*32, 128), 128, 0, s>>>(v); mark(b, "k_ct_flip");
         }
      }
   }
   launch_c2p<Q,NC,R,GR>(b, v, last, !b->bc_zerograd);                mark(b, "k_c2p");
   launch_zerograd<Q,R>(b, v);
   if( last && b->nq && b->bc_zerograd ){
      bool mri = false;
      if constexpr ( Q == 9 ) mri = b->nq == 18;
      if( mri ){
         if constexpr ( Q == 9 ) k_diag_part<Q,R,18><<<ncb, CB, 0, s>>>(v);
      }else if( b->nq == 8 ) k_diag_part<Q,R,8><<<ncb, CB, 0, s>>>(v);
      else k_diag_part<Q,R,5><<<ncb, CB, 0, s>>>(v);
      mark(b, "k_diag_part");
   }
}

/* timestep() as one cooperative launch of k_step (the counters zeroed first) */
template<int Q, int NC, class R, int NQD>
static void launch_persist_nq(disco_batch *b, const ViewT<R> &v, int use_next){
   PersistArgs pa = b->pargs;
   pa.use_next = use_next;
   cudaMemsetAsync(b->d_pcnt, 0, b->pcnt_bytes, b->stream);
   cudaLaunchConfig_t cfg = {};
   cfg.gridDim = dim3((unsigned)b->pgrid);
   cfg.blockDim = dim3(CB);
   cfg.dynamicSmemBytes = 0;
   cfg.stream = b->stream;
   cudaLaunchAttribute at[1];
   at[0].id = cudaLaunchAttributeCooperative;
   at[0].val.cooperative = 1;
   cfg.attrs = at;
   cfg.numAttrs = 1;
   cudaLaunchKernelEx(&cfg, k_step<Q,NC,R,NQD>, v, pa);
   mark(b, "k_step");
}
template<int Q, int NC, class R>
static void launch_persist(disco_batch *b, const ViewT<R> &v, int use_next){
   if constexpr ( NC == 8 ){
      if( b->nq == 18 ){ launch_persist_nq<Q,NC,R,18>(b, v, use_next); return; }
   }
   if( b->nq == 8 ) launch_persist_nq<Q,NC,R,8>(b, v, use_next);
   else launch_persist_nq<Q,NC,R,5>(b, v, use_next);
}
/* resident k_step CTAs per SM for the batch's instantiation */
template<int Q, int NC, class R, int NQD>
static int persist_occ_nq(){
   int nb = 0;
   if( cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_step<Q,NC,R,NQD>, CB, 0) != cudaSuccess ) return 0;
   return nb;
}
template<class R>
static int persist_blocks_per_sm_t(const disco_batch *b){
   if( b->NC == 8 ) return b->nq == 18 ? persist_occ_nq<9,8,R,18>() : b->nq == 8 ? persist_occ_nq<9,8,R,8>()
                                                                                  : persist_occ_nq<9,8,R,5>();
   return b->nq == 8 ? persist_occ_nq<6,5,R,8>() : persist_occ_nq<6,5,R,5>();
}

/* timestep() (timestep.c:7-45). */
template<int Q, int NC, class R, bool GR = false>
static void launch_step_qt(disco_batch *b, const ViewT<R> &v, int use_next){
   if( b->sched == DISCO_SCHED_PERSISTENT ){ launch_persist<Q,NC,R>(b, v, use_next); return; }
   cudaStream_t s = b->stream;
   unsigned nd = nblk(b->ndisk, 64);
   k_disk_begin<R><<<nd, 64, 0, s>>>(v, b->ndisk, use_next);          mark(b, "k_disk_begin");
   if( b->timestep_mode == 1 ){
      launch_substep<Q,NC,R,GR>(b, v, 0.0, 1, 1, 1.0);
      k_disk_mid<R><<<nd, 64, 0, s>>>(v, b->ndisk, 0.0, 1, 1);       mark(b, "k_disk_mid");
   }else{
      launch_substep<Q,NC,R,GR>(b, v, 0.0, 1, 0, 1.0);
      k_disk_mid<R><<<nd, 64, 0, s>>>(v, b->ndisk, 0.0, 1, 1);       mark(b, "k_disk_mid");
      launch_substep<Q,NC,R,GR>(b, v, 0.5, 0, 1, 0.5);
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
static void launch_restart_t(disco_batch *b, const ViewT<R> &v){
   if( b->NC == 8 ) launch_restart_qt<9,8,R>(b, v); else launch_restart_qt<6,5,R>(b, v);
}
template<class R>
static void launch_step_t(disco_batch *b, const ViewT<R> &v, int use_next){
   if constexpr ( sizeof(R) == sizeof(double) ){
      if( b->gr ){ launch_step_qt<9,8,R,true>(b, v, use_next); return; }
   }
   if( b->NC == 8 ) launch_step_qt<9,8,R>(b, v, use_next); else launch_step_qt<6,5,R>(b, v, use_next);
}
template<class R>
static void launch_prim2cons_t(disco_batch *b, const ViewT<R> &v){
   unsigned ncb = (unsigned)b->cblk.size();
   if( b->NC == 8 ) k_prim2cons<9,8,R><<<ncb, CB, 0, b->stream>>>(v);
   else k_prim2cons<6,5,R><<<ncb, CB, 0, b->stream>>>(v);
}

/* report() (report.c:7-202) on the device: per-block partials, then per-disk lines */
template<class R>
static void launch_report_t(disco_batch *b, const ViewT<R> &v){
   unsigned ncb = (unsigned)b->cblk.size();
   if( b->NC == 8 ) k_report_part<9,8,R><<<ncb, CB, 0, b->stream>>>(v, b->d_rpart);
   else k_report_part<6,5,R><<<ncb, CB, 0, b->stream>>>(v, b->d_rpart);
   k_report_finish<R><<<nblk(b->ndisk, 64), 64, 0, b->stream>>>(v, b->d_rpart, b->d_ann_blk0,
                                                                b->d_ann_nblk, b->d_rout, b->ndisk);
}

/* FP32 mixed-form launches, defined in disco_batch_mixed.cu */
void mixed_launch_report(disco_batch *b);
void mixed_launch_mindt(disco_batch *b);
void mixed_launch_setup(disco_batch *b);
void mixed_launch_restart(disco_batch *b);
void mixed_launch_step(disco_batch *b, int use_next);
void mixed_launch_prim2cons(disco_batch *b);
void mixed_launch_faces(disco_batch *b);
int mixed_prepare_zerograd(disco_batch *b);
int mixed_persist_blocks_per_sm(const disco_batch *b);

/* host <-> device copy on the batch's stream, completed on return
 * (disco_batch.cu; used by the writers of disco_output.cu) */
cudaError_t batch_xfer(const disco_batch *b, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind);
