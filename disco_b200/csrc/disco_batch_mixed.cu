/*
 * The FP32 mixed form's launches (DISCO_PREC_MIXED): the templated kernels of
 * disco_kernels.cuh instantiated with R = float.  This file is compiled with
 * FMA contraction (--fmad=true); the FP64 path in disco_batch.cu is not.
 */
#define DISCO_MIXED_TU 1
#include "disco_batch_impl.cuh"

void mixed_launch_mindt(disco_batch *b){ launch_mindt_t(b, b->vf); }
void mixed_launch_setup(disco_batch *b){ launch_setup_t(b, b->vf); }
void mixed_launch_restart(disco_batch *b){ launch_restart_t(b, b->vf); }
void mixed_launch_step(disco_batch *b, int use_next){ launch_step_t(b, b->vf, use_next); }
void mixed_launch_report(disco_batch *b){ launch_report_t(b, b->vf); }
void mixed_launch_prim2cons(disco_batch *b){
   launch_prim2cons_t(b, b->vf);
}
void mixed_launch_faces(disco_batch *b){
   k_I0<float><<<nblk((size_t)b->vf.Nann*32, 128), 128, 0, b->stream>>>(b->vf);
   k_faces<6,float><<<(unsigned)b->fblk.size(), FB, 0, b->stream>>>(b->vf, 0);
}
int mixed_prepare_zerograd(disco_batch *b){
   return prepare_zerograd<6,float>(b) || prepare_zerograd<9,float>(b);
}
int mixed_persist_blocks_per_sm(const disco_batch *b){ return persist_blocks_per_sm_t<float>(b); }
