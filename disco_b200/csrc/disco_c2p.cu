/*
 * GRMHD cons -> prim on the GPU: the batched form of calc_prim's per-cell
 * cons2prim (misc.c:290-325 -> Hydro/grmhd2.c:253-270, Noble-2D Newton
 * :1096-1313), its inverse prim2cons (:88-180), and the learned initial
 * guess with its training kernels.  C ABI in include/disco_c2p.h.
 *
 * Solve: one thread per cell, FP64 throughout, compiled with --fmad=false so
 * the Schwarzschild-KS path rounds exactly as the reference (only + - * /
 * sqrt, all IEEE on both sides).  The kernel is persistent (a grid of
 * resident blocks striding over the cells) so that the network's weights
 * are staged into shared memory once per block.
 *
 * Network: 8 -> 64 -> 64 -> 2, tanh, BF16 weights and activations as
 * tensor-core operands with FP32 accumulation (mma.sync m16n8k16; a warp
 * evaluates its 32 cells as two 16-row tiles, the FP32 accumulator fragment
 * of one layer becoming, packed to BF16, the A fragment of the next).
 * Training: by default the forward and backward contractions of each
 * 128-sample group on the tensor cores through tcgen05.mma with tensor-
 * memory accumulators (mlp_tcgen05.cuh); or the same forward and the
 * backward on the FP32 CUDA cores over 128-sample groups held in shared
 * memory (per-thread register accumulators for dW, one atomic per weight
 * per block).  Then Adam on FP32 master weights, which writes the BF16
 * copy the kernels read.
 */
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <string>
#include <vector>
#include "disco_b200.h"
#include "disco_c2p.h"
#include "grmhd.cuh"
#include "gr_torus.h"

using namespace disco;

static_assert(MLP_NPARAM == DISCO_MLP_NPARAM && MLP_NNORM == DISCO_MLP_NNORM, "network size");
static_assert(sizeof(disco_gr_torus) == sizeof(gr_torus_par), "torus struct");

/* Network image as the kernels read it (straight into shared memory).
 * B operands are W[out][in] rows, contiguous in `in` (the mma "col" B);
 * W2/W3 rows are padded to 72 so that the fragment loads of a warp hit 32
 * distinct banks; W3 has 8 rows, rows 2..7 zero (N = 8 tile). */
struct MlpPacked {
   __nv_bfloat16 W1[MLP_H][8];
   __nv_bfloat16 W2[MLP_H][72];
   __nv_bfloat16 W3[8][72];
   float b1[MLP_H], b2[MLP_H], b3[8];
   float norm[MLP_NNORM];
};
static_assert(sizeof(MlpPacked) % 16 == 0, "packed image is copied as int4");

/* Parameter offsets in the flat layout W1 b1 W2 b2 W3 b3 */
#define OFF_W1 0
#define OFF_B1 (OFF_W1 + MLP_NW1)
#define OFF_W2 (OFF_B1 + MLP_H)
#define OFF_B2 (OFF_W2 + MLP_NW2)
#define OFF_W3 (OFF_B2 + MLP_H)
#define OFF_B3 (OFF_W3 + MLP_NW3)

struct StatsDev {
   unsigned long long ncell, iters_sum;
   unsigned int iters_max, n_fallback, n_fail, pad;
   unsigned long long hist[64];
};
static_assert(sizeof(StatsDev) == sizeof(disco_gr_stats), "stats layout");

/* ------------------------------------------------------------------ */
/* tensor-core pieces                                                  */

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi){
   __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
   return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void mma_bf16_16816(float *c, uint32_t a0, uint32_t a1, uint32_t a2,
                                               uint32_t a3, uint32_t b0, uint32_t b1){
   asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16 *p){
   return *reinterpret_cast<const uint32_t*>(p);
}

/* tanh: the training kernels use tanhf, whose error is far below the BF16
 * rounding of the activations that follows, so their gradients can be
 * checked against a double-precision restatement; inference uses the
 * hardware approximation tanh.approx.f32 (relative error about 2^-11, also
 * below that rounding).  The packed tanh.approx.bf16x2 was measured no
 * faster here and costs the guess accuracy (its input is rounded first). */
template<bool FAST>
__device__ __forceinline__ float act(float x){
   if( FAST ){
      float y;
      asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
      return y;
   }
   return tanhf(x);
}

/* Forward of one 16-row tile (rows mt*16 .. mt*16+15 of the warp's 32) of
 * normalised BF16 inputs Xs[32][8].  Writes the two outputs of each row to
 * Y[32][2]; with STORE, also the FP32 tanh activations of both hidden layers
 * to H1/H2 (row stride ld). */
template<bool STORE, bool FAST>
__device__ __forceinline__ void mlp_fwd_tile(const MlpPacked &W, const __nv_bfloat16 *Xs, int mt,
                                             int lane, float *H1, float *H2, int ld, float *Y){
   const int g = lane >> 2, t = lane & 3;
   const int r0 = mt*16 + g, r1 = r0 + 8;
   const uint32_t xa0 = ld32(Xs + r0*8 + 2*t);
   const uint32_t xa1 = ld32(Xs + r1*8 + 2*t);
   uint32_t A[4][4];
#pragma unroll
   for( int nt=0 ; nt<8 ; ++nt ){
      const int col = nt*8 + 2*t;
      float c[4] = {W.b1[col], W.b1[col+1], W.b1[col], W.b1[col+1]};
      mma_bf16_16816(c, xa0, xa1, 0u, 0u, ld32(&W.W1[nt*8+g][2*t]), 0u);
      const float h0 = act<FAST>(c[0]), h1 = act<FAST>(c[1]), h2 = act<FAST>(c[2]), h3 = act<FAST>(c[3]);
      if( STORE ){
         H1[r0*ld + col] = h0; H1[r0*ld + col + 1] = h1;
         H1[r1*ld + col] = h2; H1[r1*ld + col + 1] = h3;
      }
      A[nt >> 1][2*(nt & 1)]     = pack_bf16(h0, h1);
      A[nt >> 1][2*(nt & 1) + 1] = pack_bf16(h2, h3);
   }
   uint32_t A3[4][4];
#pragma unroll
   for( int nt=0 ; nt<8 ; ++nt ){
      const int col = nt*8 + 2*t;
      float c[4] = {W.b2[col], W.b2[col+1], W.b2[col], W.b2[col+1]};
#pragma unroll
      for( int kt=0 ; kt<4 ; ++kt )
         mma_bf16_16816(c, A[kt][0], A[kt][1], A[kt][2], A[kt][3],
                        ld32(&W.W2[nt*8+g][kt*16 + 2*t]), ld32(&W.W2[nt*8+g][kt*16 + 8 + 2*t]));
      const float h0 = act<FAST>(c[0]), h1 = act<FAST>(c[1]), h2 = act<FAST>(c[2]), h3 = act<FAST>(c[3]);
      if( STORE ){
         H2[r0*ld + col] = h0; H2[r0*ld + col + 1] = h1;
         H2[r1*ld + col] = h2; H2[r1*ld + col + 1] = h3;
      }
      A3[nt >> 1][2*(nt & 1)]     = pack_bf16(h0, h1);
      A3[nt >> 1][2*(nt & 1) + 1] = pack_bf16(h2, h3);
   }
   float c[4] = {W.b3[2*t], W.b3[2*t+1], W.b3[2*t], W.b3[2*t+1]};
#pragma unroll
   for( int kt=0 ; kt<4 ; ++kt )
      mma_bf16_16816(c, A3[kt][0], A3[kt][1], A3[kt][2], A3[kt][3],
                     ld32(&W.W3[g][kt*16 + 2*t]), ld32(&W.W3[g][kt*16 + 8 + 2*t]));
   if( t == 0 ){
      Y[2*r0] = c[0]; Y[2*r0 + 1] = c[1];
      Y[2*r1] = c[2]; Y[2*r1 + 1] = c[3];
   }
}

__device__ __forceinline__ void copy_packed(MlpPacked *dst, const MlpPacked *src){
   const int4 *s = reinterpret_cast<const int4*>(src);
   int4 *d = reinterpret_cast<int4*>(dst);
   for( int k=threadIdx.x ; k<(int)(sizeof(MlpPacked)/16) ; k+=blockDim.x ) d[k] = s[k];
}

/* ------------------------------------------------------------------ */
/* state kernels                                                       */

__global__ void k_gr_grid(int Nr, int Nz, int Np, double rmin, double rmax, double zmin,
                          double zmax, int log_r, long n, double *x){
   long c = (long)blockIdx.x*blockDim.x + threadIdx.x;
   if( c >= n ) return;
   int i = (int)(c % Np);
   long jk = c / Np;
   int j = (int)(jk % Nr), k = (int)(jk / Nr);
   double rm, rp;
   if( log_r ){
      double L = log(rmax/rmin);
      rm = rmin*exp(L*(double)j/Nr);
      rp = rmin*exp(L*(double)(j+1)/Nr);
   }else{
      rm = rmin + (rmax-rmin)*(double)j/Nr;
      rp = rmin + (rmax-rmin)*(double)(j+1)/Nr;
   }
   double zm = zmin + (zmax-zmin)*(double)k/Nz, zp = zmin + (zmax-zmin)*(double)(k+1)/Nz;
   x[c]       = 2.0*(rp*rp + rp*rm + rm*rm)/(3.0*(rp + rm));
   x[n + c]   = ((double)i + 0.5)*(2.0*M_PI/(double)Np);
   x[2*n + c] = 0.5*(zm + zp);
}

__global__ void k_gr_torus(gr_torus_par tp, long n, const double *x, double *prim){
   long c = (long)blockIdx.x*blockDim.x + threadIdx.x;
   if( c >= n ) return;
   double xx[3] = {x[c], x[n+c], x[2*n+c]}, p[9];
   gr_torus_prim(&tp, xx, (uint64_t)c, p);
   for( int q=0 ; q<9 ; ++q ) prim[q*n + c] = p[q];
}

__global__ void k_gr_perturb(long n, const double *prim, double *out, uint64_t seed, double eps){
   long c = (long)blockIdx.x*blockDim.x + threadIdx.x;
   if( c >= n ) return;
   double p[9], o[9];
   for( int q=0 ; q<9 ; ++q ) p[q] = prim[q*n + c];
   gr_perturb(p, o, seed, (uint64_t)c, eps);
   for( int q=0 ; q<9 ; ++q ) out[q*n + c] = o[q];
}

__global__ void k_gr_p2c(GRParams P, long n, const double *prim, const double *x, double *cons){
   long c = (long)blockIdx.x*blockDim.x + threadIdx.x;
   if( c >= n ) return;
   double xx[3] = {x[c], x[n+c], x[2*n+c]}, p[9], u[9];
   for( int q=0 ; q<9 ; ++q ) p[q] = prim[q*n + c];
   Metric3 g;
   metric_at(P, xx, g);
   gr_prim2cons(P, g, p, u, xx);
   for( int q=0 ; q<9 ; ++q ) cons[q*n + c] = u[q];
}

/* ------------------------------------------------------------------ */
/* the solve                                                           */

#define C2P_BLOCK 256
#define C2P_WARPS (C2P_BLOCK/32)

struct C2PSmem {
   MlpPacked W;
   __nv_bfloat16 X[C2P_WARPS][32*8];
   float Y[C2P_WARPS][32*2];
};

/* One thread per cell.  Only the five numbers the Newton iteration reads
 * (s2, e, Q, psi, n) stay live across it: the metric and the rest of the
 * invariants, which only the recovery needs, are computed again afterwards
 * from a second (cached) read of the cell's cons and position.  The solve is
 * bound by the latency of its FP64 division chain, so resident warps matter
 * more than the few spills that 3 blocks of 256 per SM (80 registers) cost
 * in the set-up and recovery: measured 12% faster than 2 blocks. */
template<bool LEARNED, bool DUMP>
__global__ void __launch_bounds__(C2P_BLOCK, 3)
k_gr_c2p(GRParams P, long n, const double *__restrict__ cons, const double *__restrict__ x,
         double *__restrict__ prim, unsigned char *__restrict__ iters, float *__restrict__ pairs,
         const MlpPacked *__restrict__ mlp, StatsDev *__restrict__ stats){
   extern __shared__ __align__(16) unsigned char c2p_smem_raw[];
   C2PSmem &S = *reinterpret_cast<C2PSmem*>(c2p_smem_raw);
   __shared__ unsigned long long s_hist[64];
   __shared__ unsigned long long s_sum;
   __shared__ unsigned int s_max, s_fb, s_fail;
   for( int k=threadIdx.x ; k<64 ; k+=blockDim.x ) s_hist[k] = 0;
   if( threadIdx.x == 0 ){ s_sum = 0; s_max = 0; s_fb = 0; s_fail = 0; }
   if( LEARNED ) copy_packed(&S.W, mlp);
   __syncthreads();

   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   unsigned long long it_sum = 0;
   unsigned int it_max = 0, nfb = 0, nfail = 0;

   for( long base = (long)blockIdx.x*C2P_BLOCK ; base < n ; base += (long)gridDim.x*C2P_BLOCK ){
      const long c = base + threadIdx.x;
      const bool active = c < n;
      C2PInv I;
      double sig = 1.0;
      float f[8];
      {
         double u[9], p[9], xx[3];
         if( active ){
#pragma unroll
            for( int q=0 ; q<9 ; ++q ){ u[q] = cons[q*n + c]; p[q] = prim[q*n + c]; }
            xx[0] = x[c]; xx[1] = x[n + c]; xx[2] = x[2*n + c];
         }else{
            /* a benign state for the idle lanes of the last tile */
#pragma unroll
            for( int q=0 ; q<9 ; ++q ){ u[q] = 1.0; p[q] = 1.0; }
            xx[0] = 10.0; xx[1] = 0.0; xx[2] = 0.0;
         }
         Metric3 g;
         metric_at(P, xx, g);
         c2p_invariants(P, g, u, p, xx, I);
      }
      if( LEARNED || DUMP ) sig = mlp_features(I, f);
      double v2 = I.v20, eta = I.eta0;
      bool guess_ok = true;
      if( LEARNED ){
         __nv_bfloat16 *Xs = S.X[warp];
         bool fin = active && sig < 1e30;
#pragma unroll
         for( int k=0 ; k<8 ; ++k ) fin = fin && isfinite(f[k]);
#pragma unroll
         for( int k=0 ; k<8 ; k+=2 ){
            const float a = fin ? (f[k] - S.W.norm[k])*S.W.norm[8+k] : 0.f;
            const float b = fin ? (f[k+1] - S.W.norm[k+1])*S.W.norm[8+k+1] : 0.f;
            *reinterpret_cast<uint32_t*>(Xs + lane*8 + k) = pack_bf16(a, b);
         }
         __syncwarp();
         mlp_fwd_tile<false, true>(S.W, Xs, 0, lane, nullptr, nullptr, 0, S.Y[warp]);
         mlp_fwd_tile<false, true>(S.W, Xs, 1, lane, nullptr, nullptr, 0, S.Y[warp]);
         __syncwarp();
         const float y0 = S.Y[warp][2*lane], y1 = S.Y[warp][2*lane + 1];
         __syncwarp();
         const double d0 = sig*(double)(y0*S.W.norm[18] + S.W.norm[16]);
         const double d1 = sig*(double)(y1*S.W.norm[19] + S.W.norm[17]);
         const double etag = I.eta0*(double)__expf((float)d0);
         const double v2g = fmin(fmax(I.v20 + d1, 0.0), 0.99999999);
         if( fin && etag >= 1.0 && etag < 1e300 && v2g == v2g ){ v2 = v2g; eta = etag; }
         else guess_ok = false;
      }
      if( active ){
         int ok = 0, k = 0;
         if( guess_ok ) k = c2p_newton(P, I, &v2, &eta, &ok);
         if( LEARNED && !ok ){
            v2 = I.v20; eta = I.eta0;
            k += c2p_newton(P, I, &v2, &eta, &ok);
            nfb++;
         }
         if( !ok ) nfail++;
         {
            /* recovery: the metric and invariants again, from a second read */
            double u[9], p[9], xx[3];
#pragma unroll
            for( int q=0 ; q<9 ; ++q ){ u[q] = __ldcg(cons + q*n + c); p[q] = 1.0; }
            xx[0] = __ldcg(x + c); xx[1] = __ldcg(x + n + c); xx[2] = __ldcg(x + 2*n + c);
            Metric3 g;
            metric_at(P, xx, g);
            C2PInv J;
            c2p_invariants(P, g, u, p, xx, J);
            c2p_recover(P, g, J, v2, eta, u, p, xx);
#pragma unroll
            for( int q=0 ; q<9 ; ++q ) prim[q*n + c] = p[q];
         }
         if( iters ) iters[c] = (unsigned char)(k < 255 ? k : 255);
         if( DUMP ){
            float *pr = pairs + 10*c;
#pragma unroll
            for( int q=0 ; q<8 ; ++q ) pr[q] = f[q];
            const float nanf_ = __int_as_float(0x7fc00000);
            pr[8] = ok ? (float)(log1p((eta - I.eta0)/I.eta0)/sig) : nanf_;
            pr[9] = ok ? (float)((v2 - I.v20)/sig) : nanf_;
         }
         it_sum += (unsigned long long)k;
         it_max = k > (int)it_max ? (unsigned)k : it_max;
         atomicAdd(&s_hist[k < 63 ? k : 63], 1ull);
      }
   }
   /* block totals, then one atomic each into the global report */
#pragma unroll
   for( int o=16 ; o>0 ; o>>=1 ){
      it_sum += __shfl_xor_sync(0xffffffffu, it_sum, o);
      it_max = max(it_max, __shfl_xor_sync(0xffffffffu, it_max, o));
      nfb += __shfl_xor_sync(0xffffffffu, nfb, o);
      nfail += __shfl_xor_sync(0xffffffffu, nfail, o);
   }
   if( lane == 0 ){
      atomicAdd(&s_sum, it_sum); atomicMax(&s_max, it_max);
      atomicAdd(&s_fb, nfb); atomicAdd(&s_fail, nfail);
   }
   __syncthreads();
   if( threadIdx.x < 64 && s_hist[threadIdx.x] ) atomicAdd(&stats->hist[threadIdx.x], s_hist[threadIdx.x]);
   if( threadIdx.x == 0 ){
      atomicAdd(&stats->iters_sum, s_sum); atomicMax(&stats->iters_max, s_max);
      if( s_fb ) atomicAdd(&stats->n_fallback, s_fb);
      if( s_fail ) atomicAdd(&stats->n_fail, s_fail);
   }
}

/* ------------------------------------------------------------------ */
/* training                                                            */

#define TR_BLOCK 128
#define TR_LD 65       /* odd row stride: per-sample rows hit distinct banks */

struct TrainSmem {
   MlpPacked W;
   __nv_bfloat16 X[TR_BLOCK/32][32*8];
   float Xf[TR_BLOCK][8];
   float Y[TR_BLOCK/32][32*2];
   float DY[TR_BLOCK][2];
   float H1[TR_BLOCK*TR_LD];
   float H2[TR_BLOCK*TR_LD];
};

__device__ __forceinline__ float bf16r(float v){
   return __bfloat162float(__float2bfloat16_rn(v));
}
__device__ __forceinline__ float bf(const __nv_bfloat16 &v){ return __bfloat162float(v); }

/* Loss and gradient over nsamp samples in groups of TR_BLOCK.  Sample s is
 * pair s (sampled = 0) or pair hash(seed, step, s) mod n (sampled = 1).
 * dy = (y - t)/nsamp for samples with finite targets, 0 otherwise. */
__global__ void __launch_bounds__(TR_BLOCK)
k_mlp_grad(const MlpPacked *__restrict__ mlp, long n, const float *__restrict__ pairs, long nsamp,
           int sampled, uint64_t seed, int step, float *__restrict__ grad, double *__restrict__ loss){
   extern __shared__ __align__(16) unsigned char tr_smem_raw[];
   TrainSmem &S = *reinterpret_cast<TrainSmem*>(tr_smem_raw);
   copy_packed(&S.W, mlp);
   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   /* register accumulators: W3/b3 (b), W2/b2 (d), W1/b1 (f) */
   const int o3 = tid >> 6, k3 = tid & 63;
   float aW3 = 0.f, ab3 = 0.f;
   const int kb = tid >> 3, jb = tid & 7;
   float aW2[4][8], ab2[4];
#pragma unroll
   for( int a=0 ; a<4 ; ++a ){ ab2[a] = 0.f;
#pragma unroll
      for( int b=0 ; b<8 ; ++b ) aW2[a][b] = 0.f; }
   const int j1 = tid >> 1, i1 = (tid & 1)*4;
   float aW1[4] = {0.f, 0.f, 0.f, 0.f}, ab1 = 0.f;
   double lsum = 0.0;
   __syncthreads();

   const float invn = 1.0f/(float)nsamp;
   for( long base = (long)blockIdx.x*TR_BLOCK ; base < nsamp ; base += (long)gridDim.x*TR_BLOCK ){
      const long s = base + tid;
      const bool active = s < nsamp;
      long idx = s;
      if( sampled ) idx = (long)(grt_mix(seed ^ grt_mix(((uint64_t)step << 32) ^ (uint64_t)s)) % (uint64_t)n);
      float f[8], tg[2] = {0.f, 0.f};
      if( active ){
#pragma unroll
         for( int q=0 ; q<8 ; ++q ) f[q] = pairs[10*idx + q];
         tg[0] = pairs[10*idx + 8]; tg[1] = pairs[10*idx + 9];
      }
      bool valid = active && isfinite(tg[0]) && isfinite(tg[1]);
#pragma unroll
      for( int q=0 ; q<8 ; ++q ) valid = valid && isfinite(f[q]);
      __nv_bfloat16 *Xs = S.X[warp];
#pragma unroll
      for( int q=0 ; q<8 ; q+=2 ){
         float a = valid ? (f[q] - S.W.norm[q])*S.W.norm[8+q] : 0.f;
         float b = valid ? (f[q+1] - S.W.norm[q+1])*S.W.norm[8+q+1] : 0.f;
         *reinterpret_cast<uint32_t*>(Xs + lane*8 + q) = pack_bf16(a, b);
         S.Xf[tid][q] = bf16r(a); S.Xf[tid][q+1] = bf16r(b);
      }
      __syncwarp();
      float *H1w = S.H1 + warp*32*TR_LD, *H2w = S.H2 + warp*32*TR_LD;
      mlp_fwd_tile<true, false>(S.W, Xs, 0, lane, H1w, H2w, TR_LD, S.Y[warp]);
      mlp_fwd_tile<true, false>(S.W, Xs, 1, lane, H1w, H2w, TR_LD, S.Y[warp]);
      __syncwarp();
      {
         const float t0 = (tg[0] - S.W.norm[16])/S.W.norm[18];
         const float t1 = (tg[1] - S.W.norm[17])/S.W.norm[19];
         const float d0 = S.Y[warp][2*lane] - t0, d1 = S.Y[warp][2*lane + 1] - t1;
         if( valid ) lsum += (double)d0*d0 + (double)d1*d1;
         S.DY[tid][0] = valid ? d0*invn : 0.f;
         S.DY[tid][1] = valid ? d1*invn : 0.f;
      }
      __syncthreads();
      /* (b) dW3[o][k] = sum_s dy[s][o] bf16(h2[s][k]), db3 */
      for( int s2=0 ; s2<TR_BLOCK ; ++s2 ){
         const float d = S.DY[s2][o3];
         aW3 += d*bf16r(S.H2[s2*TR_LD + k3]);
         if( k3 == 0 ) ab3 += d;
      }
      __syncthreads();
      /* (c) da2 = (W3^T dy)(1 - h2^2), in place of h2 */
      {
         const float dy0 = S.DY[tid][0], dy1 = S.DY[tid][1];
         float *h = S.H2 + tid*TR_LD;
         for( int k=0 ; k<MLP_H ; ++k ){
            const float hv = h[k];
            h[k] = (bf(S.W.W3[0][k])*dy0 + bf(S.W.W3[1][k])*dy1)*(1.f - hv*hv);
         }
      }
      __syncthreads();
      /* (d) dW2[k][j] = sum_s da2[s][k] bf16(h1[s][j]), db2 */
      for( int s2=0 ; s2<TR_BLOCK ; ++s2 ){
         const float *d2 = S.H2 + s2*TR_LD + kb*4;
         const float *h1 = S.H1 + s2*TR_LD + jb*8;
         float hv[8];
#pragma unroll
         for( int b=0 ; b<8 ; ++b ) hv[b] = bf16r(h1[b]);
#pragma unroll
         for( int a=0 ; a<4 ; ++a ){
            const float dv = d2[a];
            if( jb == 0 ) ab2[a] += dv;
#pragma unroll
            for( int b=0 ; b<8 ; ++b ) aW2[a][b] += dv*hv[b];
         }
      }
      __syncthreads();
      /* (e) da1 = (W2^T da2)(1 - h1^2), in place of h1 */
      {
         float *h = S.H1 + tid*TR_LD;
         const float *d2 = S.H2 + tid*TR_LD;
         for( int j=0 ; j<MLP_H ; ++j ){
            float acc = 0.f;
#pragma unroll 8
            for( int k=0 ; k<MLP_H ; ++k ) acc += bf(S.W.W2[k][j])*d2[k];
            const float hv = h[j];
            h[j] = acc*(1.f - hv*hv);
         }
      }
      __syncthreads();
      /* (f) dW1[j][i] = sum_s da1[s][j] x[s][i], db1 */
      for( int s2=0 ; s2<TR_BLOCK ; ++s2 ){
         const float d = S.H1[s2*TR_LD + j1];
         if( i1 == 0 ) ab1 += d;
#pragma unroll
         for( int a=0 ; a<4 ; ++a ) aW1[a] += d*S.Xf[s2][i1 + a];
      }
      __syncthreads();
   }
   atomicAdd(&grad[OFF_W3 + o3*MLP_H + k3], aW3);
   if( k3 == 0 ) atomicAdd(&grad[OFF_B3 + o3], ab3);
#pragma unroll
   for( int a=0 ; a<4 ; ++a ){
      const int k = kb*4 + a;
      if( jb == 0 ) atomicAdd(&grad[OFF_B2 + k], ab2[a]);
#pragma unroll
      for( int b=0 ; b<8 ; ++b ) atomicAdd(&grad[OFF_W2 + k*MLP_H + jb*8 + b], aW2[a][b]);
   }
#pragma unroll
   for( int a=0 ; a<4 ; ++a ) atomicAdd(&grad[OFF_W1 + j1*8 + i1 + a], aW1[a]);
   if( i1 == 0 ) atomicAdd(&grad[OFF_B1 + j1], ab1);
#pragma unroll
   for( int o=16 ; o>0 ; o>>=1 ) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
   if( lane == 0 && lsum != 0.0 ) atomicAdd(loss, lsum/(2.0*(double)nsamp));
}

#include "mlp_tcgen05.cuh"

/* Write a parameter into the packed image (W rounded to BF16) */
__device__ __forceinline__ void pack_param(MlpPacked *P, int p, float w){
   if( p < OFF_B1 )      P->W1[p >> 3][p & 7] = __float2bfloat16_rn(w);
   else if( p < OFF_W2 ) P->b1[p - OFF_B1] = w;
   else if( p < OFF_B2 ){ int q = p - OFF_W2; P->W2[q >> 6][q & 63] = __float2bfloat16_rn(w); }
   else if( p < OFF_W3 ) P->b2[p - OFF_B2] = w;
   else if( p < OFF_B3 ){ int q = p - OFF_W3; P->W3[q >> 6][q & 63] = __float2bfloat16_rn(w); }
   else                  P->b3[p - OFF_B3] = w;
}

__global__ void k_mlp_pack(const float *__restrict__ master, MlpPacked *P){
   int p = blockIdx.x*blockDim.x + threadIdx.x;
   if( p < MLP_NPARAM ) pack_param(P, p, master[p]);
}

/* Adam (bias-corrected) on the FP32 master weights; writes the packed image
 * and clears the gradient. */
__global__ void k_mlp_adam(float *__restrict__ master, float *__restrict__ m, float *__restrict__ v,
                           float *__restrict__ grad, MlpPacked *P, float lr, float bc1, float bc2){
   int p = blockIdx.x*blockDim.x + threadIdx.x;
   if( p >= MLP_NPARAM ) return;
   const float b1 = 0.9f, b2 = 0.999f, epsa = 1e-8f;
   float gv = grad[p];
   if( !(gv == gv) ) gv = 0.f;
   float mv = b1*m[p] + (1.f - b1)*gv;
   float vv = b2*v[p] + (1.f - b2)*gv*gv;
   m[p] = mv; v[p] = vv;
   float w = master[p] - lr*(mv/bc1)/(sqrtf(vv/bc2) + epsa);
   master[p] = w;
   grad[p] = 0.f;
   pack_param(P, p, w);
}

/* Sums of the features and targets (and squares) of pairs with finite
 * targets: acc[0..9] sums, acc[10..19] sums of squares, acc[20] count. */
__global__ void k_mlp_moments(long n, const float *__restrict__ pairs, double *acc){
   __shared__ double s[21];
   if( threadIdx.x < 21 ) s[threadIdx.x] = 0.0;
   __syncthreads();
   double a[21];
   for( int q=0 ; q<21 ; ++q ) a[q] = 0.0;
   for( long c = (long)blockIdx.x*blockDim.x + threadIdx.x ; c < n ; c += (long)gridDim.x*blockDim.x ){
      const float *pr = pairs + 10*c;
      bool fin = isfinite(pr[8]) && isfinite(pr[9]);
      for( int q=0 ; q<8 ; ++q ) fin = fin && isfinite(pr[q]);
      if( !fin ) continue;
      for( int q=0 ; q<10 ; ++q ){ double v = pr[q]; a[q] += v; a[10+q] += v*v; }
      a[20] += 1.0;
   }
   for( int q=0 ; q<21 ; ++q ){
      double v = a[q];
      for( int o=16 ; o>0 ; o>>=1 ) v += __shfl_xor_sync(0xffffffffu, v, o);
      if( (threadIdx.x & 31) == 0 ) atomicAdd(&s[q], v);
   }
   __syncthreads();
   if( threadIdx.x < 21 ) atomicAdd(&acc[threadIdx.x], s[threadIdx.x]);
}

/* ------------------------------------------------------------------ */
/* host side                                                           */

struct disco_gr {
   int device;
   GRParams P;
   cudaStream_t stream;
   int nsm;
   MlpPacked *d_mlp;
   float *d_master, *d_m, *d_v, *d_grad;
   double *d_loss, *d_acc;
   StatsDev *d_stats;
   float h_norm[MLP_NNORM];
   bool have_mlp;
   long adam_t;
   int backend;               /* DISCO_MLP_TENSOR or DISCO_MLP_CUDA_CORES */
   int *d_err;                /* a tensor-core wait ran out */
   int c2p_blocks[4];
   std::string err;
};

static int fail(disco_gr *h, int code, const char *what, cudaError_t e = cudaSuccess){
   if( h ){
      char b[256];
      snprintf(b, sizeof b, "%s%s%s", what, e != cudaSuccess ? ": " : "",
               e != cudaSuccess ? cudaGetErrorString(e) : "");
      h->err = b;
   }
   return code;
}

#define GR_CK(call) do{ cudaError_t e_ = (call); if( e_ != cudaSuccess ) return fail(h, DISCO_ERR_CUDA, #call, e_); }while(0)

static inline unsigned nb(long n, int b){ return (unsigned)((n + b - 1)/b); }

template<bool L, bool D>
static int c2p_setup_attr(disco_gr *h, int slot){
   cudaError_t e = cudaFuncSetAttribute(k_gr_c2p<L, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)sizeof(C2PSmem));
   if( e != cudaSuccess ) return fail(h, DISCO_ERR_CUDA, "c2p smem attribute", e);
   int per = 0;
   e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_gr_c2p<L, D>, C2P_BLOCK, sizeof(C2PSmem));
   if( e != cudaSuccess ) return fail(h, DISCO_ERR_CUDA, "c2p occupancy", e);
   h->c2p_blocks[slot] = (per > 0 ? per : 1)*h->nsm;
   return DISCO_OK;
}

extern "C" {

int disco_gr_create(int device, const disco_gr_params *p, disco_gr **out){
   if( !p || !out ) return DISCO_ERR_ARG;
   *out = nullptr;
   if( !(p->gamma_law > 1.0) || !(p->tol > 0.0) || p->max_iter < 1 || p->max_iter > 100000 ||
       p->nextra < 0 || (p->metric != DISCO_GR_SCHW_KS && p->metric != DISCO_GR_KERR_KS) ||
       !(p->M > 0.0) || !(fabs(p->a) < p->M || (p->metric == DISCO_GR_SCHW_KS)) )
      return DISCO_ERR_ARG;
   int ndev = 0;
   if( cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 ) return DISCO_ERR_NO_DEVICE;
   if( device < 0 || device >= ndev ) return DISCO_ERR_ARG;
   disco_gr *h = new disco_gr();
   h->device = device;
   h->P.gam = p->gamma_law; h->P.rho_floor = p->rho_floor; h->P.p_floor = p->p_floor;
   h->P.M = p->M; h->P.a = p->metric == DISCO_GR_KERR_KS ? p->a : 0.0;
   h->P.tol = p->tol; h->P.metric = p->metric; h->P.nextra = p->nextra; h->P.max_iter = p->max_iter;
   h->stream = 0;
   h->have_mlp = false;
   h->adam_t = 0;
   h->backend = DISCO_MLP_TENSOR;
   h->d_err = nullptr;
   int rc = DISCO_OK;
   do{
      if( cudaSetDevice(device) != cudaSuccess ){ rc = DISCO_ERR_CUDA; break; }
      cudaDeviceGetAttribute(&h->nsm, cudaDevAttrMultiProcessorCount, device);
      if( cudaMalloc(&h->d_mlp, sizeof(MlpPacked)) != cudaSuccess ||
          cudaMalloc(&h->d_master, 4*MLP_NPARAM*sizeof(float)) != cudaSuccess ||
          cudaMalloc(&h->d_loss, 64*sizeof(double)) != cudaSuccess ||
          cudaMalloc(&h->d_stats, sizeof(StatsDev)) != cudaSuccess ){ rc = DISCO_ERR_CUDA; break; }
      h->d_m = h->d_master + MLP_NPARAM; h->d_v = h->d_m + MLP_NPARAM; h->d_grad = h->d_v + MLP_NPARAM;
      h->d_acc = h->d_loss + 32;
      if( cudaMemset(h->d_mlp, 0, sizeof(MlpPacked)) != cudaSuccess ||
          cudaMemset(h->d_master, 0, 4*MLP_NPARAM*sizeof(float)) != cudaSuccess ){ rc = DISCO_ERR_CUDA; break; }
      if( (rc = c2p_setup_attr<false, false>(h, 0)) ) break;
      if( (rc = c2p_setup_attr<false, true>(h, 1)) ) break;
      if( (rc = c2p_setup_attr<true, false>(h, 2)) ) break;
      if( (rc = c2p_setup_attr<true, true>(h, 3)) ) break;
      if( cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(TrainSmem)) != cudaSuccess ){ rc = DISCO_ERR_CUDA; break; }
      if( cudaFuncSetAttribute(k_mlp_grad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sizeof(TcSmem)) != cudaSuccess ){ rc = DISCO_ERR_CUDA; break; }
      if( cudaMalloc(&h->d_err, sizeof(int)) != cudaSuccess ||
          cudaMemset(h->d_err, 0, sizeof(int)) != cudaSuccess ){ rc = DISCO_ERR_CUDA; break; }
   }while(0);
   if( rc != DISCO_OK ){ disco_gr_destroy(h); return rc; }
   for( int k=0 ; k<8 ; ++k ){ h->h_norm[k] = 0.f; h->h_norm[8+k] = 1.f; }
   h->h_norm[16] = 0.f; h->h_norm[17] = 0.f; h->h_norm[18] = 1.f; h->h_norm[19] = 1.f;
   *out = h;
   return DISCO_OK;
}

void disco_gr_destroy(disco_gr *h){
   if( !h ) return;
   cudaSetDevice(h->device);
   cudaFree(h->d_mlp); cudaFree(h->d_master); cudaFree(h->d_loss); cudaFree(h->d_stats);
   cudaFree(h->d_err);
   delete h;
}

int disco_gr_set_stream(disco_gr *h, void *stream){
   if( !h ) return DISCO_ERR_ARG;
   h->stream = (cudaStream_t)stream;
   return DISCO_OK;
}

const char *disco_gr_last_error(disco_gr *h){
   return h ? h->err.c_str() : "null handle";
}

static int check_n(disco_gr *h, long n){
   if( n <= 0 || n > (long)1 << 28 ) return fail(h, DISCO_ERR_ARG, "cell count out of range");
   return DISCO_OK;
}

int disco_gr_grid(disco_gr *h, int Nr, int Nz, int Np, double rmin, double rmax,
                  double zmin, double zmax, int log_r, double *x){
   if( !h || !x || Nr < 1 || Nz < 1 || Np < 1 || !(rmin > 0.0) || !(rmax > rmin) || !(zmax > zmin) )
      return fail(h, DISCO_ERR_ARG, "grid arguments");
   long n = (long)Nr*Nz*Np;
   if( check_n(h, n) ) return DISCO_ERR_ARG;
   GR_CK(cudaSetDevice(h->device));
   k_gr_grid<<<nb(n, 256), 256, 0, h->stream>>>(Nr, Nz, Np, rmin, rmax, zmin, zmax, log_r, n, x);
   GR_CK(cudaGetLastError());
   return DISCO_OK;
}

int disco_gr_torus_prims(disco_gr *h, const disco_gr_torus *tp, long n, const double *x, double *prim){
   if( !h || !tp || !x || !prim ) return fail(h, DISCO_ERR_ARG, "null argument");
   if( check_n(h, n) ) return DISCO_ERR_ARG;
   GR_CK(cudaSetDevice(h->device));
   gr_torus_par t;
   memcpy(&t, tp, sizeof t);
   k_gr_torus<<<nb(n, 256), 256, 0, h->stream>>>(t, n, x, prim);
   GR_CK(cudaGetLastError());
   return DISCO_OK;
}

int disco_gr_perturb(disco_gr *h, long n, const double *prim, double *out, unsigned long long seed,
                     double eps){
   if( !h || !prim || !out ) return fail(h, DISCO_ERR_ARG, "null argument");
   if( check_n(h, n) ) return DISCO_ERR_ARG;
   GR_CK(cudaSetDevice(h->device));
   k_gr_perturb<<<nb(n, 256), 256, 0, h->stream>>>(n, prim, out, seed, eps);
   GR_CK(cudaGetLastError());
   return DISCO_OK;
}

int disco_gr_prim2cons(disco_gr *h, long n, const double *prim, const double *x, double *cons){
   if( !h || !prim || !x || !cons ) return fail(h, DISCO_ERR_ARG, "null argument");
   if( check_n(h, n) ) return DISCO_ERR_ARG;
   GR_CK(cudaSetDevice(h->device));
   k_gr_p2c<<<nb(n, 256), 256, 0, h->stream>>>(h->P, n, prim, x, cons);
   GR_CK(cudaGetLastError());
   return DISCO_OK;
}

int disco_gr_cons2prim(disco_gr *h, long n, const double *cons, const double *x, double *prim,
                       int guess, unsigned char *iters, float *pairs, disco_gr_stats *stats){
   if( !h || !cons || !x || !prim ) return fail(h, DISCO_ERR_ARG, "null argument");
   if( check_n(h, n) ) return DISCO_ERR_ARG;
   if( guess != DISCO_GUESS_PREVIOUS && guess != DISCO_GUESS_LEARNED )
      return fail(h, DISCO_ERR_ARG, "unknown guess");
   if( guess == DISCO_GUESS_LEARNED && !h->have_mlp )
      return fail(h, DISCO_ERR_STATE, "learned guess requested before the network was set or trained");
   GR_CK(cudaSetDevice(h->device));
   GR_CK(cudaMemsetAsync(h->d_stats, 0, sizeof(StatsDev), h->stream));
   const bool L = guess == DISCO_GUESS_LEARNED, D = pairs != nullptr;
   const int slot = (L ? 2 : 0) + (D ? 1 : 0);
   unsigned grid = (unsigned)h->c2p_blocks[slot];
   if( grid > nb(n, C2P_BLOCK) ) grid = nb(n, C2P_BLOCK);
   const size_t sm = sizeof(C2PSmem);
   if( L && D )       k_gr_c2p<true, true><<<grid, C2P_BLOCK, sm, h->stream>>>(h->P, n, cons, x, prim, iters, pairs, h->d_mlp, h->d_stats);
   else if( L )       k_gr_c2p<true, false><<<grid, C2P_BLOCK, sm, h->stream>>>(h->P, n, cons, x, prim, iters, pairs, h->d_mlp, h->d_stats);
   else if( D )       k_gr_c2p<false, true><<<grid, C2P_BLOCK, sm, h->stream>>>(h->P, n, cons, x, prim, iters, pairs, h->d_mlp, h->d_stats);
   else               k_gr_c2p<false, false><<<grid, C2P_BLOCK, sm, h->stream>>>(h->P, n, cons, x, prim, iters, pairs, h->d_mlp, h->d_stats);
   GR_CK(cudaGetLastError());
   if( stats ){
      StatsDev s;
      GR_CK(cudaMemcpyAsync(&s, h->d_stats, sizeof s, cudaMemcpyDeviceToHost, h->stream));
      GR_CK(cudaStreamSynchronize(h->stream));
      memcpy(stats, &s, sizeof s);
      stats->ncell = n;
   }
   return DISCO_OK;
}

static int repack(disco_gr *h){
   k_mlp_pack<<<nb(MLP_NPARAM, 256), 256, 0, h->stream>>>(h->d_master, h->d_mlp);
   GR_CK(cudaGetLastError());
   GR_CK(cudaMemcpyAsync((char*)h->d_mlp + offsetof(MlpPacked, norm), h->h_norm,
                         sizeof(h->h_norm), cudaMemcpyHostToDevice, h->stream));
   GR_CK(cudaStreamSynchronize(h->stream));
   return DISCO_OK;
}

static int reset_adam(disco_gr *h){
   GR_CK(cudaMemsetAsync(h->d_m, 0, 3*MLP_NPARAM*sizeof(float), h->stream));
   h->adam_t = 0;
   return DISCO_OK;
}

int disco_gr_mlp_init(disco_gr *h, unsigned long long seed){
   if( !h ) return DISCO_ERR_ARG;
   GR_CK(cudaSetDevice(h->device));
   std::vector<float> w(MLP_NPARAM, 0.f);
   uint64_t st = seed;
   auto uni = [&](){ st += 0x9e3779b97f4a7c15ULL; return (double)(grt_mix(st) >> 11)*(1.0/9007199254740992.0); };
   struct { int off, fo, fi; } L[3] = {{OFF_W1, MLP_H, MLP_IN}, {OFF_W2, MLP_H, MLP_H}, {OFF_W3, MLP_OUT, MLP_H}};
   for( auto &l : L ){
      double lim = sqrt(6.0/(double)(l.fo + l.fi));
      for( int k=0 ; k<l.fo*l.fi ; ++k ) w[l.off + k] = (float)((2.0*uni() - 1.0)*lim);
   }
   GR_CK(cudaMemcpyAsync(h->d_master, w.data(), MLP_NPARAM*sizeof(float), cudaMemcpyHostToDevice, h->stream));
   if( int rc = reset_adam(h) ) return rc;
   if( int rc = repack(h) ) return rc;
   h->have_mlp = true;
   return DISCO_OK;
}

int disco_gr_mlp_set(disco_gr *h, const float *param, const float *norm){
   if( !h || !param || !norm ) return fail(h, DISCO_ERR_ARG, "null argument");
   GR_CK(cudaSetDevice(h->device));
   for( int k=0 ; k<MLP_NNORM ; ++k ){
      if( !isfinite(norm[k]) ) return fail(h, DISCO_ERR_ARG, "non-finite normalisation");
      h->h_norm[k] = norm[k];
   }
   GR_CK(cudaMemcpyAsync(h->d_master, param, MLP_NPARAM*sizeof(float), cudaMemcpyHostToDevice, h->stream));
   if( int rc = reset_adam(h) ) return rc;
   if( int rc = repack(h) ) return rc;
   h->have_mlp = true;
   return DISCO_OK;
}

int disco_gr_mlp_get(disco_gr *h, float *param, float *norm){
   if( !h || !param || !norm ) return fail(h, DISCO_ERR_ARG, "null argument");
   GR_CK(cudaSetDevice(h->device));
   MlpPacked P;
   GR_CK(cudaMemcpyAsync(&P, h->d_mlp, sizeof P, cudaMemcpyDeviceToHost, h->stream));
   GR_CK(cudaStreamSynchronize(h->stream));
   auto f = [](__nv_bfloat16 v){ uint16_t b; memcpy(&b, &v, 2); uint32_t u = (uint32_t)b << 16; float o; memcpy(&o, &u, 4); return o; };
   for( int j=0 ; j<MLP_H ; ++j ) for( int i=0 ; i<MLP_IN ; ++i ) param[OFF_W1 + j*8 + i] = f(P.W1[j][i]);
   for( int j=0 ; j<MLP_H ; ++j ) param[OFF_B1 + j] = P.b1[j];
   for( int k=0 ; k<MLP_H ; ++k ) for( int j=0 ; j<MLP_H ; ++j ) param[OFF_W2 + k*MLP_H + j] = f(P.W2[k][j]);
   for( int k=0 ; k<MLP_H ; ++k ) param[OFF_B2 + k] = P.b2[k];
   for( int o=0 ; o<MLP_OUT ; ++o ) for( int k=0 ; k<MLP_H ; ++k ) param[OFF_W3 + o*MLP_H + k] = f(P.W3[o][k]);
   for( int o=0 ; o<MLP_OUT ; ++o ) param[OFF_B3 + o] = P.b3[o];
   memcpy(norm, h->h_norm, sizeof(h->h_norm));
   return DISCO_OK;
}

int disco_gr_mlp_fit_norm(disco_gr *h, long n, const float *pairs){
   if( !h || !pairs ) return fail(h, DISCO_ERR_ARG, "null argument");
   if( check_n(h, n) ) return DISCO_ERR_ARG;
   GR_CK(cudaSetDevice(h->device));
   GR_CK(cudaMemsetAsync(h->d_acc, 0, 21*sizeof(double), h->stream));
   unsigned grid = nb(n, 256);
   if( grid > (unsigned)(8*h->nsm) ) grid = 8*h->nsm;
   k_mlp_moments<<<grid, 256, 0, h->stream>>>(n, pairs, h->d_acc);
   GR_CK(cudaGetLastError());
   double a[21];
   GR_CK(cudaMemcpyAsync(a, h->d_acc, sizeof a, cudaMemcpyDeviceToHost, h->stream));
   GR_CK(cudaStreamSynchronize(h->stream));
   if( a[20] < 2.0 ) return fail(h, DISCO_ERR_ARG, "fewer than two pairs with finite targets");
   for( int q=0 ; q<10 ; ++q ){
      double mean = a[q]/a[20];
      double var = a[10+q]/a[20] - mean*mean;
      double sd = var > 0.0 ? sqrt(var) : 0.0;
      if( !(sd > 1e-30) ) sd = 1.0;
      if( q < 8 ){ h->h_norm[q] = (float)mean; h->h_norm[8+q] = (float)(1.0/sd); }
      else { h->h_norm[16 + (q-8)] = (float)mean; h->h_norm[18 + (q-8)] = (float)sd; }
   }
   return repack(h);
}

static int launch_grad(disco_gr *h, long n, const float *pairs, long nsamp, int sampled,
                       uint64_t seed, int step, double *loss_slot){
   unsigned grid = nb(nsamp, TR_BLOCK);
   if( grid > (unsigned)(2*h->nsm) ) grid = 2*h->nsm;
   if( h->backend == DISCO_MLP_TENSOR )
      k_mlp_grad_tc<<<grid, TC_BLOCK, sizeof(TcSmem), h->stream>>>(h->d_mlp, n, pairs, nsamp, sampled,
                                                                  seed, step, h->d_grad, loss_slot,
                                                                  h->d_err);
   else
      k_mlp_grad<<<grid, TR_BLOCK, sizeof(TrainSmem), h->stream>>>(h->d_mlp, n, pairs, nsamp, sampled,
                                                                  seed, step, h->d_grad, loss_slot);
   GR_CK(cudaGetLastError());
   return DISCO_OK;
}

/* after a synchronisation: a tensor-core wait that ran out */
static int tc_status(disco_gr *h){
   int e = 0;
   GR_CK(cudaMemcpy(&e, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
   if( e ){
      cudaMemset(h->d_err, 0, sizeof(int));
      return fail(h, DISCO_ERR_INTERNAL, "tensor-core training kernel: an MMA wait ran out");
   }
   return DISCO_OK;
}

int disco_gr_mlp_set_backend(disco_gr *h, int backend){
   if( !h || (backend != DISCO_MLP_TENSOR && backend != DISCO_MLP_CUDA_CORES) ) return DISCO_ERR_ARG;
   h->backend = backend;
   return DISCO_OK;
}

int disco_gr_mlp_grad(disco_gr *h, long n, const float *pairs, float *grad, double *loss){
   if( !h || !pairs || !grad || !loss ) return fail(h, DISCO_ERR_ARG, "null argument");
   if( check_n(h, n) ) return DISCO_ERR_ARG;
   if( !h->have_mlp ) return fail(h, DISCO_ERR_STATE, "network not set");
   GR_CK(cudaSetDevice(h->device));
   GR_CK(cudaMemsetAsync(h->d_grad, 0, MLP_NPARAM*sizeof(float), h->stream));
   GR_CK(cudaMemsetAsync(h->d_loss, 0, sizeof(double), h->stream));
   if( int rc = launch_grad(h, n, pairs, n, 0, 0, 0, h->d_loss) ) return rc;
   GR_CK(cudaMemcpyAsync(grad, h->d_grad, MLP_NPARAM*sizeof(float), cudaMemcpyDeviceToHost, h->stream));
   GR_CK(cudaMemcpyAsync(loss, h->d_loss, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
   GR_CK(cudaMemsetAsync(h->d_grad, 0, MLP_NPARAM*sizeof(float), h->stream));
   GR_CK(cudaStreamSynchronize(h->stream));
   return tc_status(h);
}

int disco_gr_mlp_train(disco_gr *h, long n, const float *pairs, int steps, int batch, float lr,
                       unsigned long long seed, double *loss_hist){
   if( !h || !pairs || steps < 1 || batch < 1 || !(lr > 0.f) ) return fail(h, DISCO_ERR_ARG, "train arguments");
   if( check_n(h, n) ) return DISCO_ERR_ARG;
   if( !h->have_mlp ) return fail(h, DISCO_ERR_STATE, "network not initialised");
   GR_CK(cudaSetDevice(h->device));
   double *d_hist = nullptr;
   GR_CK(cudaMallocAsync(&d_hist, (size_t)steps*sizeof(double), h->stream));
   GR_CK(cudaMemsetAsync(d_hist, 0, (size_t)steps*sizeof(double), h->stream));
   GR_CK(cudaMemsetAsync(h->d_grad, 0, MLP_NPARAM*sizeof(float), h->stream));
   int rc = DISCO_OK;
   for( int s=0 ; s<steps && rc == DISCO_OK ; ++s ){
      rc = launch_grad(h, n, pairs, batch, 1, seed, s, d_hist + s);
      if( rc ) break;
      h->adam_t++;
      const double frac = (double)s/(double)steps;
      const float lrs = (float)(lr*(0.05 + 0.95*0.5*(1.0 + cos(M_PI*frac))));
      const float bc1 = (float)(1.0 - pow(0.9, (double)h->adam_t));
      const float bc2 = (float)(1.0 - pow(0.999, (double)h->adam_t));
      k_mlp_adam<<<nb(MLP_NPARAM, 256), 256, 0, h->stream>>>(h->d_master, h->d_m, h->d_v, h->d_grad,
                                                             h->d_mlp, lrs, bc1, bc2);
      cudaError_t e = cudaGetLastError();
      if( e != cudaSuccess ) rc = fail(h, DISCO_ERR_CUDA, "adam launch", e);
   }
   if( rc == DISCO_OK && loss_hist )
      if( cudaMemcpyAsync(loss_hist, d_hist, (size_t)steps*sizeof(double), cudaMemcpyDeviceToHost,
                          h->stream) != cudaSuccess ) rc = fail(h, DISCO_ERR_CUDA, "loss history copy");
   cudaFreeAsync(d_hist, h->stream);
   GR_CK(cudaStreamSynchronize(h->stream));
   if( rc == DISCO_OK ) rc = tc_status(h);
   return rc;
}

} // extern "C"
