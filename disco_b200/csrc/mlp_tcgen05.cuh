/*
 * The network's training gradient on the 5th-generation tensor cores:
 * tcgen05.mma (BF16 operands in shared memory, FP32 accumulators in tensor
 * memory) for the four contractions of a 128-sample group, the rest of the
 * backward on the CUDA cores.  Same loss, samples and parameter layout as
 * k_mlp_grad (the CUDA-core kernel it stands beside); included by
 * disco_c2p.cu after MlpPacked, pack_bf16 and grt_mix.
 *
 * Per group of 128 samples (thread t = sample t = accumulator row / TMEM
 * lane t), every MMA M = 128, K = 16 per instruction:
 *   D  = X  W1^T      N = 64, K = 16 (8 inputs, zero-padded)   -> H1 = tanh(D + b1)
 *   D  = H1 W2^T      N = 64, K = 64                           -> H2 = tanh(D + b2)
 *   (Y = H2 W3^T + b3, dY, dA2 = (dY W3)(1 - H2^2) on the CUDA cores)
 *   D  = dA2 W2       N = 64, K = 64                           -> dA1 = D (1 - H1^2)
 *   G2 += dA2^T [H1 1] rows k (64 of 128, the rest zero rows), N = 80, K = 128 samples
 *   G1 += dA1^T [X 1]  rows j (64 of 128), N = 16, K = 128 samples
 *   G3 += [H2 1]^T dY  rows k (65 of 128), N = 16 (2 used), K = 128 samples
 * A column of ones beside H1 and X, and a row of ones under H2^T, make the
 * same products give the bias gradients (db2, db1, db3) with the weight
 * gradients (dW2, dW1, dW3).  G1-G3 accumulate in tensor memory over the
 * block's groups and are added to the gradient once at the end.  The
 * transposed products read the same shared-memory tiles as the forward
 * ones, through MN-major descriptors.
 *
 * Operand tiles are the canonical no-swizzle layout: 8 x 8 BF16 core
 * matrices of 128 contiguous bytes (row r at byte 16 r), a descriptor's
 * SBO the byte distance between core matrices along M / N and LBO along K.
 * Every wait on the MMA barrier is bounded (a clock budget); a wait that
 * runs out sets *err, and the block stops issuing MMAs and frees its tensor
 * memory.  One block per SM (shared memory > half the SM's), 256 tensor-
 * memory columns each, so the allocation never waits.
 */
#pragma once

namespace disco {

#define TC_BLOCK 128
#define TC_COLS 256            /* TMEM columns per block: D 0-63, G2 64-143, G1 144-159, G3 160-175 */
#define TC_WAIT_CYCLES (1ll << 31)   /* about one second at the SM clock */

struct TcSmem {
   /* UMMA operand tiles, [row group][column group][8 x 8] BF16 */
   __nv_bfloat16 W1b[8*2*64];    /* B of X W1^T:  N = j (8 groups), K = i (2) */
   __nv_bfloat16 W2b[8*8*64];    /* B of H1 W2^T: N = k, K = j */
   __nv_bfloat16 W2t[8*8*64];    /* B of dA2 W2:  N = j, K = k */
   __nv_bfloat16 Xb[16*2*64];    /* [s group][i group]; i 8 = 1, i 9..15 zero */
   __nv_bfloat16 H1b[16*10*64];  /* [s group][j group]; j 64 = 1, j 65..79 zero */
   __nv_bfloat16 DA2b[16*16*64]; /* [s group][k group]; k groups 8..15 zero (the padded M of G2) */
   __nv_bfloat16 DA1b[16*16*64]; /* [s group][j group]; j groups 8..15 zero */
   __nv_bfloat16 H2b[16*16*64];  /* [s group][k group]; k 64 = 1, the rest of 8..15 zero */
   __nv_bfloat16 DYb[16*2*64];   /* [s group][o group]; o 2..15 zero */
   float b1[MLP_H], b2[MLP_H], W3[2][MLP_H], b3[2], norm[MLP_NNORM];
   uint64_t bar;
   uint32_t tmem;
   int abort;
};

/* byte offset of element (r, c) of a tile stored [rg][cg] with ncg column groups */
__device__ __forceinline__ int tc_off(int r, int c, int ncg){
   return (((r >> 3)*ncg + (c >> 3))*64 + (r & 7)*8 + (c & 7))*2;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p){
   return (uint32_t)__cvta_generic_to_shared(p);
}

/* shared-memory matrix descriptor, no swizzle (layout type 0), version 1 */
__device__ __forceinline__ uint64_t tc_desc(uint32_t addr, uint32_t lbo, uint32_t sbo){
   return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
          ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

/* instruction descriptor of kind::f16: BF16 A and B, FP32 D, M = 128 */
__host__ __device__ constexpr uint32_t tc_idesc(int N, bool a_mn, bool b_mn){
   return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
          ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, int acc){
   asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0)
                : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *bar){
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                :: "r"(smem_u32(bar)) : "memory");
}

/* bounded wait for the barrier's phase `parity` to complete */
__device__ __forceinline__ bool tc_wait(uint64_t *bar, uint32_t parity){
   const uint32_t a = smem_u32(bar);
   const long long t0 = clock64();
   for( ;; ){
      uint32_t done;
      asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                   "selp.b32 %0, 1, 0, P1;\n\t}" : "=r"(done) : "r"(a), "r"(parity) : "memory");
      if( done ) return true;
      if( clock64() - t0 > TC_WAIT_CYCLES ) return false;
   }
}

/* 16 FP32 columns [col, col+16) of this thread's TMEM lane (its warp's quarter) */
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float *v){
   uint32_t r[16];
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                  "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
                  "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr));
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for( int q=0 ; q<16 ; ++q ) v[q] = __uint_as_float(r[q]);
}

__device__ __forceinline__ void tc_fence_before(){ asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after(){ asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_async_smem(){ asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

/* a row of 8 values of a tile as one 16-byte store */
__device__ __forceinline__ void tc_put8(__nv_bfloat16 *tile, int r, int cg, int ncg, const float *v){
   uint4 u;
   u.x = pack_bf16(v[0], v[1]); u.y = pack_bf16(v[2], v[3]);
   u.z = pack_bf16(v[4], v[5]); u.w = pack_bf16(v[6], v[7]);
   *reinterpret_cast<uint4*>(reinterpret_cast<char*>(tile) + tc_off(r, cg*8, ncg)) = u;
}

/* Loss and gradient over nsamp samples (as k_mlp_grad); err: wait timed out */
__global__ void __launch_bounds__(TC_BLOCK, 1)
k_mlp_grad_tc(const MlpPacked *__restrict__ mlp, long n, const float *__restrict__ pairs, long nsamp,
              int sampled, uint64_t seed, int step, float *__restrict__ grad, double *__restrict__ loss,
              int *__restrict__ err){
   extern __shared__ __align__(1024) unsigned char tc_smem_raw[];
   TcSmem &S = *reinterpret_cast<TcSmem*>(tc_smem_raw);
   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

   /* weights into the operand tiles, the rest as FP32 */
   for( int e=tid ; e<MLP_H*16 ; e+=TC_BLOCK ){
      const int j = e >> 4, i = e & 15;
      const __nv_bfloat16 w = i < 8 ? mlp->W1[j][i] : __float2bfloat16_rn(0.f);
      *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(S.W1b) + tc_off(j, i, 2)) = w;
   }
   for( int e=tid ; e<MLP_H*MLP_H ; e+=TC_BLOCK ){
      const int k = e >> 6, j = e & 63;
      const __nv_bfloat16 w = mlp->W2[k][j];
      *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(S.W2b) + tc_off(k, j, 8)) = w;
      *reinterpret_cast<__nv_bfloat16*>(reinterpret_cast<char*>(S.W2t) + tc_off(j, k, 8)) = w;
   }
   {  /* the pad groups: zero, and the ones of the bias products (each
       * thread its own sample row; the rows are rewritten per group only in
       * their data groups) */
      uint4 z = make_uint4(0, 0, 0, 0);
      for( int e=tid ; e<(int)(sizeof(S.DA2b)/16) ; e+=TC_BLOCK ){
         reinterpret_cast<uint4*>(S.DA2b)[e] = z;
         reinterpret_cast<uint4*>(S.DA1b)[e] = z;
         reinterpret_cast<uint4*>(S.H2b)[e] = z;
      }
      /* the zeroing above covers other threads' rows: finish it before any
       * thread writes its ones column into H2b */
      __syncthreads();
      float one[8] = {1.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f}, zero[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      tc_put8(S.Xb, tid, 1, 2, one);
      tc_put8(S.H1b, tid, 8, 10, one);
      tc_put8(S.H1b, tid, 9, 10, zero);
      tc_put8(S.H2b, tid, 8, 16, one);
      tc_put8(S.DYb, tid, 1, 2, zero);
   }
   if( tid < MLP_H ){
      S.b1[tid] = mlp->b1[tid]; S.b2[tid] = mlp->b2[tid];
      S.W3[0][tid] = __bfloat162float(mlp->W3[0][tid]); S.W3[1][tid] = __bfloat162float(mlp->W3[1][tid]);
   }
   if( tid < MLP_NNORM ) S.norm[tid] = mlp->norm[tid];
   if( tid < 2 ) S.b3[tid] = mlp->b3[tid];
   if( tid == 0 ){
      S.abort = 0;
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(&S.bar)), "r"(1) : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
   }
   if( warp == 0 ){
      asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                   :: "r"(smem_u32(&S.tmem)), "r"(TC_COLS) : "memory");
      asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
   }
   tc_fence_async_smem();
   tc_fence_before();
   __syncthreads();
   tc_fence_after();
   const uint32_t tm = S.tmem;
   const uint32_t lane_base = tm + ((uint32_t)(32*warp) << 16);
   uint32_t parity = 0;
   bool live = true;
   double lsum = 0.0;
   const float invn = 1.0f/(float)nsamp;

   const uint32_t aX = smem_u32(S.Xb), aH1 = smem_u32(S.H1b), aDA2 = smem_u32(S.DA2b),
                  aDA1 = smem_u32(S.DA1b), aW1 = smem_u32(S.W1b), aW2 = smem_u32(S.W2b),
                  aW2t = smem_u32(S.W2t), aH2 = smem_u32(S.H2b), aDY = smem_u32(S.DYb);
   /* wait for the MMAs just committed; every thread learns whether to go on */
   auto sync_mma = [&]() -> bool {
      const bool ok = tc_wait(&S.bar, parity);
      parity ^= 1u;
      if( !ok ) S.abort = 1;
      tc_fence_after();
      __syncthreads();
      return S.abort == 0;
   };
   /* generic-proxy tile writes visible to the MMAs, then one thread issues */
   auto publish = [&](){
      tc_fence_async_smem();
      tc_fence_before();
      __syncthreads();
      tc_fence_after();
   };

   int g = 0;
   for( long base = (long)blockIdx.x*TC_BLOCK ; base < nsamp && live ; base += (long)gridDim.x*TC_BLOCK, ++g ){
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
      float x[8];
#pragma unroll
      for( int q=0 ; q<8 ; ++q ) x[q] = valid ? (f[q] - S.norm[q])*S.norm[8+q] : 0.f;
      tc_put8(S.Xb, tid, 0, 2, x);           /* group 1 holds the ones column */
      publish();
      if( tid == 0 ){
         tc_mma(tm, tc_desc(aX, 128, 256), tc_desc(aW1, 128, 256), tc_idesc(64, false, false), 0);
         tc_commit(&S.bar);
      }
      if( !sync_mma() ){ live = false; break; }

      /* H1 = tanh(X W1^T + b1) */
      float h1[MLP_H];
#pragma unroll
      for( int c=0 ; c<4 ; ++c ) tc_ld16(lane_base + 16*c, h1 + 16*c);
#pragma unroll
      for( int j=0 ; j<MLP_H ; ++j ) h1[j] = tanhf(h1[j] + S.b1[j]);
#pragma unroll
      for( int jg=0 ; jg<8 ; ++jg ) tc_put8(S.H1b, tid, jg, 10, h1 + 8*jg);
      publish();
      if( tid == 0 ){
#pragma unroll
         for( int q=0 ; q<4 ; ++q )
            tc_mma(tm, tc_desc(aH1 + 256*q, 128, 1280), tc_desc(aW2 + 256*q, 128, 1024),
                   tc_idesc(64, false, false), q > 0);
         tc_commit(&S.bar);
      }
      if( !sync_mma() ){ live = false; break; }

      /* H2, Y, dY on the CUDA cores; dA2 into its tile */
      float h2[MLP_H];
#pragma unroll
      for( int c=0 ; c<4 ; ++c ) tc_ld16(lane_base + 16*c, h2 + 16*c);
      float y0 = S.b3[0], y1 = S.b3[1];
#pragma unroll
      for( int k=0 ; k<MLP_H ; ++k ){
         h2[k] = tanhf(h2[k] + S.b2[k]);
         const float hb = __bfloat162float(__float2bfloat16_rn(h2[k]));
         y0 += hb*S.W3[0][k];
         y1 += hb*S.W3[1][k];
      }
      const float t0 = (tg[0] - S.norm[16])/S.norm[18];
      const float t1 = (tg[1] - S.norm[17])/S.norm[19];
      const float d0 = y0 - t0, d1 = y1 - t1;
      if( valid ) lsum += (double)d0*d0 + (double)d1*d1;
      const float dy0 = valid ? d0*invn : 0.f, dy1 = valid ? d1*invn : 0.f;
      float da2[MLP_H];
#pragma unroll
      for( int k=0 ; k<MLP_H ; ++k ) da2[k] = (S.W3[0][k]*dy0 + S.W3[1][k]*dy1)*(1.f - h2[k]*h2[k]);
#pragma unroll
      for( int kg=0 ; kg<8 ; ++kg ){
         tc_put8(S.DA2b, tid, kg, 16, da2 + 8*kg);
         tc_put8(S.H2b, tid, kg, 16, h2 + 8*kg);
      }
      {
         float dy[8] = {dy0, dy1, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
         tc_put8(S.DYb, tid, 0, 2, dy);
      }
      publish();
      if( tid == 0 ){
         /* dA2 W2 -> D; G2 += dA2^T [H1 1] (MN-major: rows k, 16 groups, 8 of
          * them zero); G3 += [H2 1]^T dY (rows k and the ones row 64) */
#pragma unroll
         for( int q=0 ; q<4 ; ++q )
            tc_mma(tm, tc_desc(aDA2 + 256*q, 128, 2048), tc_desc(aW2t + 256*q, 128, 1024),
                   tc_idesc(64, false, false), q > 0);
#pragma unroll
         for( int q=0 ; q<8 ; ++q ){
            const int acc = (g > 0 || q > 0) ? 1 : 0;
            tc_mma(tm + 64, tc_desc(aDA2 + 4096*q, 2048, 128), tc_desc(aH1 + 2560*q, 1280, 128),
                   tc_idesc(80, true, true), acc);
            tc_mma(tm + 160, tc_desc(aH2 + 4096*q, 2048, 128), tc_desc(aDY + 512*q, 256, 128),
                   tc_idesc(16, true, true), acc);
         }
         tc_commit(&S.bar);
      }
      if( !sync_mma() ){ live = false; break; }

      /* dA1 = (dA2 W2)(1 - H1^2) into its tile; G1 += dA1^T X */
      float da1[MLP_H];
#pragma unroll
      for( int c=0 ; c<4 ; ++c ) tc_ld16(lane_base + 16*c, da1 + 16*c);
#pragma unroll
      for( int j=0 ; j<MLP_H ; ++j ) da1[j] *= (1.f - h1[j]*h1[j]);
#pragma unroll
      for( int jg=0 ; jg<8 ; ++jg ) tc_put8(S.DA1b, tid, jg, 16, da1 + 8*jg);
      publish();
      if( tid == 0 ){
#pragma unroll
         for( int q=0 ; q<8 ; ++q )
            tc_mma(tm + 144, tc_desc(aDA1 + 4096*q, 2048, 128), tc_desc(aX + 512*q, 256, 128),
                   tc_idesc(16, true, true), (g > 0 || q > 0) ? 1 : 0);
         tc_commit(&S.bar);
      }
      if( !sync_mma() ){ live = false; break; }
   }

   if( S.abort ){
      if( tid == 0 ) atomicOr(err, 1);
   }else if( g > 0 && warp < 3 ){
      /* rows r = lane of warps 0-2: G2 row k: dW2[k][j] (columns 0-63) and
       * db2[k] (column 64); G1 row j: dW1[j][i] (columns 0-7) and db1[j]
       * (column 8); G3 row k: dW3[o][k] (columns 0, 1), row 64: db3 */
      const int r = 32*warp + lane;
      float v[16];
      if( r < MLP_H ){
#pragma unroll
         for( int c=0 ; c<4 ; ++c ){
            tc_ld16(lane_base + 64 + 16*c, v);
#pragma unroll
            for( int q=0 ; q<16 ; ++q ) atomicAdd(&grad[OFF_W2 + r*MLP_H + 16*c + q], v[q]);
         }
         tc_ld16(lane_base + 128, v);
         atomicAdd(&grad[OFF_B2 + r], v[0]);
         tc_ld16(lane_base + 144, v);
#pragma unroll
         for( int q=0 ; q<8 ; ++q ) atomicAdd(&grad[OFF_W1 + r*8 + q], v[q]);
         atomicAdd(&grad[OFF_B1 + r], v[8]);
         tc_ld16(lane_base + 160, v);
         atomicAdd(&grad[OFF_W3 + r], v[0]);
         atomicAdd(&grad[OFF_W3 + MLP_H + r], v[1]);
      }else{
         /* warp 2: the tcgen05.ld is warp-wide; lane 0 (row 64) keeps db3 */
#pragma unroll
         for( int c=0 ; c<4 ; ++c ) tc_ld16(lane_base + 64 + 16*c, v);
         tc_ld16(lane_base + 128, v);
         tc_ld16(lane_base + 144, v);
         tc_ld16(lane_base + 160, v);
         if( r == MLP_H ){ atomicAdd(&grad[OFF_B3], v[0]); atomicAdd(&grad[OFF_B3 + 1], v[1]); }
      }
   }
   if( !S.abort ){
#pragma unroll
      for( int o=16 ; o>0 ; o>>=1 ) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
      if( lane == 0 && lsum != 0.0 ) atomicAdd(loss, lsum/(2.0*(double)nsamp));
   }
   tc_fence_before();
   __syncthreads();
   tc_fence_after();
   if( warp == 0 )
      asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tm), "r"(TC_COLS) : "memory");
}

} /* namespace disco */
