/*
 * disco_mindt_noalloc: the CFL time step (getmindt) of one disk whose cell
 * state already lives in the caller's device memory, computed without any
 * device allocation.
 *
 * Who needs it: callers that may not call cudaMalloc at all -- a host code
 * that hands the library memory from its own pool and forbids the library
 * from growing device usage behind its back, or a driver loop that runs
 * inside a region where allocation is not allowed (an allocator that is
 * locked for the duration of a run, a memory budget that is already fully
 * committed).  disco_batch_mindt needs a batch, and creating a batch
 * allocates; this entry point needs only the caller's arrays.
 *
 * Its working memory is one file-scope device array, disco_noalloc_scratch
 * (struct NoAllocScratch below, about 3.2 MiB).  Every GPU that loads the library holds
 * that array until the process exits, whether or not this function is used.
 * Host code cannot use the array's name as a device address, so the first
 * call on each device looks the address up with cudaGetSymbolAddress (with
 * that device current) and keeps it; make that first call before any stream
 * capture.  All calls share the one array and it keeps the last call's
 * contents, so calls that overlap on the GPU (two streams, two host threads)
 * race: serialise them.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>
#include "disco_b200.h"
#include "disco_device.cuh"

using namespace disco;

/* Limits of the static scratch (all must hold for a call to be accepted;
 * otherwise the call prints the limit and returns DISCO_ERR_ARG). */
#define NA_MAX_ANN    65536          /* annuli (Nr*Nz)                        */
#define NA_MAX_EDGES  8192           /* r_jph / z_kph entries each            */
#define NA_BLOCK      256
#define NA_MAX_BLOCKS 262144         /* cells <= NA_MAX_BLOCKS*NA_BLOCK = 64Mi */

struct NoAllocScratch {
   int4 ann[NA_MAX_ANN];                  /* cell offset, Np, j, k            */
   double rj[NA_MAX_EDGES];
   double zk[NA_MAX_EDGES];
   unsigned long long part[NA_MAX_BLOCKS];/* per-block minima (double bits)   */
   unsigned long long result;
   int err;
};

static __device__ __align__(256) NoAllocScratch disco_noalloc_scratch;

/* Device address of the scratch per device ordinal, looked up once. */
#define NA_MAX_DEV 64
static NoAllocScratch *g_scratch_addr[NA_MAX_DEV];

/* The viscous limit of euler.c's mindt (:357-375) needs only these
 * parameters of the disk: Use_Viscosity, Use_As_Alpha, Viscosity. */
struct NoAllocVisc { int visc, alpha; double nu; };

__global__ void k_noalloc_mindt(NoAllocScratch *S, int nann, int ncell,
                                const double *prim, const double *piph, const double *dphi,
                                const double *wiph, double gam, double Pmax,
                                int NgRa, int NgRb, int NgZa, int NgZb, int Nr, int Nz,
                                NoAllocVisc vp_){
   __shared__ unsigned long long s_min[NA_BLOCK/32];
   int c = blockIdx.x*blockDim.x + threadIdx.x;
   double dtc = 1.0e300;
   int err = 0;
   if( c < ncell ){
      int lo = 0, hi = nann - 1;                 /* annulus of cell c */
      while( lo < hi ){
         int mid = (lo + hi + 1) >> 1;
         if( S->ann[mid].x <= c ) lo = mid; else hi = mid - 1;
      }
      int4 a = S->ann[lo];
      int j = a.z, k = a.w, np = a.y, i = c - a.x;
      bool real = j >= NgRa && j < Nr - NgRb && k >= NgZa && k < Nz - NgZb;
      if( real ){                                  /* misc.c:57-76, euler.c:332 */
         const double *rj = S->rj + 1, *zk = S->zk + 1;
         double rp = rj[j], rm = rj[j-1], zp = zk[k], zm = zk[k-1];
         double ph = piph[c], phim = ph - dphi[c];
         int cprev = a.x + (i == 0 ? np-1 : i-1);
         double w = .5*(wiph[cprev] + wiph[c]);
         double r = centroid_r(rp, rm);
         double vp = (prim[UPP*ncell + c] - w)*r;
         double cs = sqrt(gam*prim[PPP*ncell + c]/prim[RHO*ncell + c]);
         double maxvr = cs + fabs(prim[URR*ncell + c]);
         double maxvp = cs + fabs(vp);
         double maxvz = cs + fabs(prim[UZZ*ncell + c]);
         double dtr = (rp-rm)/maxvr;
         double dtp = (.5*(rp+rm))*get_dp(ph, phim, Pmax, &err)/maxvp;
         double dtz = (zp-zm)/maxvz;
         double dtm = dtr;
         if( dtm > dtp ) dtm = dtp;
         if( dtm > dtz ) dtm = dtz;
         if( vp_.visc ){                           /* euler.c:357-375 */
            DiskParams P;
            P.gam = gam; P.visc = 1; P.visc_alpha = vp_.alpha; P.visc_nu = vp_.nu;
            double pc[6];
            for( int q=0 ; q<6 ; ++q ) pc[q] = prim[q*ncell + c];
            dtm = visc_dt_limit(P, pc, r, dtm, rp, rm, zp, zm, get_dp(ph, phim, Pmax, &err));
         }
         if( dtm == dtm ) dtc = dtm;
      }
   }
   if( err ) atomicOr(&S->err, err);
   unsigned long long bits = dbits(dtc);
   for( int o=16 ; o>0 ; o>>=1 ){
      unsigned long long ob = __shfl_down_sync(0xffffffffu, bits, o);
      bits = ob < bits ? ob : bits;
   }
   if( (threadIdx.x & 31) == 0 ) s_min[threadIdx.x >> 5] = bits;
   __syncthreads();
   if( threadIdx.x == 0 ){
      unsigned long long m = s_min[0];
      for( int w=1 ; w<NA_BLOCK/32 ; ++w ) m = s_min[w] < m ? s_min[w] : m;
      S->part[blockIdx.x] = m;
   }
}

/* One block: min over the per-block minima and maxDT/CFL, times CFL. */
__global__ void k_noalloc_finish(NoAllocScratch *S, int nblocks, double dt0){
   __shared__ unsigned long long s_min[NA_BLOCK/32];
   unsigned long long m = dbits(dt0);
   for( int b=threadIdx.x ; b<nblocks ; b+=blockDim.x ) m = S->part[b] < m ? S->part[b] : m;
   for( int o=16 ; o>0 ; o>>=1 ){
      unsigned long long ob = __shfl_down_sync(0xffffffffu, m, o);
      m = ob < m ? ob : m;
   }
   if( (threadIdx.x & 31) == 0 ) s_min[threadIdx.x >> 5] = m;
   __syncthreads();
   if( threadIdx.x == 0 ){
      unsigned long long r = s_min[0];
      for( int w=1 ; w<NA_BLOCK/32 ; ++w ) r = s_min[w] < r ? s_min[w] : r;
      S->result = r;
   }
}

extern "C" int disco_mindt_noalloc(const disco_params *p, int hydro, int Nr, int Nz,
                                   const int *Ng, const int *Np, const double *r_jph,
                                   const double *z_kph, const double *prim, const double *piph,
                                   const double *dphi, const double *wiph, void *stream,
                                   double *dt){
   if( !p || !Ng || !Np || !r_jph || !z_kph || !prim || !piph || !dphi || !wiph || !dt )
      return DISCO_ERR_ARG;
   if( hydro != DISCO_HYDRO_EULER ) return DISCO_ERR_UNSUPPORTED;
   /* the sizes are checked before any product of them is formed */
   if( Nr < 1 || Nz < 1 || Nr > NA_MAX_EDGES-1 || Nz > NA_MAX_EDGES-1 ||
       (long long)Nr*(long long)Nz > NA_MAX_ANN ){
      fprintf(stderr, "disco_mindt_noalloc: grid of %d x %d annuli exceeds the scratch limits "
                      "(%d annuli, %d edges per direction)\n", Nr, Nz, NA_MAX_ANN, NA_MAX_EDGES);
      return DISCO_ERR_ARG;
   }
   const int nann = Nr*Nz;
   long long ncell = 0;
   int4 tab[1024];
   int dev = 0;
   if( cudaGetDevice(&dev) != cudaSuccess ) return DISCO_ERR_NO_DEVICE;
   if( dev < 0 || dev >= NA_MAX_DEV ) return DISCO_ERR_ARG;
   /* The scratch used below is the current device's copy, so the caller's
    * arrays must live on that device too (a stream of another device would
    * fail at the first copy; an array of another device would be read
    * through the wrong device's scratch). */
   {
      const void *arrs[4] = {prim, piph, dphi, wiph};
      for( int m=0 ; m<4 ; ++m ){
         cudaPointerAttributes at;
         if( cudaPointerGetAttributes(&at, arrs[m]) != cudaSuccess ){ cudaGetLastError(); return DISCO_ERR_ARG; }
         if( at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged ) return DISCO_ERR_ARG;
         if( at.device != dev ) return DISCO_ERR_ARG;
      }
   }
   for( int a=0 ; a<nann ; ++a ){
      if( Np[a] < 1 ) return DISCO_ERR_ARG;
      ncell += Np[a];
   }
   long long nblocks = (ncell + NA_BLOCK - 1)/NA_BLOCK;
   if( ncell < 1 || nblocks > NA_MAX_BLOCKS ){
      fprintf(stderr, "disco_mindt_noalloc: %lld cells exceeds the scratch limit of %d\n",
              ncell, NA_MAX_BLOCKS*NA_BLOCK);
      return DISCO_ERR_ARG;
   }
   /* once per device, with it current: the scratch's device address */
   if( !g_scratch_addr[dev] ){
      void *ptr = NULL;
      if( cudaGetSymbolAddress(&ptr, disco_noalloc_scratch) != cudaSuccess || !ptr )
         return DISCO_ERR_CUDA;
      g_scratch_addr[dev] = (NoAllocScratch *)ptr;
   }
   NoAllocScratch *S = g_scratch_addr[dev];
   cudaStream_t s = (cudaStream_t)stream;
   /* annulus table and grid edges into the scratch, in chunks from the stack */
   long long off = 0;
   for( int a0=0 ; a0<nann ; a0+=1024 ){
      int n = nann - a0 < 1024 ? nann - a0 : 1024;
      for( int t=0 ; t<n ; ++t ){
         int a = a0 + t;
         tab[t] = make_int4((int)off, Np[a], a % Nr, a / Nr);
         off += Np[a];
      }
      if( cudaMemcpyAsync(S->ann + a0, tab, n*sizeof(int4), cudaMemcpyHostToDevice, s) != cudaSuccess )
         return DISCO_ERR_CUDA;
      if( cudaStreamSynchronize(s) != cudaSuccess ) return DISCO_ERR_CUDA;
   }
   if( cudaMemcpyAsync(S->rj, r_jph, (Nr+1)*sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
       cudaMemcpyAsync(S->zk, z_kph, (Nz+1)*sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess ||
       cudaMemsetAsync(&S->err, 0, sizeof(int), s) != cudaSuccess )
      return DISCO_ERR_CUDA;
   k_noalloc_mindt<<<(unsigned)nblocks, NA_BLOCK, 0, s>>>(S, nann, (int)ncell, prim, piph, dphi, wiph,
                                                         p->Adiabatic_Index, p->phimax,
                                                         Ng[0], Ng[1], Ng[2], Ng[3], Nr, Nz,
                                                         NoAllocVisc{p->visc_flag ? 1 : 0,
                                                                     p->alpha_flag ? 1 : 0,
                                                                     p->viscosity});
   double dt0 = p->maxDT / p->CFL;                       /* misc.c:52-54 */
   if( dt0 <= 0.0 ) dt0 = 1.0e100;
   k_noalloc_finish<<<1, NA_BLOCK, 0, s>>>(S, (int)nblocks, dt0);
   if( cudaGetLastError() != cudaSuccess ) return DISCO_ERR_CUDA;
   unsigned long long bits = 0;
   int err = 0;
   if( cudaMemcpyAsync(&bits, &S->result, sizeof bits, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
       cudaMemcpyAsync(&err, &S->err, sizeof err, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
       cudaStreamSynchronize(s) != cudaSuccess )
      return DISCO_ERR_CUDA;
   double mn;
   memcpy(&mn, &bits, sizeof mn);
   *dt = mn*p->CFL;
   return err ? DISCO_ERR_PHI_WRAP : DISCO_OK;
}
