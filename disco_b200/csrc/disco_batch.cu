/*
 * C ABI of the B200 Disco timestep (include/disco_b200.h): batch set-up,
 * host <-> device state transfer, and the per-step launch sequence that
 * replaces timestep()/onestep() (timestep.c:7-45, onestep.c:84-229).
 *
 * One batch = one or more independent disks in one set of ragged SoA
 * arrays.  A substep is begin / I0 / faces / gradr / flux_r / flux_p /
 * update / c2p, a step two substeps plus three tiny per-disk kernels; the
 * multi-step driver captures one step in a CUDA graph and replays it with
 * dt left on the device by the previous step's fused getmindt.
 *
 * Two precisions share the code: DISCO_PREC_FP64 (ViewT<double>, the
 * reference's arithmetic) and DISCO_PREC_MIXED (ViewT<float>: FP32 prim,
 * slopes and fluxes; FP64 geometry, mesh, dt and Kahan-compensated cons).
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <vector>
#include <algorithm>
#include "disco_batch_impl.cuh"

static int cuda_status(cudaError_t e){
   return e == cudaSuccess ? DISCO_OK : DISCO_ERR_CUDA;
}
#define CK(x) do{ cudaError_t _e = (x); if( _e != cudaSuccess ){ \
   fprintf(stderr, "disco_b200: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(_e), __FILE__, __LINE__); \
   return DISCO_ERR_CUDA; } }while(0)


static void *dalloc_bytes(disco_batch *b, size_t bytes){
   void *p = NULL;
   if( bytes == 0 ) bytes = 8;
   if( cudaMalloc(&p, bytes) != cudaSuccess ) return NULL;
   cudaMemset(p, 0, bytes);
   b->allocs.push_back(p);
   return p;
}
template<class T>
static T *dalloc(disco_batch *b, size_t n){ return (T *)dalloc_bytes(b, n*sizeof(T)); }
template<class T>
static T *dupload(disco_batch *b, const std::vector<T> &h){
   T *p = dalloc<T>(b, h.size());
   if( p && !h.empty() ) cudaMemcpy(p, h.data(), h.size()*sizeof(T), cudaMemcpyHostToDevice);
   return p;
}

extern "C" int disco_abi_version(void){ return DISCO_ABI_VERSION; }

extern "C" const char *disco_strerror(int s){
   switch( s ){
      case DISCO_OK: return "ok";
      case DISCO_ERR_ARG: return "bad argument";
      case DISCO_ERR_CUDA: return "CUDA runtime error";
      case DISCO_ERR_UNSUPPORTED: return "module combination not built";
      case DISCO_ERR_PHI_WRAP: return "phi wrap loop hit its cap (non-finite piph)";
      case DISCO_ERR_NONFINITE: return "non-finite or non-positive dt";
      case DISCO_ERR_NO_DEVICE: return "no CUDA device";
      case DISCO_ERR_STATE: return "call out of order";
      case DISCO_ERR_INTERNAL: return "device consistency check failed";
      case DISCO_ERR_IO: return "file not written, read or parsed";
   }
   return "unknown status";
}

/* Each side of the modules composed from boundary_functions.c (0 inner r,
 * 1 outer r, 2 lower z, 3 upper z): fixed (set_cell_init, boundary_fixed_*),
 * zero-gradient copy (boundary_zerograd_*, diode 0 or 1), mirror copy
 * (boundary_reflect_*: the annulus as far inside as the ghost is outside,
 * then reflect_prims' normal velocity negated), or nothing. */
enum { SIDE_NONE = 0, SIDE_FIXED, SIDE_ZG, SIDE_ZG_DIODE, SIDE_REFLECT,
       SIDE_NOSLIP,             /* mirror copy, all three velocity components negated */
       SIDE_ZG_DIODE_PHIWIN };  /* zero-gradient with the diode, then fixed on 0.3 pi < phi < 1.7 pi */
static int side_mode(int boundary, int s){
   static const int zg[4] = {SIDE_ZG, SIDE_ZG, SIDE_ZG, SIDE_ZG};
   static const int zgd[4] = {SIDE_ZG_DIODE, SIDE_ZG_DIODE, SIDE_ZG_DIODE, SIDE_ZG_DIODE};
   static const int acc3[4] = {SIDE_ZG_DIODE, SIDE_FIXED, SIDE_FIXED, SIDE_FIXED};
   static const int frz[4] = {SIDE_FIXED, SIDE_FIXED, SIDE_REFLECT, SIDE_REFLECT};      /* fixRrefZ.c */
   static const int tube[4] = {SIDE_NONE, SIDE_REFLECT, SIDE_ZG, SIDE_ZG};             /* tube.c */
   static const int sgb[4] = {SIDE_REFLECT, SIDE_REFLECT, SIDE_REFLECT, SIDE_ZG_DIODE}; /* surfaceGravBox.c */
   static const int gap[4] = {SIDE_ZG_DIODE, SIDE_FIXED, SIDE_ZG_DIODE, SIDE_ZG_DIODE}; /* fixed_gap.c */
   static const int flow[4] = {SIDE_NOSLIP, SIDE_ZG_DIODE_PHIWIN, SIDE_FIXED, SIDE_FIXED}; /* flowthrough.c */
   switch( boundary ){
      case DISCO_BC_ZEROGRAD: return zg[s];
      case DISCO_BC_OUTFLOW3D: case DISCO_BC_ZEROGRAD_OMK: return zgd[s];
      case DISCO_BC_ACCRETE3D: return acc3[s];
      case DISCO_BC_FIXRREFZ: return frz[s];
      case DISCO_BC_TUBE: return tube[s];
      case DISCO_BC_SURFACEGRAVBOX: return sgb[s];
      case DISCO_BC_FIXED_GAP: return gap[s];
      case DISCO_BC_FLOWTHROUGH: return flow[s];
   }
   return SIDE_NONE;
}
static bool side_copies(int m){
   return m == SIDE_ZG || m == SIDE_ZG_DIODE || m == SIDE_REFLECT || m == SIDE_NOSLIP ||
          m == SIDE_ZG_DIODE_PHIWIN;
}
static bool side_mirror(int m){ return m == SIDE_REFLECT || m == SIDE_NOSLIP; }
/* the fixed sides of the newer composed modules (fixed_ghost_init bc 11) */
static int side_fixed_mask(int boundary){
   if( boundary != DISCO_BC_FIXRREFZ && boundary != DISCO_BC_TUBE && boundary != DISCO_BC_FLOWTHROUGH &&
       boundary != DISCO_BC_SURFACEGRAVBOX && boundary != DISCO_BC_FIXED_GAP ) return 0;
   int m = 0;
   for( int s=0 ; s<4 ; ++s ) if( side_mode(boundary, s) == SIDE_FIXED ) m |= 1 << s;
   return m ? m : 16;          /* 16: composed, no fixed side */
}

static void fill_disk_params(DiskParams &D, const disco_params &p, const disco_modules &m){
   memset(&D, 0, sizeof D);
   D.gam = p.Adiabatic_Index; D.PLM = p.PLM; D.CFL = p.CFL; D.maxDT = p.maxDT;
   D.Pmax = p.phimax; D.rho_floor = p.Density_Floor; D.p_floor = p.Pressure_Floor;
   D.RotOmega = p.RotOmega; D.Mach = p.Disk_Mach;
   D.Cs2_M = p.metricPar[2]; D.Cs2_H0 = p.initPar[4]; D.Cs2_r1 = p.initPar[2];
   D.mesh_motion = p.Mesh_Motion; D.riemann = p.Riemann_Solver; D.en_om = p.Energy_Omega;
   D.mesh_om = p.Exact_Mesh_Omega; D.isothermal = p.isothermal_flag;
   D.cs2_profile = p.Cs2_Profile; D.grav2D = p.grav2D; D.polar = p.NoBC_Rmin == 1;
   D.timestep = p.Timestep;
   D.atmos = p.include_atmos ? 1 : 0;
   D.visc = p.visc_flag ? 1 : 0;
   D.visc_alpha = p.alpha_flag ? 1 : 0;
   D.visc_nu = p.viscosity;
   D.noise_type = (p.noiseType >= 1 && p.noiseType <= 3) ? p.noiseType : 0;
   D.noise_abs = p.noiseAbs; D.noise_rel = p.noiseRel;
   D.rotframe = p.RotFrame;
   D.planets_move = (m.planets == DISCO_PLANETS_CM2 || m.planets == DISCO_PLANETS_BINARY_SOFT ||
                     m.planets == DISCO_PLANETS_CIRCULAR || m.planets == DISCO_PLANETS_CM);
   /* Planets/cm.c:47-53: the softening relaxes as smooth + exp(-t/30) */
   D.pl_eps_decay = m.planets == DISCO_PLANETS_CM;
   D.pl_smooth = 0.5/p.Disk_Mach;
   D.ic.mach = p.Disk_Mach; D.ic.amp = p.initPar[1];
   D.ic.rmin = p.rmin; D.ic.rmax = p.rmax; D.ic.phimax = p.phimax;
   D.ic.seed = (uint64_t)(int64_t)p.initPar0;
   D.ic.kind = (int)p.initPar[2];
   D.ic_module = m.initial == DISCO_IC_MHD_SHEAR_NOISE ? 1 : m.initial == DISCO_IC_GR_TORUS_NOISE ? 2 : 0;
   D.gr = m.hydro == DISCO_HYDRO_GRMHD ? 1 : 0;
   D.gr_metric = m.metric == DISCO_METRIC_KERR_KS_RPZ ? 1 : 0;
   D.gr_M = p.metricPar[2];
   D.gr_a = m.metric == DISCO_METRIC_KERR_KS_RPZ ? p.metricPar[3] : 0.0;
   D.ic_gr.seed = (uint64_t)(int64_t)p.initPar0; D.ic_gr.amp = p.initPar[1];
   D.ic_gr.rc = p.initPar[2]; D.ic_gr.wr = p.initPar[3]; D.ic_gr.hr = p.initPar[4];
   D.ic_gr.beta = p.initPar[5]; D.ic_gr.rho_atm = p.initPar[6]; D.ic_gr.p_atm = p.initPar[7];
   D.ic_gr.s_cut = p.initPar[8];
   D.ic_gr.M = p.metricPar[2]; D.ic_gr.a = D.gr_a;
   D.ic_gr.rmin = p.rmin; D.ic_gr.rmax = p.rmax; D.ic_gr.zmin = p.zmin; D.ic_gr.zmax = p.zmax;
   D.ic_gr.phimax = p.phimax;
   D.bc_horizon = m.boundary == DISCO_BC_HORIZON ? 8 : m.boundary == DISCO_BC_HORIZON3D ? 9 :
                  m.boundary == DISCO_BC_HORIZON_BIN ? 10 : 0;
   D.side_fixed = side_fixed_mask(m.boundary) & 15;
   D.ic_mhd.seed = (uint64_t)(int64_t)p.initPar0; D.ic_mhd.amp = p.initPar[1];
   D.ic_mhd.cs = p.initPar[3]; D.ic_mhd.beta = p.initPar[4]; D.ic_mhd.gam = p.Adiabatic_Index;
   D.ic_mhd.rmin = p.rmin; D.ic_mhd.rmax = p.rmax; D.ic_mhd.zmin = p.zmin; D.ic_mhd.zmax = p.zmax;
   D.ic_mhd.phimax = p.phimax; D.ic_mhd.kind = (int)p.initPar[2];
   D.ic_mhd.beta_phi = p.initPar[5]; D.ic_mhd.b_r = p.initPar[6];
}

static void init_planets(DiskState &S, DiskParams &D, const disco_params &p, const disco_modules &m){
   memset(S.pl, 0, sizeof S.pl);
   switch( m.planets ){
      case DISCO_PLANETS_SUN:                          /* Planets/sun.c:9-17 */
         D.npl = 1; S.pl[0].M = 1.0; break;
      case DISCO_PLANETS_CM2: {                        /* Planets/cm2.c:14-38 */
         D.npl = 2;
         double a = 1.0, q = p.Mass_Ratio, mu = q/(1.+q), om = pow(a,-1.5);
         S.pl[0].M = 1.-mu; S.pl[0].omega = om; S.pl[0].r = a*mu; S.pl[0].phi = M_PI;
         S.pl[1].M = mu;    S.pl[1].omega = om; S.pl[1].r = a*(1.-mu);
         break; }
      case DISCO_PLANETS_BINARY_SOFT: {                /* new module: softened equal-mass binary */
         /* separation 1, circular, softening Init_Par8 (Init_Par5-7 belong
          * to the disk's initial conditions) */
         D.npl = 2;
         double a = 1.0, eps = p.initPar[8];
         double om = 1.0/(a*sqrt(a));
         S.pl[0].M = 0.5; S.pl[0].omega = om; S.pl[0].r = 0.5*a; S.pl[0].phi = M_PI; S.pl[0].eps = eps;
         S.pl[1].M = 0.5; S.pl[1].omega = om; S.pl[1].r = 0.5*a; S.pl[1].phi = 0.0;  S.pl[1].eps = eps;
         break; }
      case DISCO_PLANETS_CIRCULAR: {                   /* Planets/circular.c:19-39 */
         D.npl = 2;
         S.pl[0].M = 1.0;
         S.pl[1].M = p.Mass_Ratio; S.pl[1].omega = 1.0; S.pl[1].r = 1.0; S.pl[1].eps = 0.5/p.Disk_Mach;
         break; }
      case DISCO_PLANETS_CM: {                         /* Planets/cm.c:21-45 */
         D.npl = 2;
         double a = 1.0, q = p.Mass_Ratio, mu = q/(1.+q), om = pow(a,-1.5), sm = 0.5/p.Disk_Mach;
         S.pl[0].M = 1.-mu; S.pl[0].omega = om; S.pl[0].r = a*mu; S.pl[0].phi = M_PI; S.pl[0].eps = sm;
         S.pl[1].M = mu;    S.pl[1].omega = om; S.pl[1].r = a*(1.-mu); S.pl[1].eps = sm;
         break; }
      default:                                          /* Planets/none.c:9-17 */
         D.npl = 1; S.pl[0].M = 0.0; S.pl[0].eps = 1.0; break;
   }
}

/* The radius of a track's face centres, evaluated on the host with the
 * device's operations and order (each an IEEE-rounded double operation, no
 * contraction: the sum of products as in centroid_r), and 1/(1/r) for the
 * B-field scale factor of the CT edge values. */
static double host_centroid_r(double xp, double xm){
   volatile double a = xp*xp, bb = xp*xm, c = xm*xm;
   double s = (a + bb) + c;
   volatile double num = 2.0*s, den = 3.0*(xp+xm);
   return num / den;
}
static void push_track_r(disco_batch *b, double r){
   b->tr_r.push_back(r);
   volatile double inv = 1.0/r;
   b->tr_irf.push_back(1.0/inv);
}

/* the FP32 view: same allocations, R* pointers reinterpreted */
static void make_float_view(disco_batch *b){
   ViewT<double> &d = b->vd;
   ViewT<float> &f = b->vf;
   memcpy(&f, &d, sizeof f);
   f.prim = (float *)d.prim; f.gradp = (float *)d.gradp; f.gradr = (float *)d.gradr;
   f.gradz = (float *)d.gradz;
   f.fS = (float *)d.fS; f.fG = (float *)d.fG;
   f.ctE = (float *)d.ctE; f.ctB = (float *)d.ctB;
   f.pE = (float *)d.pE; f.pB = (float *)d.pB; f.pEr = (float *)d.pEr; f.pBz = (float *)d.pBz;
   f.fEt = (float *)d.fEt; f.fBt = (float *)d.fBt; f.fEphi = (float *)d.fEphi;
}

extern "C" void disco_batch_destroy(disco_batch *b);

/* ---- the one-launch step (disco_step_persist.cuh) ---------------------- */

#ifndef PERSIST_TILE
#define PERSIST_TILE 8
#endif

/* the module selections the persistent step covers */
static bool persist_eligible(const disco_batch *b){
   return !b->ct && !b->any_3d && !b->bc_zerograd && !b->any_mm3 && !b->any_visc &&
          b->timestep_mode == 0 && (b->bc_fixed == 0 || b->bc_fixed == 1 || b->bc_fixed == 3);
}

/* The work list: every block of both substeps and the per-disk items, each
 * with a position P in its disk's pipeline such that everything an item
 * reads from has a smaller P: with W = 16 positions per annulus, substep
 * base B (8, or W (Nr+4) + 8 for the second substep) and j the annulus (for
 * a track, its inner annulus):
 *   begin(j) B + Wj      I0(j..)  B + Wj + 1       faces(j,j+1) B + W(j+1) + 2
 *   grad(j)  B + W(j+1) + 3   flux(j,j+1) B + W(j+2) + 4
 *   update(j) B + W(j+2) + 5  c2p(j) B + W(j+2) + 6
 *   timestep() start 0, planets after substep 1 W(Nr+4) + 4,
 *   diagnostics of annuli ..j  second B + W(j+2) + 7, end 2W(Nr+4) + 16.
 * Keys are P over the disk's total (all disks advance together), cut into
 * tiles of about 8 grids' worth of items; inside a tile the order is
 * (substep, stage, key).  Every dependency has a smaller key and an earlier
 * (substep, stage), so it comes earlier in the list. */
static int build_persist_plan(disco_batch *b){
   b->persist_ok = 0;
   int bps = b->prec == DISCO_PREC_MIXED ? mixed_persist_blocks_per_sm(b) : persist_blocks_per_sm_t<double>(b);
   int nsm = 0;
   if( cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, b->device) != cudaSuccess ) return DISCO_ERR_CUDA;
   if( bps < 1 || nsm < 1 ) return DISCO_OK;           /* not resident: keep the kernels */
   const long G = (long)bps*nsm;
   const int nann = (int)b->ann_np.size(), ntr = (int)b->tr_a.size(), nd = b->ndisk;
   std::vector<int> nu(nann, 0), nf(ntr, 0), ndc(nd, 0);
   for( const int2 &u : b->ublk ) nu[u.x]++;
   for( const int2 &f : b->fblk ) nf[f.x]++;
   for( int a=0 ; a<nann ; ++a ) ndc[b->ann_disk[a]] += b->ann_nblk[a];
   struct It { int4 w; int sub, rank, disk, tile; double key; };
   std::vector<It> L;
   L.reserve(2*(3*b->cblk.size() + 2*b->fblk.size() + b->ublk.size()) + 4*nd + nann);
   const long W = 16;
   auto add = [&](int stage, int sub, int rank, int x, int n, int d, long P){
      long Nr = b->disk_Nr[d];
      double tot = (double)(2*W*(Nr+4) + 16);
      It it;
      it.w = make_int4(stage | (sub << 4), x, n, 0);
      it.sub = sub; it.rank = rank; it.disk = d; it.tile = 0;
      it.key = (double)P / tot;
      L.push_back(it);
   };
   auto base = [&](int sub, int d){ return sub ? W*((long)b->disk_Nr[d] + 4) + 8 : 8L; };
   for( int d=0 ; d<nd ; ++d ) add(PS_DBEGIN, 0, 0, d, 1, d, 0);
   for( int sub=0 ; sub<2 ; ++sub ){
      for( int cb=0 ; cb<(int)b->cblk.size() ; ++cb ){
         int a = b->cblk[cb].x, d = b->ann_disk[a];
         long j = b->ann_j[a], B = base(sub, d);
         add(PS_BEGIN, sub, 1, cb, 1, d, B + W*j);
         add(PS_GRAD, sub, 4, cb, 1, d, B + W*(j+1) + 3);
         add(PS_C2P, sub, 7, cb, 1, d, B + W*(j+2) + 6);
      }
      for( int d=0 ; d<nd ; ++d ){
         int a0 = b->dparams[d].ann0, na = b->disk_Nr[d]*b->disk_Nz[d];
         for( int a=a0 ; a<a0+na ; a+=4 ){
            int n = a0 + na - a < 4 ? a0 + na - a : 4;
            add(PS_I0, sub, 2, a, n, d, base(sub, d) + W*b->ann_j[a] + 1);
         }
      }
      for( int fb=0 ; fb<(int)b->fblk.size() ; ++fb ){
         int t = b->fblk[fb].x, d = b->ann_disk[b->tr_a[t]];
         long j = b->tr_j[t], B = base(sub, d);
         add(PS_FACES, sub, 3, fb, 1, d, B + W*(j+1) + 2);
         add(PS_FLUX, sub, 5, fb, 1, d, B + W*(j+2) + 4);
      }
      for( int ub=0 ; ub<(int)b->ublk.size() ; ++ub ){
         int a = b->ublk[ub].x, d = b->ann_disk[a];
         add(PS_UPDATE, sub, 6, ub, 1, d, base(sub, d) + W*(long)(b->ann_j[a]+2) + 5);
      }
   }
   for( int d=0 ; d<nd ; ++d ) add(PS_DMID, 0, 8, d, 1, d, W*((long)b->disk_Nr[d] + 4) + 4);
   if( b->nq ){
      for( int d=0 ; d<nd ; ++d ){
         int a0 = b->dparams[d].ann0, na = b->disk_Nr[d]*b->disk_Nz[d];
         for( int a=a0 ; a<a0+na ; a+=CB ){
            int n = a0 + na - a < CB ? a0 + na - a : CB;
            add(PS_DIAGFIN, 1, 8, a, n, d, base(1, d) + W*(long)(b->ann_j[a+n-1]+2) + 7);
         }
      }
   }
   for( int d=0 ; d<nd ; ++d ) add(PS_DTAIL, 1, 9, d, 1, d, 2*W*((long)b->disk_Nr[d] + 4) + 16);
   /* tiles of PERSIST_TILE grids' worth of items (DISCO_PERSIST_TILE in the
    * environment overrides it; a huge value gives one tile, i.e. stage by
    * stage over the whole batch) */
   long tf = PERSIST_TILE;
   if( const char *e = getenv("DISCO_PERSIST_TILE") ){ long x = atol(e); if( x > 0 ) tf = x; }
   long NT = (long)L.size() / (tf*G);
   if( NT < 1 ) NT = 1;
   for( It &it : L ){
      long tl = (long)(it.key*(double)NT);
      it.tile = (int)(tl < NT-1 ? tl : NT-1);
   }
   std::stable_sort(L.begin(), L.end(), [](const It &x, const It &y){
      if( x.tile != y.tile ) return x.tile < y.tile;
      if( x.sub != y.sub ) return x.sub < y.sub;
      if( x.rank != y.rank ) return x.rank < y.rank;
      if( x.key != y.key ) return x.key < y.key;
      if( x.disk != y.disk ) return x.disk < y.disk;
      return x.w.y < y.w.y;
   });
   std::vector<int4> items(L.size());
   for( size_t i=0 ; i<L.size() ; ++i ) items[i] = L[i].w;
   /* completion counters */
   PersistArgs &pa = b->pargs;
   memset(&pa, 0, sizeof pa);
   int o = 0;
   for( int sub=0 ; sub<2 ; ++sub ){
      pa.o_begin[sub] = o; o += nann;
      pa.o_I0[sub] = o;    o += nann;
      pa.o_faces[sub] = o; o += ntr;
      pa.o_grad[sub] = o;  o += nann;
      pa.o_flux[sub] = o;  o += ntr;
      pa.o_upd[sub] = o;   o += nann;
      pa.o_c2p[sub] = o;   o += nann;
      pa.o_c2pd[sub] = o;  o += nd;
   }
   pa.o_d0 = o; o += nd;
   pa.o_d1 = o; o += nd;
   int octl = o; o += 2;
   b->d_pcnt = dalloc<int>(b, (size_t)o);
   b->pcnt_bytes = (size_t)o*sizeof(int);
   b->d_pitems = dupload(b, items);
   b->pnitems = (int)items.size();
   b->pgrid = (int)G;
   pa.items = b->d_pitems;
   pa.nitems = b->pnitems;
   pa.cnt = b->d_pcnt;
   pa.ctl = b->d_pcnt + octl;
   pa.nc = b->d_ann_nblk;
   pa.nu = dupload(b, nu);
   pa.nf = dupload(b, nf);
   pa.ndc = dupload(b, ndc);
   pa.Qrz = b->d_Qrz;
   pa.ann_blk0 = b->d_ann_blk0;
   pa.ann_nblk = b->d_ann_nblk;
   pa.bc = b->bc_fixed;
   pa.diag = !b->bc_zerograd;
   if( !b->d_pcnt || !b->d_pitems || !pa.nu || !pa.nf || !pa.ndc ) return DISCO_ERR_CUDA;
   b->persist_ok = 1;
   return DISCO_OK;
}

extern "C" int disco_batch_create(int device, const disco_modules *mods, int precision,
                                  int ndisk, const disco_params *params,
                                  const int *Nr, const int *Nz, const int *Ng,
                                  const int *Np, const double *r_jph, const double *z_kph,
                                  disco_batch **out){
   if( !mods || !params || !Nr || !Nz || !Ng || !Np || !r_jph || !z_kph || !out || ndisk < 1 )
      return DISCO_ERR_ARG;
   *out = NULL;
   int ndev = 0;
   if( cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1 ) return DISCO_ERR_NO_DEVICE;
   if( device < 0 || device >= ndev ) return DISCO_ERR_ARG;
   if( precision != DISCO_PREC_FP64 && precision != DISCO_PREC_MIXED ) return DISCO_ERR_ARG;
   /* euler (NUM_C 5) or mhd (NUM_C 8), NUM_N 1.  Without in.par
    * Constrained_Transport, B evolves through the fluxes and CT_MODE 1/2 only
    * sizes the reference's face-flux storage, which then never reaches the
    * cells; MHD builds need it (with CT_MODE 0, flip_fluxes, bfields.c:
    * 760-814, writes through zero-length Phi arrays into the cell's real
    * flag and the next cell's prims), so it is accepted.  Constrained
    * transport itself is built in both forms, for every disk of the batch
    * or none. */
   /* grmhd2 (HYDRO = grmhd2, NUM_C 8) carries B like mhd; it is built for
    * the FP64 path with the HLL solver, without constrained transport or
    * point masses, for the schw_ks_rpz metric and the Kerr-Schild one */
   const bool gr = mods->hydro == DISCO_HYDRO_GRMHD;
   bool mhd = mods->hydro == DISCO_HYDRO_MHD || gr;
   if( !((mods->hydro == DISCO_HYDRO_EULER && mods->num_c == 5) || (mhd && mods->num_c == 8)) ||
       mods->num_n != 1 || mods->ct_mode < 0 || mods->ct_mode > 2 )
      return DISCO_ERR_UNSUPPORTED;
   if( gr ){
      if( precision != DISCO_PREC_FP64 || params[0].CT || mods->planets != DISCO_PLANETS_NONE ||
          mods->analysis == DISCO_DIAG_MHDMRI ||
          (mods->metric != DISCO_METRIC_SCHW_KS_RPZ && mods->metric != DISCO_METRIC_KERR_KS_RPZ) )
         return DISCO_ERR_UNSUPPORTED;
      for( int d=0 ; d<ndisk ; ++d ) if( params[d].Riemann_Solver != 0 ) return DISCO_ERR_UNSUPPORTED;
   }
   int ct = params[0].CT ? mods->ct_mode : 0;
   for( int d=0 ; d<ndisk ; ++d ) if( (params[d].CT ? 1 : 0) != (params[0].CT ? 1 : 0) ) return DISCO_ERR_ARG;
   if( params[0].CT ){
      /* CT_MODE 1 stores no z-face fluxes, so it is built for 2D disks */
      if( !mhd || mods->ct_mode < 1 ) return DISCO_ERR_UNSUPPORTED;
      for( int d=0 ; d<ndisk ; ++d )
         if( Nz[d] > 1 && mods->ct_mode != 2 ) return DISCO_ERR_UNSUPPORTED;
   }
   if( mods->boundary < DISCO_BC_FIXED || mods->boundary > DISCO_BC_FLOWTHROUGH )
      return DISCO_ERR_UNSUPPORTED;
   /* tube sets no inner r ghosts (Boundary/tube.c): grids without them */
   if( mods->boundary == DISCO_BC_TUBE )
      for( int d=0 ; d<ndisk ; ++d ) if( Ng[4*d+0] != 0 ) return DISCO_ERR_UNSUPPORTED;
   /* polar3d, horizon, horizon3d and horizon_bin set the outer r and the z
    * ghosts only (Boundary/polar3d.c, horizon.c, horizon3d.c,
    * horizon_bin.c): grids without inner ghosts */
   if( mods->boundary == DISCO_BC_POLAR3D || mods->boundary == DISCO_BC_HORIZON ||
       mods->boundary == DISCO_BC_HORIZON3D || mods->boundary == DISCO_BC_HORIZON_BIN )
      for( int d=0 ; d<ndisk ; ++d ) if( Ng[4*d+0] != 0 ) return DISCO_ERR_UNSUPPORTED;
   /* Boundary/polar.c sets the outer r and the z ghosts only: it is meant
    * for a grid whose inner edge is the axis (NoBC_Rmin 1, no inner ghosts);
    * with inner ghosts their prims would never be set */
   if( mods->boundary == DISCO_BC_POLAR )
      for( int d=0 ; d<ndisk ; ++d ) if( Ng[4*d+0] != 0 ) return DISCO_ERR_UNSUPPORTED;
   if( mods->analysis == DISCO_DIAG_MHDMRI && !mhd ) return DISCO_ERR_UNSUPPORTED;   /* reads B */
   if( mods->initial != DISCO_IC_KEPLER_NOISE && mods->initial != DISCO_IC_MHD_SHEAR_NOISE &&
       mods->initial != DISCO_IC_GR_TORUS_NOISE && mods->initial != DISCO_IC_HOST )
      return DISCO_ERR_UNSUPPORTED;
   if( mods->initial == DISCO_IC_GR_TORUS_NOISE && !gr ) return DISCO_ERR_UNSUPPORTED;
   /* a host-evaluated Initial module cannot refill ghosts on the device */
   if( mods->initial == DISCO_IC_HOST && mods->boundary != DISCO_BC_ZEROGRAD &&
       mods->boundary != DISCO_BC_OUTFLOW3D )
      return DISCO_ERR_UNSUPPORTED;
   for( int d=0 ; d<ndisk ; ++d ){
      if( Nr[d] < 2 ) return DISCO_ERR_ARG;
      if( params[d].Timestep != params[0].Timestep ) return DISCO_ERR_ARG;
      if( params[d].R_Periodic ) return DISCO_ERR_UNSUPPORTED;
      /* periodic z is MPI's exchangeData (exchange.c:174-175): in the serial
       * reference it copies nothing and the z ghosts are never set */
      if( params[d].Z_Periodic && Nz[d] > 1 ) return DISCO_ERR_UNSUPPORTED;
      if( params[d].Riemann_Solver > (mhd ? 2 : 1) ) return DISCO_ERR_UNSUPPORTED;   /* HLLD needs B */
      /* viscosity is the Euler module's (Hydro/mhd.c has none) */
      if( (params[d].visc_flag && mhd) || params[d].RotFrame ) return DISCO_ERR_UNSUPPORTED;
   }
   CK(cudaSetDevice(device));
   disco_batch *b = new disco_batch();
   b->device = device; b->mods = *mods; b->prec = precision; b->ndisk = ndisk;
   b->NC = mods->num_c; b->Q = mods->num_c + mods->num_n;
   b->timestep_mode = params[0].Timestep == 1 ? 1 : 0;
   /* the fixed ghost sets of fixed_ghost_init: polar3d is accrete3d's fixed
    * set (boundary_fixed_rout / _zbot / _ztop) without its inner copy */
   b->bc_fixed = mods->boundary == DISCO_BC_FIXED ? 1 : mods->boundary == DISCO_BC_FIXED3D ? 2 :
                 mods->boundary == DISCO_BC_POLAR ? 3 :
                 (mods->boundary == DISCO_BC_ACCRETE3D || mods->boundary == DISCO_BC_POLAR3D) ? 6 :
                 mods->boundary == DISCO_BC_HORIZON ? 8 : mods->boundary == DISCO_BC_HORIZON3D ? 9 :
                 mods->boundary == DISCO_BC_HORIZON_BIN ? 10 :
                 side_fixed_mask(mods->boundary) ? 11 : 0;
   /* modules built from boundary_functions.c's copies (zero-gradient, with
    * or without the outflow diode, and mirror copies): the sides whose
    * ghosts k_zerograd fills */
   b->bc_zerograd = 0;
   for( int s=0 ; s<4 ; ++s ) if( side_copies(side_mode(mods->boundary, s)) ) b->bc_zerograd = 1;
   b->zg_diode = 0;                          /* per pair (zg_side) */
   b->zg_omk = mods->boundary == DISCO_BC_ZEROGRAD_OMK;
   b->d_zg_side = NULL;
   b->d_noise = NULL;
   b->any_visc = 0;
   for( int d=0 ; d<ndisk ; ++d ) if( params[d].visc_flag ) b->any_visc = 1;
   b->gr = gr ? 1 : 0;
   b->d_zg_pairs = NULL;
   b->zg_smem = 0;
   b->nq = mods->analysis == DISCO_DIAG_DISK2D ? 5 : mods->analysis == DISCO_DIAG_EULER ? 8 :
           mods->analysis == DISCO_DIAG_MHDMRI ? 18 : 0;
   b->params.assign(params, params + ndisk);
   b->any_mm3 = 0;
   b->any_3d = 0;
   b->graph = NULL;
   b->have_cells = 0;
   b->stream = NULL;
   b->own_stream = NULL;
   b->tape = NULL; b->tape_names = NULL;
   b->ct = ct;
   b->nfs = ct == 2 ? 5 : 3;
   b->line_ne = 0;

   /* ---- topology */
   int cell = 0, ann = 0, face = 0, roff = 0, zoff = 0, npoff = 0;
   b->ncell = 0; b->nreal = 0;
   std::vector<DiskState> dstate(ndisk);
   b->dparams.resize(ndisk);
   for( int d=0 ; d<ndisk ; ++d ){
      const disco_params &p = params[d];
      DiskParams &D = b->dparams[d];
      fill_disk_params(D, p, *mods);
      memset(&dstate[d], 0, sizeof(DiskState));
      init_planets(dstate[d], D, p, *mods);
      dstate[d].t = p.t_min;
      if( p.Mesh_Motion == 3 ) b->any_mm3 = 1;
      int nr = Nr[d], nz = Nz[d];
      D.Nr = nr; D.Nz = nz;
      D.NgRa = Ng[4*d+0]; D.NgRb = Ng[4*d+1]; D.NgZa = Ng[4*d+2]; D.NgZb = Ng[4*d+3];
      D.ann0 = ann; D.cell0 = cell;
      D.rj0 = roff; D.zk0 = zoff;
      for( int j=0 ; j<=nr ; ++j ) b->rj.push_back(r_jph[roff + j]);
      for( int k=0 ; k<=nz ; ++k ) b->zk.push_back(z_kph[zoff + k]);
      int nreal = 0;
      for( int k=0 ; k<nz ; ++k ) for( int j=0 ; j<nr ; ++j ){
         int np = Np[npoff + j + nr*k];
         if( np < 4 ){ delete b; return DISCO_ERR_ARG; }
         b->ann_off.push_back(cell); b->ann_np.push_back(np); b->ann_disk.push_back(d);
         b->ann_j.push_back(j); b->ann_k.push_back(k);
         b->ann_blk0.push_back((int)b->cblk.size());
         int nb = 0;
         for( int i0=0 ; i0<np ; i0+=CB ){ b->cblk.push_back(make_int2(ann, i0)); ++nb; }
         for( int i0=0 ; i0<np ; i0+=CB-1 ) b->ublk.push_back(make_int2(ann, i0));
         b->ann_nblk.push_back(nb);
         if( j >= D.NgRa && j < nr-D.NgRb && k >= D.NgZa && k < nz-D.NgZb ) nreal += np;
         cell += np; ++ann;
      }
      /* r tracks (faces_alt.c:87-100): (Nr-1)*Nz tracks, track JK = j + (Nr-1)*k */
      D.trr0 = (int)b->tr_a.size();
      D.ntrr = (nr-1)*nz;
      D.face_r0 = face;
      const double *rj = r_jph + roff + 1;
      int jmin = D.NgRa == 0 ? 0 : D.NgRa-1;            /* trans_flux, misc.c:459-471 */
      int jmax = D.NgRb == 0 ? nr-1 : nr-D.NgRb;
      /* with CT one more layer of fluxes outside the real cells (:449-471) */
      int kminr = ct ? (D.NgZa == 0 ? 0 : D.NgZa-1) : D.NgZa;
      int kmaxr = ct ? (D.NgZb == 0 ? nz : nz-D.NgZb+1) : nz-D.NgZb;
      for( int k=0 ; k<nz ; ++k ) for( int j=0 ; j<nr-1 ; ++j ){
         int t = (int)b->tr_a.size();
         int A = D.ann0 + j + nr*k, B = A + 1;
         b->tr_a.push_back(A); b->tr_b.push_back(B); b->tr_off.push_back(face);
         b->tr_j.push_back(j); b->tr_k.push_back(k);
         b->tr_flux.push_back(j >= jmin && j < jmax && k >= kminr && k < kmaxr);
         /* dxL/dxR, faces_alt.c:112-118 */
         double rm = 2.0*(rj[j]*rj[j] + rj[j]*rj[j-1] + rj[j-1]*rj[j-1]) / (3.0*(rj[j]+rj[j-1]));
         double rp = 2.0*(rj[j+1]*rj[j+1] + rj[j+1]*rj[j] + rj[j]*rj[j]) / (3.0*(rj[j+1]+rj[j]));
         b->tr_dxL.push_back(rj[j] - rm);
         b->tr_dxR.push_back(rp - rj[j]);
         b->tr_dim.push_back(1);
         push_track_r(b, .5*(rj[j]+rj[j]));              /* addFace cm[0], faces_alt.c:10-16 */
         int nf = b->ann_np[A] + b->ann_np[B];
         for( int f0=0 ; f0<nf ; f0+=FB ) b->fblk.push_back(make_int2(t, f0));
         face += nf;
      }
      /* z tracks (faces_alt.c:83-100 with dim 2): Nr*(Nz-1) tracks, track
       * JK = j + Nr*k joins (j,k) and (j,k+1) */
      D.trz0 = (int)b->tr_a.size();
      D.ntrz = nr*(nz-1);
      if( nz > 1 ) b->any_3d = 1;
      const double *zkp = z_kph + zoff + 1;
      int kminz = D.NgZa == 0 ? 0 : D.NgZa-1;           /* trans_flux dim 2, misc.c:474-489 */
      int kmaxz = D.NgZb == 0 ? nz-1 : nz-D.NgZb;
      int jminz = ct ? (D.NgRa == 0 ? 0 : D.NgRa-1) : D.NgRa;
      int jmaxz = ct ? (D.NgRb == 0 ? nr : nr-D.NgRb+1) : nr-D.NgRb;
      for( int k=0 ; k<nz-1 ; ++k ) for( int j=0 ; j<nr ; ++j ){
         int t = (int)b->tr_a.size();
         int A = D.ann0 + j + nr*k, B = A + nr;
         b->tr_a.push_back(A); b->tr_b.push_back(B); b->tr_off.push_back(face);
         b->tr_j.push_back(j); b->tr_k.push_back(k);
         b->tr_flux.push_back(j >= jminz && j < jmaxz && k >= kminz && k < kmaxz);
         /* dxL/dxR, faces_alt.c:119-125 */
         double zm = 0.5*(zkp[k]+zkp[k-1]);
         double zp = 0.5*(zkp[k+1]+zkp[k]);
         b->tr_dxL.push_back(zkp[k] - zm);
         b->tr_dxR.push_back(zp - zkp[k]);
         b->tr_dim.push_back(2);
         push_track_r(b, host_centroid_r(rj[j], rj[j-1]));
         int nf = b->ann_np[A] + b->ann_np[B];
         for( int f0=0 ; f0<nf ; f0+=FB ) b->fblk.push_back(make_int2(t, f0));
         face += nf;
      }
      /* (r, z) edge lines of make_edge_adjust (bfields.c:922-1125), line
       * j + (Nr-1)*k between annuli (j,k), (j+1,k), (j,k+1), (j+1,k+1) */
      D.ln0 = (int)b->line_off.size();
      if( ct == 2 && nz > 1 ){
         for( int k=0 ; k<nz-1 ; ++k ) for( int j=0 ; j<nr-1 ; ++j ){
            int A = D.ann0 + j + nr*k;
            b->line_off.push_back(b->line_ne);
            b->line_ne += b->ann_np[A] + b->ann_np[A+1] + b->ann_np[A+nr] + b->ann_np[A+nr+1];
         }
      }
      b->disk_Nr.push_back(nr); b->disk_Nz.push_back(nz); b->disk_nreal.push_back(nreal);
      b->nreal += nreal;
      roff += nr+1; zoff += nz+1; npoff += nr*nz;
   }
   b->ann_off.push_back(cell);
   b->tr_off.push_back(face);
   b->line_off.push_back(b->line_ne);
   b->ncell = cell;

   /* k_faces' block order: per disk and layer k, for each j the r track
    * (j,k)-(j+1,k) and the z track (j,k)-(j,k+1), so that the tracks reading
    * an annulus run close together and its cells are read from L2; and the
    * flux kernels' blocks, per direction, of the tracks with fluxes */
   for( int d=0 ; d<ndisk ; ++d ){
      const DiskParams &D = b->dparams[d];
      auto push = [&](int t){
         int nf = b->ann_np[b->tr_a[t]] + b->ann_np[b->tr_b[t]];
         for( int f0=0 ; f0<nf ; f0+=FB ) b->fblk_rz.push_back(make_int2(t, f0));
      };
      for( int k=0 ; k<D.Nz ; ++k ) for( int j=0 ; j<D.Nr ; ++j ){
         if( j < D.Nr-1 ) push(D.trr0 + j + (D.Nr-1)*k);
         if( k < D.Nz-1 ) push(D.trz0 + j + D.Nr*k);
      }
   }
   if( b->fblk_rz.size() != b->fblk.size() ){ delete b; return DISCO_ERR_INTERNAL; }
   for( const int2 &fb : b->fblk )
      if( b->tr_flux[fb.x] ) b->fblk_fl[b->tr_dim[fb.x] - 1].push_back(fb);

   /* zerograd layers (boundary_functions.c:269-440): r ghosts from the real
    * cells outwards, then z ghosts (all j, ghosts included); sides[] of each
    * pair: 0 inner r, 1 outer r, 2 lower z, 3 upper z */
   if( b->bc_zerograd ){
      int smode[4];
      for( int s=0 ; s<4 ; ++s ) smode[s] = side_mode(mods->boundary, s);
      /* zg_side: the side, | 4 with the diode, | 8 for a mirror copy, | 16
       * negating all three velocity components (no-slip); 32 marks a
       * window-only entry (pair (ghost, ghost)): flowthrough's azimuthal
       * fixed window, run as its own layer after every r copy, since the
       * second ghost layer copies the first before the window is set */
      auto flags = [&](int s){
         const int m = smode[s];
         return (unsigned char)(s | ((m == SIDE_ZG_DIODE || m == SIDE_ZG_DIODE_PHIWIN) ? 4 : 0) |
                                (side_mirror(m) ? 8 : 0) | (m == SIDE_NOSLIP ? 16 : 0));
      };
      int maxr = 0, maxz = 0;
      for( int d=0 ; d<ndisk ; ++d ){
         const DiskParams &D = b->dparams[d];
         maxr = std::max(maxr, std::max(D.NgRa, D.NgRb));
         if( D.Nz > 1 && !params[d].Z_Periodic ) maxz = std::max(maxz, std::max(D.NgZa, D.NgZb));
      }
      for( int l=0 ; l<maxr ; ++l ){
         b->zg_off.push_back((int)b->zg_pairs.size());
         for( int d=0 ; d<ndisk ; ++d ){
            const DiskParams &D = b->dparams[d];
            for( int k=0 ; k<D.Nz ; ++k ){
               int base = D.ann0 + D.Nr*k;
               /* a z ghost layer of a fixed z side ends fixed (the z pass runs
                * after the r copies), so its r ghosts need no copy */
               if( (k < D.NgZa && smode[2] == SIDE_FIXED) || (k >= D.Nz - D.NgZb && smode[3] == SIDE_FIXED) )
                  continue;
               if( l < D.NgRa && side_copies(smode[0]) ){
                  int j = D.NgRa-1-l, j1 = side_mirror(smode[0]) ? 2*D.NgRa-j-1 : j+1;
                  b->zg_pairs.push_back(make_int2(base+j, base+j1)); b->zg_side.push_back(flags(0));
               }
               if( l < D.NgRb && side_copies(smode[1]) ){
                  int j = D.Nr-D.NgRb+l, j1 = side_mirror(smode[1]) ? 2*(D.Nr-D.NgRb)-j-1 : j-1;
                  b->zg_pairs.push_back(make_int2(base+j, base+j1)); b->zg_side.push_back(flags(1));
               }
            }
         }
      }
      if( smode[1] == SIDE_ZG_DIODE_PHIWIN ){
         b->zg_off.push_back((int)b->zg_pairs.size());
         for( int d=0 ; d<ndisk ; ++d ){
            const DiskParams &D = b->dparams[d];
            for( int k=0 ; k<D.Nz ; ++k ){
               if( (k < D.NgZa && smode[2] == SIDE_FIXED) || (k >= D.Nz - D.NgZb && smode[3] == SIDE_FIXED) )
                  continue;
               for( int j=D.Nr-D.NgRb ; j<D.Nr ; ++j ){
                  int A = D.ann0 + j + D.Nr*k;
                  b->zg_pairs.push_back(make_int2(A, A)); b->zg_side.push_back((unsigned char)(1 | 32));
               }
            }
         }
      }
      for( int l=0 ; l<maxz ; ++l ){
         b->zg_off.push_back((int)b->zg_pairs.size());
         for( int d=0 ; d<ndisk ; ++d ){
            const DiskParams &D = b->dparams[d];
            if( D.Nz < 2 || params[d].Z_Periodic ) continue;
            for( int j=0 ; j<D.Nr ; ++j ){
               if( l < D.NgZa && side_copies(smode[2]) ){
                  int k = D.NgZa-1-l, k1 = side_mirror(smode[2]) ? 2*D.NgZa-k-1 : k+1;
                  b->zg_pairs.push_back(make_int2(D.ann0 + j + D.Nr*k, D.ann0 + j + D.Nr*k1));
                  b->zg_side.push_back(flags(2));
               }
               if( l < D.NgZb && side_copies(smode[3]) ){
                  int k = D.Nz-D.NgZb+l, k1 = side_mirror(smode[3]) ? 2*(D.Nz-D.NgZb)-k-1 : k-1;
                  b->zg_pairs.push_back(make_int2(D.ann0 + j + D.Nr*k, D.ann0 + j + D.Nr*k1));
                  b->zg_side.push_back(flags(3));
               }
            }
         }
      }
      b->zg_off.push_back((int)b->zg_pairs.size());
      size_t sm = 0;
      for( const int2 &pr : b->zg_pairs ){
         size_t n0 = b->ann_np[pr.x], n1 = b->ann_np[pr.y];
         sm = std::max(sm, 16*(n0 + n1) + 8*n0);
      }
      b->zg_smem = (sm + 15) & ~(size_t)15;
      if( b->zg_smem > 200*1024 ){ delete b; return DISCO_ERR_UNSUPPORTED; }
   }

   ViewT<double> &v = b->vd;
   memset(&v, 0, sizeof v);
   v.Ncell = cell; v.Nann = ann; v.Ntr = (int)b->tr_a.size(); v.Nf = face;
   v.nq = b->nq;
   v.dtfac = 1.0;
   v.ann_off = dupload(b, b->ann_off); v.ann_np = dupload(b, b->ann_np);
   v.ann_disk = dupload(b, b->ann_disk); v.ann_j = dupload(b, b->ann_j); v.ann_k = dupload(b, b->ann_k);
   v.tr_a = dupload(b, b->tr_a); v.tr_b = dupload(b, b->tr_b); v.tr_off = dupload(b, b->tr_off);
   v.tr_flux = dupload(b, b->tr_flux); v.tr_j = dupload(b, b->tr_j); v.tr_k = dupload(b, b->tr_k);
   v.tr_dxL = dupload(b, b->tr_dxL); v.tr_dxR = dupload(b, b->tr_dxR);
   v.tr_dim = dupload(b, b->tr_dim);
   v.tr_r = dupload(b, b->tr_r); v.tr_irf = dupload(b, b->tr_irf);
   for( int a=0 ; a<ann ; ++a ){
      const DiskParams &D = b->dparams[b->ann_disk[a]];
      const double *rjd = b->rj.data() + D.rj0 + 1;
      const int j = b->ann_j[a];
      b->ann_rc.push_back(host_centroid_r(rjd[j], rjd[j-1]));
   }
   v.ann_rc = dupload(b, b->ann_rc);
   v.cblk = dupload(b, b->cblk); v.fblk = dupload(b, b->fblk); v.ublk = dupload(b, b->ublk);
   b->d_fblk_rz = dupload(b, b->fblk_rz);
   b->d_fblk_fl[0] = dupload(b, b->fblk_fl[0]); b->d_fblk_fl[1] = dupload(b, b->fblk_fl[1]);
   v.rj = dupload(b, b->rj); v.zk = dupload(b, b->zk);
   v.dp = dupload(b, b->dparams);
   v.ds = dupload(b, dstate);
   b->d_ann_blk0 = dupload(b, b->ann_blk0); b->d_ann_nblk = dupload(b, b->ann_nblk);
   size_t N = (size_t)cell, Qn = (size_t)b->Q*N, Qf = (size_t)b->Q*face;
   size_t rs = precision == DISCO_PREC_MIXED ? sizeof(float) : sizeof(double);
   v.prim = (double *)dalloc_bytes(b, Qn*rs);
   v.gradp = (double *)dalloc_bytes(b, Qn*rs);
   v.gradr = (double *)dalloc_bytes(b, Qn*rs);
   v.gradz = b->any_3d ? (double *)dalloc_bytes(b, Qn*rs) : NULL;
   v.fS = (double *)dalloc_bytes(b, Qf*rs);
   v.fG = (double *)dalloc_bytes(b, Qf*rs);
   v.cons = dalloc<double>(b, Qn); v.RKcons = dalloc<double>(b, Qn);
   v.ccarry = precision == DISCO_PREC_MIXED ? dalloc<float>(b, Qn) : NULL;
   v.piph = dalloc<double>(b, N); v.dphi = dalloc<double>(b, N);
   v.wiph = dalloc<double>(b, N); v.piph_new = dalloc<double>(b, N);
   v.I0 = dalloc<int>(b, ann);
   v.consL = dalloc<int>(b, N); v.consR = dalloc<int>(b, N);
   v.consZL = b->any_3d ? dalloc<int>(b, N) : NULL;
   v.consZR = b->any_3d ? dalloc<int>(b, N) : NULL;
   v.fL = dalloc<int>(b, face); v.fR = dalloc<int>(b, face);
   v.fLR = dalloc<unsigned char>(b, face);
   v.fphic = dalloc<double>(b, face); v.fdA = dalloc<double>(b, face); v.fdp = dalloc<double>(b, face);
   v.diag_part = dalloc<double>(b, b->cblk.size()*DIAG_SLOTS);
   v.ann_om = dalloc<double>(b, ann); v.ann_om1 = dalloc<double>(b, ann);
   v.tr_om = dalloc<double>(b, v.Ntr);
   b->d_Qrz = dalloc<double>(b, (size_t)ann*(b->nq ? b->nq : 1));
   v.err = dalloc<int>(b, 1);
   b->d_err = v.err;
   if( b->gr ){
      v.gr_ann = dalloc<GRAnn>(b, ann);
      v.gr_tr = dalloc<Metric3>(b, v.Ntr > 0 ? v.Ntr : 1);
   }
   v.topo = dalloc<int>(b, 1);
   if( mods->boundary == DISCO_BC_HORIZON_BIN )        /* the sticky not-real flags (zeroed) */
      v.xflag = dalloc<unsigned char>(b, N);
   if( ct ){
      v.ct = ct;
      v.nfs = b->nfs;
      size_t ne = ct == 2 ? 8 : 4;
      auto ralloc = [&](size_t n){ return (double *)dalloc_bytes(b, n*rs); };   /* R-typed */
      v.Phi = dalloc<double>(b, b->nfs*N); v.RKPhi = dalloc<double>(b, b->nfs*N);
      v.ctE = ralloc(ne*N); v.ctB = ralloc(ne*N);
      v.pE = ralloc(N); v.pB = ralloc(N);
      v.fEt = ralloc(face); v.fBt = ralloc(face);
      v.fX = dalloc<double>(b, face);
      v.fFlip = dalloc<unsigned char>(b, face);
      if( ct == 2 ){
         v.pEr = ralloc(N); v.pBz = ralloc(N);
         v.fEphi = ralloc(face);
         /* avg_Efields' z-pole branch: the annuli of a z boundary without
          * ghosts (bottom layer when NgZa = 0, top when NgZb = 0) */
         for( int d=0 ; d<ndisk ; ++d ){
            const DiskParams &D = b->dparams[d];
            if( D.Nz < 2 ) continue;
            for( int j=0 ; j<D.Nr ; ++j ){
               if( D.NgZa == 0 ) b->zpole.push_back(make_int2(D.ann0 + j, 0));
               if( D.NgZb == 0 ) b->zpole.push_back(make_int2(D.ann0 + j + D.Nr*(D.Nz-1), 1));
            }
         }
         if( !b->zpole.empty() ){
            v.ctPole = dalloc<double>(b, N);
            b->d_zpole = dupload(b, b->zpole);
         }
         if( b->any_3d ){
            v.rk = dalloc<int>(b, 4*N);
            v.lineX = dalloc<double>(b, (size_t)b->line_ne);
            v.line_off = dupload(b, b->line_off);
         }
      }
   }
   if( b->bc_zerograd && !b->zg_pairs.empty() ){
      b->d_zg_pairs = dupload(b, b->zg_pairs);
      b->d_zg_side = dupload(b, b->zg_side);
   }
   make_float_view(b);
   if( prepare_zerograd<6,double>(b) || prepare_zerograd<9,double>(b) ||
       (precision == DISCO_PREC_MIXED && mixed_prepare_zerograd(b)) ){
      disco_batch_destroy(b); return DISCO_ERR_CUDA;
   }
   for( void *p : b->allocs ) if( !p ){ disco_batch_destroy(b); return DISCO_ERR_CUDA; }
   if( cudaStreamCreateWithFlags(&b->own_stream, cudaStreamNonBlocking) != cudaSuccess ){
      disco_batch_destroy(b); return DISCO_ERR_CUDA;
   }
   b->stream = b->own_stream;
   {
      int nx = ann > v.Ntr ? ann : v.Ntr;
      k_precompute<<<nblk(nx, 128), 128, 0, b->stream>>>(v);
      if( b->gr ) k_gr_tables<double><<<nblk(nx, 128), 128, 0, b->stream>>>(v);
      k_planet_trig<double><<<nblk(ndisk, 64), 64, 0, b->stream>>>(v, ndisk);
   }
   /* the multi-kernel schedule is the default: on ragged64 the persistent
    * step measured 8.3 ms against 4.8 ms (FP64) and 7.2-7.9 against 3.9 ms
    * (mixed) in every tile size, stage-by-stage order included -- its one
    * register budget (64, with spills) keeps 8 CTAs per SM where the
    * separate kernels run 8-16, and each item adds two barriers, a fence
    * and the counter traffic */
   b->sched = DISCO_SCHED_KERNELS;
   if( persist_eligible(b) && build_persist_plan(b) != DISCO_OK ){ disco_batch_destroy(b); return DISCO_ERR_CUDA; }
   if( cudaDeviceSynchronize() != cudaSuccess ){ disco_batch_destroy(b); return DISCO_ERR_CUDA; }
   *out = b;
   return DISCO_OK;
}

extern "C" int disco_batch_set_schedule(disco_batch *b, int sched){
   if( !b ) return DISCO_ERR_ARG;
   if( sched != DISCO_SCHED_KERNELS && sched != DISCO_SCHED_PERSISTENT ) return DISCO_ERR_ARG;
   if( sched == DISCO_SCHED_PERSISTENT && !b->persist_ok ) return DISCO_ERR_UNSUPPORTED;
   if( sched == b->sched ) return DISCO_OK;
   CK(cudaSetDevice(b->device));
   CK(cudaStreamSynchronize(b->stream));
   if( b->graph ){ cudaGraphExecDestroy(b->graph); b->graph = NULL; }   /* recaptured on the next run */
   b->sched = sched;
   return DISCO_OK;
}

extern "C" int disco_batch_set_gr_dump(disco_batch *b, double *dev){
   if( !b ) return DISCO_ERR_ARG;
   if( !b->gr ) return DISCO_ERR_UNSUPPORTED;
   CK(cudaSetDevice(b->device));
   if( dev ){                       /* device memory of this batch's GPU */
      cudaPointerAttributes at;
      if( cudaPointerGetAttributes(&at, dev) != cudaSuccess || at.type != cudaMemoryTypeDevice ||
          at.device != b->device ){
         cudaGetLastError();
         return DISCO_ERR_ARG;
      }
   }
   CK(cudaStreamSynchronize(b->stream));
   if( b->graph ){ cudaGraphExecDestroy(b->graph); b->graph = NULL; }   /* recaptured on the next run */
   b->vd.gr_dump = dev;
   return DISCO_OK;
}

extern "C" int disco_batch_get_schedule(const disco_batch *b, int *sched){
   if( !b || !sched ) return DISCO_ERR_ARG;
   *sched = b->sched;
   return DISCO_OK;
}

extern "C" void disco_batch_destroy(disco_batch *b){
   if( !b ) return;
   cudaSetDevice(b->device);
   if( b->graph ) cudaGraphExecDestroy(b->graph);
   if( b->own_stream ) cudaStreamDestroy(b->own_stream);
   for( void *p : b->allocs ) if( p ) cudaFree(p);
   if( b->d_stage ) cudaFree(b->d_stage);
   if( b->d_rpart ) cudaFree(b->d_rpart);
   if( b->d_rout ) cudaFree(b->d_rout);
   delete b;
}

extern "C" int disco_batch_sizes(const disco_batch *b, int64_t *ncell, int64_t *nreal, int *q){
   if( !b ) return DISCO_ERR_ARG;
   if( ncell ) *ncell = b->ncell;
   if( nreal ) *nreal = b->nreal;
   if( q ) *q = b->Q;
   return DISCO_OK;
}

/* Host <-> device copy ordered on the batch's stream (which may be a
 * non-blocking stream of the caller), completed before returning. */
static cudaError_t xfer(const disco_batch *b, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind){
   cudaError_t e = cudaMemcpyAsync(dst, src, bytes, kind, b->stream);
   if( e != cudaSuccess ) return e;
   return cudaStreamSynchronize(b->stream);
}

/* cell-major FP64 (Q per cell) host <-> SoA device of element type T: one
 * contiguous copy through a device staging array (DMA at full speed when the
 * host buffer is pinned), transposed on the device, one thread per cell. */
template<class T>
__global__ void k_aos_to_soa(const double *src, T *dst, size_t N, int Q){
   size_t c = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
   if( c >= N ) return;
   for( int q=0 ; q<Q ; ++q ) dst[q*N + c] = (T)src[c*Q + q];
}
template<class T>
__global__ void k_soa_to_aos(const T *src, double *dst, size_t N, int Q){
   size_t c = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
   if( c >= N ) return;
   for( int q=0 ; q<Q ; ++q ) dst[c*Q + q] = (double)src[q*N + c];
}
static int staging(disco_batch *b){
   if( b->d_stage ) return DISCO_OK;
   const size_t w = (size_t)(b->Q > b->nfs ? b->Q : b->nfs);
   if( cudaMalloc(&b->d_stage, w*b->ncell*sizeof(double)) != cudaSuccess ){
      b->d_stage = NULL;
      return DISCO_ERR_CUDA;
   }
   return DISCO_OK;
}
template<class T>
static int upload_q(disco_batch *b, T *dst, const double *src, int Q = 0){
   size_t N = b->ncell;
   if( Q == 0 ) Q = b->Q;
   int s = staging(b);
   if( s ) return s;
   CK(cudaMemcpyAsync(b->d_stage, src, (size_t)Q*N*sizeof(double), cudaMemcpyHostToDevice, b->stream));
   k_aos_to_soa<T><<<nblk(N, 256), 256, 0, b->stream>>>(b->d_stage, dst, N, Q);
   CK(cudaGetLastError());
   CK(cudaStreamSynchronize(b->stream));
   return DISCO_OK;
}
template<class T>
static int download_q(disco_batch *b, double *dst, const T *src, int Q = 0){
   size_t N = b->ncell;
   if( Q == 0 ) Q = b->Q;
   int s = staging(b);
   if( s ) return s;
   k_soa_to_aos<T><<<nblk(N, 256), 256, 0, b->stream>>>(src, b->d_stage, N, Q);
   CK(cudaGetLastError());
   CK(xfer(b, dst, b->d_stage, (size_t)Q*N*sizeof(double), cudaMemcpyDeviceToHost));
   return DISCO_OK;
}
/* an R-typed cell array of the batch (prim, gradp, gradr) */
static int upload_r(disco_batch *b, double *dev, const double *src){
   if( b->prec == DISCO_PREC_MIXED ) return upload_q<float>(b, (float *)dev, src);
   return upload_q<double>(b, dev, src);
}
static int download_r(disco_batch *b, double *dst, const double *dev){
   if( b->prec == DISCO_PREC_MIXED ) return download_q<float>(b, dst, (const float *)dev);
   return download_q<double>(b, dst, dev);
}

extern "C" int disco_batch_set_cells(disco_batch *b, const double *prim, const double *cons,
                                     const double *piph, const double *dphi, const double *wiph,
                                     const int *real, const double *Phi){
   if( !b || !piph || !dphi ) return DISCO_ERR_ARG;
   (void)real;
   CK(cudaSetDevice(b->device));
   size_t N = b->ncell;
   int s;
   if( prim && (s = upload_r(b, b->vd.prim, prim)) ) return s;
   if( cons && (s = upload_q<double>(b, b->vd.cons, cons)) ) return s;
   if( b->ct ){                     /* Phi[0 .. num_faces-1] per cell, cell-major */
      if( Phi ){
         if( (s = upload_q<double>(b, b->vd.Phi, Phi, b->nfs)) ) return s;
      }else{
         CK(cudaMemsetAsync(b->vd.Phi, 0, (size_t)b->nfs*N*sizeof(double), b->stream));
      }
   }
   CK(xfer(b, b->vd.piph, piph, N*sizeof(double), cudaMemcpyHostToDevice));
   CK(xfer(b, b->vd.dphi, dphi, N*sizeof(double), cudaMemcpyHostToDevice));
   if( wiph ) CK(xfer(b, b->vd.wiph, wiph, N*sizeof(double), cudaMemcpyHostToDevice));
   if( b->vd.ccarry ) CK(cudaMemsetAsync(b->vd.ccarry, 0, (size_t)b->Q*N*sizeof(float), b->stream));
   CK(cudaMemsetAsync(b->vd.topo, 0, sizeof(int), b->stream));      /* new piph: faces stale */
   if( prim && !cons ){
      unsigned ncb = (unsigned)b->cblk.size();
      if( b->prec == DISCO_PREC_MIXED ) mixed_launch_prim2cons(b);
      else launch_prim2cons_t(b, b->vd);
      CK(cudaGetLastError());
   }
   CK(cudaStreamSynchronize(b->stream));
   b->have_cells = 1;
   return DISCO_OK;
}

extern "C" int disco_batch_get_cells(disco_batch *b, double *prim, double *cons,
                                     double *piph, double *dphi, double *wiph, double *Phi){
   if( !b ) return DISCO_ERR_ARG;
   CK(cudaSetDevice(b->device));
   CK(cudaStreamSynchronize(b->stream));
   size_t N = b->ncell;
   int s;
   if( Phi && b->ct && (s = download_q<double>(b, Phi, b->vd.Phi, b->nfs)) ) return s;
   if( prim && (s = download_r(b, prim, b->vd.prim)) ) return s;
   if( cons && (s = download_q<double>(b, cons, b->vd.cons)) ) return s;
   if( piph ) CK(xfer(b, piph, b->vd.piph, N*sizeof(double), cudaMemcpyDeviceToHost));
   if( dphi ) CK(xfer(b, dphi, b->vd.dphi, N*sizeof(double), cudaMemcpyDeviceToHost));
   if( wiph ) CK(xfer(b, wiph, b->vd.wiph, N*sizeof(double), cudaMemcpyDeviceToHost));
   return DISCO_OK;
}

static int launch_mindt(disco_batch *b){
   if( b->prec == DISCO_PREC_MIXED ) mixed_launch_mindt(b);
   else launch_mindt_t(b, b->vd);
   return cuda_status(cudaGetLastError());
}

/* a disk with Noise_Type 1-3 needs its addNoise draws (disco_batch_set_noise) */
static bool noise_missing(const disco_batch *b){
   if( b->vd.noise ) return false;
   for( int d=0 ; d<b->ndisk ; ++d ) if( b->dparams[d].noise_type ) return true;
   return false;
}

extern "C" int disco_batch_set_noise(disco_batch *b, const double *noise){
   if( !b ) return DISCO_ERR_ARG;
   CK(cudaSetDevice(b->device));
   if( !noise ){ b->vd.noise = NULL; b->vf.noise = NULL; return DISCO_OK; }
   size_t bytes = sizeof(double)*4*(size_t)b->ncell;
   if( !b->d_noise ){
      b->d_noise = (double *)dalloc_bytes(b, bytes);
      if( !b->d_noise ) return DISCO_ERR_CUDA;
   }
   CK(xfer(b, b->d_noise, noise, bytes, cudaMemcpyHostToDevice));
   b->vd.noise = b->d_noise; b->vf.noise = b->d_noise;
   return DISCO_OK;
}

extern "C" int disco_batch_setup_cells(disco_batch *b){
   if( !b ) return DISCO_ERR_ARG;
   if( b->mods.initial == DISCO_IC_HOST ) return DISCO_ERR_UNSUPPORTED;   /* set up on the host */
   if( noise_missing(b) ) return DISCO_ERR_STATE;
   CK(cudaSetDevice(b->device));
   CK(cudaMemsetAsync(b->vd.topo, 0, sizeof(int), b->stream));
   if( b->prec == DISCO_PREC_MIXED ) mixed_launch_setup(b);
   else launch_setup_t(b, b->vd);
   CK(cudaGetLastError());
   int s = launch_mindt(b);
   if( s ) return s;
   CK(cudaStreamSynchronize(b->stream));
   b->have_cells = 1;
   return DISCO_OK;
}

static int read_err(disco_batch *b){
   int e = 0;
   if( xfer(b, &e, b->d_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ) return DISCO_ERR_CUDA;
   if( e ){
      int z = 0;
      xfer(b, b->d_err, &z, sizeof(int), cudaMemcpyHostToDevice);
   }
   if( e & ERRF_WRAP ) return DISCO_ERR_PHI_WRAP;
   if( e & ERRF_NONFINITE ) return DISCO_ERR_NONFINITE;
   if( e & (ERRF_INTERNAL | ERRF_TIMEOUT) ) return DISCO_ERR_INTERNAL;
   return DISCO_OK;
}

extern "C" int disco_batch_mindt(disco_batch *b, double *dt){
   if( !b ) return DISCO_ERR_ARG;
   if( !b->have_cells ) return DISCO_ERR_STATE;
   CK(cudaSetDevice(b->device));
   int s = launch_mindt(b);
   if( s ) return s;
   CK(cudaStreamSynchronize(b->stream));
   if( dt ){
      std::vector<DiskState> st(b->ndisk);
      CK(xfer(b, st.data(), b->vd.ds, sizeof(DiskState)*b->ndisk, cudaMemcpyDeviceToHost));
      for( int d=0 ; d<b->ndisk ; ++d ) dt[d] = st[d].dt_next;
   }
   return read_err(b);
}

static void launch_step(disco_batch *b, int use_next){
   if( b->prec == DISCO_PREC_MIXED ) mixed_launch_step(b, use_next);
   else launch_step_t(b, b->vd, use_next);
}

extern "C" int disco_batch_timestep(disco_batch *b, const double *dt){
   if( !b ) return DISCO_ERR_ARG;
   if( !b->have_cells ) return DISCO_ERR_STATE;
   CK(cudaSetDevice(b->device));
   if( dt ){
      std::vector<DiskState> st(b->ndisk);
      CK(xfer(b, st.data(), b->vd.ds, sizeof(DiskState)*b->ndisk, cudaMemcpyDeviceToHost));
      for( int d=0 ; d<b->ndisk ; ++d ) st[d].dt_next = dt[d];
      CK(xfer(b, b->vd.ds, st.data(), sizeof(DiskState)*b->ndisk, cudaMemcpyHostToDevice));
   }
   launch_step(b, 1);
   CK(cudaGetLastError());
   return DISCO_OK;
}

extern "C" int disco_batch_run(disco_batch *b, int nsteps){
   if( !b || nsteps < 0 ) return DISCO_ERR_ARG;
   if( !b->have_cells ) return DISCO_ERR_STATE;
   CK(cudaSetDevice(b->device));
   if( !b->graph ){
      cudaGraph_t g;
      CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      launch_step(b, 1);
      CK(cudaStreamEndCapture(b->stream, &g));
      CK(cudaGraphInstantiate(&b->graph, g, 0));
      CK(cudaGraphDestroy(g));
   }
   for( int n=0 ; n<nsteps ; ++n ) CK(cudaGraphLaunch(b->graph, b->stream));
   CK(cudaGetLastError());
   return DISCO_OK;
}

extern "C" int disco_batch_time(const disco_batch *b, int disk, double *t, int *count){
   if( !b || disk < 0 || disk >= b->ndisk ) return DISCO_ERR_ARG;
   CK(cudaSetDevice(b->device));
   CK(cudaStreamSynchronize(b->stream));
   DiskState st;
   CK(xfer(b, &st, b->vd.ds + disk, sizeof st, cudaMemcpyDeviceToHost));
   if( t ) *t = st.t;
   if( count ) *count = st.count_steps;
   return DISCO_OK;
}

cudaError_t batch_xfer(const disco_batch *b, void *dst, const void *src, size_t bytes, cudaMemcpyKind kind){
   return xfer(b, dst, src, bytes, kind);
}

extern "C" int disco_batch_get_planets(disco_batch *b, int disk, double *rows, int cap, int *npl){
   if( !b || disk < 0 || disk >= b->ndisk ) return DISCO_ERR_ARG;
   CK(cudaSetDevice(b->device));
   int n = b->dparams[disk].npl;
   if( npl ) *npl = n;
   if( !rows ) return DISCO_OK;
   if( cap < n ) return DISCO_ERR_ARG;
   DiskState st;
   CK(xfer(b, &st, b->vd.ds + disk, sizeof st, cudaMemcpyDeviceToHost));
   for( int p=0 ; p<n ; ++p ){                     /* h5out.c:444-455 */
      const Planet &pl = st.pl[p];
      double *r = rows + DISCO_PLANET_COLS*p;
      r[0] = pl.M; r[1] = pl.vr; r[2] = pl.omega; r[3] = pl.r; r[4] = pl.phi; r[5] = pl.eps;
      r[6] = (double)pl.type;
   }
   return DISCO_OK;
}

extern "C" int disco_batch_set_planets(disco_batch *b, int disk, const double *rows, int npl){
   if( !b || !rows || disk < 0 || disk >= b->ndisk ) return DISCO_ERR_ARG;
   if( npl != b->dparams[disk].npl ) return DISCO_ERR_ARG;
   for( int p=0 ; p<npl ; ++p )
      if( rows[DISCO_PLANET_COLS*p + 6] != 0.0 ) return DISCO_ERR_UNSUPPORTED;   /* PLPOINTMASS only */
   CK(cudaSetDevice(b->device));
   DiskState st;
   CK(xfer(b, &st, b->vd.ds + disk, sizeof st, cudaMemcpyDeviceToHost));
   for( int p=0 ; p<npl ; ++p ){                   /* h5in.c:305-317 */
      Planet &pl = st.pl[p];
      const double *r = rows + DISCO_PLANET_COLS*p;
      pl.M = r[0]; pl.vr = r[1]; pl.omega = r[2]; pl.r = r[3]; pl.phi = r[4]; pl.eps = r[5];
      pl.type = 0;
   }
   CK(xfer(b, b->vd.ds + disk, &st, sizeof st, cudaMemcpyHostToDevice));
   k_planet_trig<double><<<nblk(b->ndisk, 64), 64, 0, b->stream>>>(b->vd, b->ndisk);
   CK(cudaGetLastError());
   CK(cudaStreamSynchronize(b->stream));
   return DISCO_OK;
}

extern "C" int disco_batch_set_time(disco_batch *b, int disk, double t){
   if( !b || disk < 0 || disk >= b->ndisk ) return DISCO_ERR_ARG;
   CK(cudaSetDevice(b->device));
   DiskState st;
   CK(xfer(b, &st, b->vd.ds + disk, sizeof st, cudaMemcpyDeviceToHost));
   st.t = t;
   CK(xfer(b, b->vd.ds + disk, &st, sizeof st, cudaMemcpyHostToDevice));
   return DISCO_OK;
}

extern "C" int disco_batch_restart_cells(disco_batch *b, const double *prim, const double *Phi,
                                         const double *piph){
   if( !b || !prim || !piph || (b->ct && !Phi) ) return DISCO_ERR_ARG;
   if( noise_missing(b) ) return DISCO_ERR_STATE;
   CK(cudaSetDevice(b->device));
   size_t N = b->ncell;
   int s;
   if( (s = upload_r(b, b->vd.prim, prim)) ) return s;
   if( b->ct ){
      const int F = b->nfs;
      std::vector<double> t(F*N);
      for( size_t c=0 ; c<N ; ++c ) for( int q=0 ; q<F ; ++q ) t[q*N + c] = Phi[F*c + q];
      CK(xfer(b, b->vd.Phi, t.data(), t.size()*sizeof(double), cudaMemcpyHostToDevice));
   }
   CK(xfer(b, b->vd.piph, piph, N*sizeof(double), cudaMemcpyHostToDevice));
   CK(cudaMemsetAsync(b->vd.topo, 0, sizeof(int), b->stream));
   /* diagnostics restart from zero (h5in.c:329-333), as does the step count
    * of a new process (domain.c:99) */
   std::vector<DiskState> st(b->ndisk);
   CK(xfer(b, st.data(), b->vd.ds, sizeof(DiskState)*b->ndisk, cudaMemcpyDeviceToHost));
   for( int d=0 ; d<b->ndisk ; ++d ){ st[d].t_avg = 0.0; st[d].count_steps = 0; }
   CK(xfer(b, b->vd.ds, st.data(), sizeof(DiskState)*b->ndisk, cudaMemcpyHostToDevice));
   if( b->nq ) CK(cudaMemsetAsync(b->d_Qrz, 0, sizeof(double)*b->nq*b->ann_np.size(), b->stream));
   if( b->prec == DISCO_PREC_MIXED ) mixed_launch_restart(b);
   else launch_restart_t(b, b->vd);
   CK(cudaGetLastError());
   s = launch_mindt(b);
   if( s ) return s;
   CK(cudaStreamSynchronize(b->stream));
   b->have_cells = 1;
   return read_err(b);
}

extern "C" int disco_batch_report(disco_batch *b, int disk, double *out){
   if( !b || !out || disk < 0 || disk >= b->ndisk ) return DISCO_ERR_ARG;
   if( !b->have_cells ) return DISCO_ERR_STATE;
   CK(cudaSetDevice(b->device));
   if( !b->d_rpart ){
      if( cudaMalloc(&b->d_rpart, b->cblk.size()*RP_N*sizeof(double)) != cudaSuccess ||
          cudaMalloc(&b->d_rout, (size_t)b->ndisk*17*sizeof(double)) != cudaSuccess )
         return DISCO_ERR_CUDA;
   }
   if( b->prec == DISCO_PREC_MIXED ) mixed_launch_report(b);
   else launch_report_t(b, b->vd);
   CK(cudaGetLastError());
   CK(xfer(b, out, b->d_rout + (size_t)disk*17, 17*sizeof(double), cudaMemcpyDeviceToHost));
   return read_err(b);
}

extern "C" int disco_batch_get_faces(disco_batch *b, int disk, int dim, int *nfaces,
                                     int *fIndex, int *iL, int *iR, int *LRtype, double *geom){
   if( !b || disk < 0 || disk >= b->ndisk || (dim != 1 && dim != 2) ) return DISCO_ERR_ARG;
   if( dim == 2 && b->disk_Nz[disk] < 2 ){ if( nfaces ) *nfaces = 0; return DISCO_OK; }
   CK(cudaSetDevice(b->device));
   const ViewT<double> &v = b->vd;
   unsigned nib = nblk((size_t)v.Nann*32, 128), nfb = (unsigned)b->fblk.size();
   if( b->prec == DISCO_PREC_MIXED ){
      mixed_launch_faces(b);
   }else{
      k_I0<double><<<nib, 128, 0, b->stream>>>(v);
      k_faces<6,double><<<nfb, FB, 0, b->stream>>>(v, 0);
   }
   CK(cudaGetLastError());
   CK(cudaStreamSynchronize(b->stream));
   const DiskParams &D = b->dparams[disk];
   int t0 = dim == 1 ? D.trr0 : D.trz0, nt = dim == 1 ? D.ntrr : D.ntrz;
   int f0 = b->tr_off[t0];
   int nf = b->tr_off[t0 + nt] - f0;
   if( nfaces ) *nfaces = nf;
   if( fIndex ) for( int t=0 ; t<=nt ; ++t ) fIndex[t] = b->tr_off[t0+t] - f0;
   std::vector<int> tl(nf), tr(nf);
   std::vector<unsigned char> tlr(nf);
   if( iL || iR || LRtype ){
      CK(xfer(b, tl.data(), v.fL + f0, nf*sizeof(int), cudaMemcpyDeviceToHost));
      CK(xfer(b, tr.data(), v.fR + f0, nf*sizeof(int), cudaMemcpyDeviceToHost));
      CK(xfer(b, tlr.data(), v.fLR + f0, nf, cudaMemcpyDeviceToHost));
      for( int n=0 ; n<nf ; ++n ){
         if( iL ) iL[n] = tl[n] - D.cell0;
         if( iR ) iR[n] = tr[n] - D.cell0;
         if( LRtype ) LRtype[n] = tlr[n];
      }
   }
   if( geom ){
      std::vector<double> phic(nf), dA(nf), dp(nf);
      CK(xfer(b, phic.data(), v.fphic + f0, nf*sizeof(double), cudaMemcpyDeviceToHost));
      CK(xfer(b, dA.data(), v.fdA + f0, nf*sizeof(double), cudaMemcpyDeviceToHost));
      CK(xfer(b, dp.data(), v.fdp + f0, nf*sizeof(double), cudaMemcpyDeviceToHost));
      const double *rj = b->rj.data() + D.rj0 + 1;
      const double *zk = b->zk.data() + D.zk0 + 1;
      for( int t=0 ; t<nt ; ++t ){
         int gt = t0 + t;
         int j = b->tr_j[gt], k = b->tr_k[gt];
         for( int f=b->tr_off[gt]-f0 ; f<b->tr_off[gt+1]-f0 ; ++f ){
            /* dxL, dxR, cm[0..2], dphi, dl, dA as addFace (faces_alt.c:10-34) */
            double *g = geom + 8*(size_t)f;
            g[0] = b->tr_dxL[gt]; g[1] = b->tr_dxR[gt];
            if( dim == 1 ){
               g[2] = .5*(rj[j]+rj[j]); g[3] = phic[f]; g[4] = 0.5*(zk[k]+zk[k-1]);
               g[5] = dp[f]; g[6] = zk[k]-zk[k-1]; g[7] = dA[f];
            }else{
               g[2] = 2.0*(rj[j]*rj[j] + rj[j]*rj[j-1] + rj[j-1]*rj[j-1])/(3.0*(rj[j]+rj[j-1]));
               g[3] = phic[f]; g[4] = .5*(zk[k]+zk[k]);
               g[5] = dp[f]; g[6] = rj[j]-rj[j-1]; g[7] = dA[f];
            }
         }
      }
   }
   return read_err(b);
}

extern "C" int disco_batch_get_diagnostics(disco_batch *b, int disk, double *Qrz, int *nq, double *t_avg){
   if( !b || disk < 0 || disk >= b->ndisk ) return DISCO_ERR_ARG;
   CK(cudaSetDevice(b->device));
   CK(cudaStreamSynchronize(b->stream));
   if( nq ) *nq = b->nq;
   const DiskParams &D = b->dparams[disk];
   int na = b->disk_Nr[disk]*b->disk_Nz[disk];
   if( Qrz && b->nq ) CK(xfer(b, Qrz, b->d_Qrz + (size_t)D.ann0*b->nq, sizeof(double)*na*b->nq,
                              cudaMemcpyDeviceToHost));
   if( t_avg ){
      DiskState st;
      CK(xfer(b, &st, b->vd.ds + disk, sizeof st, cudaMemcpyDeviceToHost));
      *t_avg = st.t_avg;
   }
   return DISCO_OK;
}

extern "C" int disco_batch_last_error(disco_batch *b){
   if( !b ) return DISCO_ERR_ARG;
   if( cudaSetDevice(b->device) != cudaSuccess ) return DISCO_ERR_CUDA;
   cudaError_t e = cudaStreamSynchronize(b->stream);
   if( e != cudaSuccess ) return DISCO_ERR_CUDA;
   return read_err(b);
}

extern "C" int disco_batch_debug_get(disco_batch *b, int which, double *out){
   if( !b || !out ) return DISCO_ERR_ARG;
   CK(cudaSetDevice(b->device));
   CK(cudaStreamSynchronize(b->stream));
   if( which == 0 ) return download_r(b, out, b->vd.gradp);
   if( which == 1 ) return download_r(b, out, b->vd.gradr);
   if( which == 2 ) return download_q<double>(b, out, b->vd.RKcons);
   return DISCO_ERR_ARG;
}

extern "C" int disco_batch_set_stream(disco_batch *b, void *stream){
   if( !b ) return DISCO_ERR_ARG;
   CK(cudaSetDevice(b->device));
   CK(cudaStreamSynchronize(b->stream));
   b->stream = stream ? (cudaStream_t)stream : b->own_stream;
   return DISCO_OK;
}

extern "C" int disco_batch_kernel_times(disco_batch *b, float *ms, const char **names,
                                        int cap, int *nlaunch){
   if( !b || !ms || !nlaunch || cap < 1 ) return DISCO_ERR_ARG;
   if( !b->have_cells ) return DISCO_ERR_STATE;
   CK(cudaSetDevice(b->device));
   std::vector<cudaEvent_t> ev;
   std::vector<const char *> nm;
   b->tape = &ev; b->tape_names = &nm;
   cudaEvent_t e0;
   CK(cudaEventCreate(&e0));
   CK(cudaEventRecord(e0, b->stream));
   ev.push_back(e0);
   launch_step(b, 1);
   b->tape = NULL; b->tape_names = NULL;
   CK(cudaGetLastError());
   CK(cudaStreamSynchronize(b->stream));
   int n = (int)nm.size();
   if( n > cap ) n = cap;
   for( int i=0 ; i<n ; ++i ){
      float t = 0.f;
      cudaEventElapsedTime(&t, ev[i], ev[i+1]);
      ms[i] = t;
      if( names ) names[i] = nm[i];
   }
   *nlaunch = n;
   for( cudaEvent_t e : ev ) cudaEventDestroy(e);
   return read_err(b);
}
