/*
 * Output and restart of the device-resident state, for one disk at a time:
 *   disco_batch_write_checkpoint   Output/h5out.c:349-598 (serial), in the
 *                                  .npz container of host/disco_npz.c
 *   disco_batch_write_ascii        Output/ascii.c:7-77
 *   disco_batch_restart            Restart/h5in.c:100-354, then setupCells
 *                                  with restart_flag (disco_batch_restart_cells)
 * The cell rows are packed on the device (one thread per cell, the row
 * layout of the file) and copied to the host through a pinned buffer in
 * chunks, so a checkpoint of any size needs one chunk of host staging.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>
#include <string>
#include <vector>
#include <functional>
#include "disco_batch_impl.cuh"
#include "disco_host.h"

#define CK(x) do{ cudaError_t _e = (x); if( _e != cudaSuccess ){ \
   fprintf(stderr, "disco_b200: %s failed: %s (%s:%d)\n", #x, cudaGetErrorString(_e), __FILE__, __LINE__); \
   return DISCO_ERR_CUDA; } }while(0)
#define CKS(x) do{ int _s = (x); if( _s ) return _s; }while(0)

/* NUM_FACES of the build (paul.h:33-49) */
static int num_faces(int ct_mode){ return ct_mode == 1 ? 3 : ct_mode == 2 ? 5 : 0; }

/* NUM_G (paul.h:30): ascii.c trims Ng layers of a z-periodic domain */
static const int NUM_G_GHOSTS = 2;

enum { ROWS_CELLS = 0, ROWS_ASCII = 1 };

/* One row per cell c0 .. c0+n-1:
 *   ROWS_CELLS  prim[Q] Phi[F] piph   (Cell2Doub, h5out.c:77-85; Phi zero
 *                                      when constrained transport is off)
 *   ROWS_ASCII  prim[Q] piph dphi     (what ascii.c prints besides the grid) */
template<class R>
__global__ void k_pack_rows(ViewT<R> v, size_t c0, size_t n, int Q, int F, int mode, double *out){
   size_t t = blockIdx.x*(size_t)blockDim.x + threadIdx.x;
   if( t >= n ) return;
   const size_t N = v.Ncell;
   size_t c = c0 + t;
   int ncol = mode == ROWS_CELLS ? Q + F + 1 : Q + 2;
   double *o = out + t*ncol;
   for( int q=0 ; q<Q ; ++q ) o[q] = (double)v.prim[q*N + c];
   if( mode == ROWS_CELLS ){
      for( int s=0 ; s<F ; ++s ) o[Q+s] = v.ct ? v.Phi[s*N + c] : 0.0;
      o[Q+F] = v.piph[c];
   }else{
      o[Q] = v.piph[c];
      o[Q+1] = v.dphi[c];
   }
}

/* Pack rows c0 .. c0+n-1 chunk by chunk; sink(rows, count) receives each
 * chunk in host memory. */
static int stream_rows(disco_batch *b, size_t c0, size_t n, int F, int mode,
                       const std::function<int(const double *, size_t)> &sink){
   const int ncol = mode == ROWS_CELLS ? b->Q + F + 1 : b->Q + 2;
   const size_t chunk = n < ((size_t)1 << 20) ? (n ? n : 1) : ((size_t)1 << 20);
   double *dbuf = NULL, *hbuf = NULL;
   CK(cudaSetDevice(b->device));
   CK(cudaMalloc(&dbuf, chunk*ncol*sizeof(double)));
   if( cudaMallocHost(&hbuf, chunk*ncol*sizeof(double)) != cudaSuccess ){
      cudaFree(dbuf);
      return DISCO_ERR_CUDA;
   }
   int s = DISCO_OK;
   for( size_t r0=0 ; r0<n && !s ; r0+=chunk ){
      size_t m = n - r0 < chunk ? n - r0 : chunk;
      if( b->prec == DISCO_PREC_MIXED )
         k_pack_rows<float><<<nblk(m, 256), 256, 0, b->stream>>>(b->vf, c0 + r0, m, b->Q, F, mode, dbuf);
      else
         k_pack_rows<double><<<nblk(m, 256), 256, 0, b->stream>>>(b->vd, c0 + r0, m, b->Q, F, mode, dbuf);
      if( cudaGetLastError() != cudaSuccess ||
          batch_xfer(b, hbuf, dbuf, m*ncol*sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess ){
         s = DISCO_ERR_CUDA;
         break;
      }
      s = sink(hbuf, m);
   }
   cudaFreeHost(hbuf);
   cudaFree(dbuf);
   return s;
}

/* the disk's first cell and cell count */
static void disk_cells(const disco_batch *b, int disk, size_t *c0, size_t *n){
   const DiskParams &D = b->dparams[disk];
   int na = b->disk_Nr[disk]*b->disk_Nz[disk];
   *c0 = (size_t)b->ann_off[D.ann0];
   size_t e = (size_t)b->ann_off[D.ann0 + na - 1] + b->ann_np[D.ann0 + na - 1];
   *n = e - *c0;
}

/* ------------------------------------------------------------ checkpoint */

struct ParEntry { const char *key; int isint; size_t off; };
#define PI_(k, f) { k, 1, offsetof(disco_params, f) }
#define PD_(k, f) { k, 0, offsetof(disco_params, f) }
/* writePars (h5out.c:167-330): the in.par keys this library reads */
static const ParEntry PARS[] = {
   PI_("Num_R", Num_R), PI_("Num_Z", Num_Z), PD_("aspect", aspect), PD_("T_Start", t_min),
   PD_("R_Min", rmin), PD_("R_Max", rmax), PD_("Z_Min", zmin), PD_("Z_Max", zmax),
   PD_("Phi_Max", phimax), PI_("Log_Zoning", LogZoning), PI_("R_Periodic", R_Periodic),
   PI_("Z_Periodic", Z_Periodic), PI_("NoBC_Rmin", NoBC_Rmin), PI_("NoBC_Rmax", NoBC_Rmax),
   PI_("NoBC_Zmin", NoBC_Zmin), PI_("NoBC_Zmax", NoBC_Zmax), PD_("Log_Radius", LogRadius),
   PI_("Timestep", Timestep), PD_("CFL", CFL), PD_("PLM", PLM), PD_("Max_DT", maxDT),
   PD_("Adiabatic_Index", Adiabatic_Index), PI_("Isothermal", isothermal_flag),
   PI_("Cs2_Profile", Cs2_Profile), PD_("Cs2_Par", Cs2_Par),
   PD_("Density_Floor", Density_Floor), PD_("Pressure_Floor", Pressure_Floor),
   PI_("Mesh_Motion", Mesh_Motion), PI_("Riemann_Solver", Riemann_Solver),
   PI_("Exact_Mesh_Omega", Exact_Mesh_Omega), PD_("Exact_Mesh_Omega_Par", Exact_Mesh_Omega_Par),
   PI_("Energy_Omega", Energy_Omega), PD_("Energy_Omega_Par", Energy_Omega_Par),
   PI_("RotFrame", RotFrame), PD_("RotOmega", RotOmega), PD_("RotD", RotD),
   PI_("Use_Viscosity", visc_flag), PD_("Viscosity", viscosity), PI_("Use_As_Alpha", alpha_flag),
   PD_("Mach_Number", Disk_Mach), PD_("Mass_Ratio", Mass_Ratio), PI_("Grav2D", grav2D),
   PI_("Constrained_Transport", CT),
   PD_("Metric_Par1", metricPar[1]), PD_("Metric_Par2", metricPar[2]),
   PD_("Metric_Par3", metricPar[3]), PD_("Metric_Par4", metricPar[4]),
   PI_("Init_Par0", initPar0), PD_("Init_Par1", initPar[1]), PD_("Init_Par2", initPar[2]),
   PD_("Init_Par3", initPar[3]), PD_("Init_Par4", initPar[4]), PD_("Init_Par5", initPar[5]),
   PD_("Init_Par6", initPar[6]), PD_("Init_Par7", initPar[7]), PD_("Init_Par8", initPar[8]),
};
#undef PI_
#undef PD_

static int put_string(disco_npz *z, const char *name, const char *v){
   char descr[16];
   size_t n = strlen(v) ? strlen(v) : 1;
   snprintf(descr, sizeof descr, "|S%zu", n);
   std::vector<char> buf(n, 0);
   memcpy(buf.data(), v, strlen(v));
   int64_t one = 1;
   return disco_npz_put(z, name, descr, 1, &one, buf.data());
}

/* writeOpts (h5out.c:91-160): the module selection */
static int put_opts(disco_npz *z, const disco_modules &m){
   static const char *const hydro[] = {"euler", "mhd"};
   static const char *const bc[] = {"fixed", "zerograd", "fixed3d", "polar", "outflow3d",
                                    "zerograd_omk", "accrete3d"};
   static const char *const pl[] = {"none", "sun", "cm2", "binary_soft", "circular", "cm"};
   static const char *const ic[] = {"kepler_noise", "mhd_shear_noise", "host"};
   CKS(put_string(z, "Opts/HYDRO", hydro[m.hydro]));
   CKS(put_string(z, "Opts/GEOMETRY", "cylindrical"));
   CKS(put_string(z, "Opts/BOUNDARY", bc[m.boundary]));
   CKS(put_string(z, "Opts/PLANETS", pl[m.planets]));
   CKS(put_string(z, "Opts/INITIAL", ic[m.initial]));
   CKS(put_string(z, "Opts/ANALYSIS", m.analysis == DISCO_DIAG_DISK2D ? "diag_disk2d" :
                                      m.analysis == DISCO_DIAG_EULER ? "diag_euler" :
                                      m.analysis == DISCO_DIAG_MHDMRI ? "diag_mhdmri" : "none"));
   int64_t one = 1;
   int v[3] = {m.num_c, m.num_n, m.ct_mode};
   CKS(disco_npz_put(z, "Opts/NUM_C", "<i4", 1, &one, &v[0]));
   CKS(disco_npz_put(z, "Opts/NUM_N", "<i4", 1, &one, &v[1]));
   return disco_npz_put(z, "Opts/CT_MODE", "<i4", 1, &one, &v[2]);
}

static int write_checkpoint(disco_batch *b, int disk, disco_npz *z){
   const DiskParams &D = b->dparams[disk];
   const disco_params &p = b->params[disk];
   const int Nr = b->disk_Nr[disk], Nz = b->disk_Nz[disk], na = Nr*Nz, a0 = D.ann0;
   const int Q = b->Q, F = num_faces(b->mods.ct_mode), ncol = Q + F + 1;
   size_t c0, n;
   disk_cells(b, disk, &c0, &n);
   DiskState st;
   CK(batch_xfer(b, &st, b->vd.ds + disk, sizeof st, cudaMemcpyDeviceToHost));

   /* Grid: T, the edges with their ghosts, and per annulus (k outer, j
    * inner: the reference's [Nz][Nr]) Index, Np and Id_phi0, the cell whose
    * centre has the largest cos(phi), first of equals (h5out.c:495-520) */
   std::vector<double> piph(n), dphi(n);
   CK(batch_xfer(b, piph.data(), b->vd.piph + c0, n*sizeof(double), cudaMemcpyDeviceToHost));
   CK(batch_xfer(b, dphi.data(), b->vd.dphi + c0, n*sizeof(double), cudaMemcpyDeviceToHost));
   std::vector<int> Index(na), Np(na), Id(na);
   for( int jk=0 ; jk<na ; ++jk ){
      int off = b->ann_off[a0 + jk] - (int)c0, np = b->ann_np[a0 + jk];
      Index[jk] = off;
      Np[jk] = np;
      double phi0 = M_PI;
      int id = 0;
      for( int i=0 ; i<np ; ++i ){
         double phi = piph[off + i] - .5*dphi[off + i];
         if( cos(phi0) < cos(phi) ){ phi0 = phi; id = off + i; }
      }
      Id[jk] = id;
   }
   int64_t one = 1, sh2[2] = {Nz, Nr}, shr = Nr + 1, shz = Nz + 1;
   CKS(disco_npz_put(z, "Grid/T", "<f8", 1, &one, &st.t));
   CKS(disco_npz_put(z, "Grid/r_jph", "<f8", 1, &shr, b->rj.data() + D.rj0));
   CKS(disco_npz_put(z, "Grid/z_kph", "<f8", 1, &shz, b->zk.data() + D.zk0));
   CKS(disco_npz_put(z, "Grid/Index", "<i4", 2, sh2, Index.data()));
   CKS(disco_npz_put(z, "Grid/Np", "<i4", 2, sh2, Np.data()));
   CKS(disco_npz_put(z, "Grid/Id_phi0", "<i4", 2, sh2, Id.data()));

   /* Data/Cells, streamed from the device */
   int64_t shc[2] = {(int64_t)n, ncol};
   CKS(disco_npz_begin(z, "Data/Cells", "<f8", 2, shc));
   CKS(stream_rows(b, c0, n, F, ROWS_CELLS, [&](const double *rows, size_t m){
      return disco_npz_append(z, rows, m*ncol*sizeof(double));
   }));
   CKS(disco_npz_end(z));

   /* Data/Planets (h5out.c:444-456) */
   std::vector<double> pl((size_t)D.npl*DISCO_PLANET_COLS);
   int npl = 0;
   CKS(disco_batch_get_planets(b, disk, pl.data(), D.npl, &npl));
   int64_t shp[2] = {npl, DISCO_PLANET_COLS};
   CKS(disco_npz_put(z, "Data/Planets", "<f8", 2, shp, pl.data()));

   /* Data/Diagnostics: avg_diagnostics divides the window's sums by its
    * length (analysis.c:29-49), output() then zeroes them (h5out.c:586) */
   int nq = b->nq;
   std::vector<double> Qrz((size_t)na*nq);
   if( nq ){
      CK(batch_xfer(b, Qrz.data(), b->d_Qrz + (size_t)a0*nq, sizeof(double)*na*nq, cudaMemcpyDeviceToHost));
      double dt = st.t_avg;
      for( size_t i=0 ; i<Qrz.size() ; ++i ) Qrz[i] /= dt;
   }
   int64_t shd[3] = {Nz, Nr, nq};
   CKS(disco_npz_put(z, "Data/Diagnostics", "<f8", 3, shd, Qrz.data()));

   for( const ParEntry &e : PARS ){
      std::string nm = std::string("Pars/") + e.key;
      const char *src = (const char *)&p + e.off;
      CKS(disco_npz_put(z, nm.c_str(), e.isint ? "<i4" : "<f8", 1, &one, src));
   }
   CKS(put_opts(z, b->mods));

   /* zero_diagnostics */
   if( nq ) CK(cudaMemsetAsync(b->d_Qrz + (size_t)a0*nq, 0, sizeof(double)*na*nq, b->stream));
   CK(batch_xfer(b, &st, b->vd.ds + disk, sizeof st, cudaMemcpyDeviceToHost));
   st.t_avg = 0.0;
   CK(batch_xfer(b, b->vd.ds + disk, &st, sizeof st, cudaMemcpyHostToDevice));
   return DISCO_OK;
}

extern "C" int disco_batch_write_checkpoint(disco_batch *b, int disk, const char *filestart){
   if( !b || !filestart || disk < 0 || disk >= b->ndisk ) return DISCO_ERR_ARG;
   if( !b->have_cells ) return DISCO_ERR_STATE;
   std::string path = std::string(filestart) + ".npz";
   disco_npz *z = NULL;
   CKS(disco_npz_create(path.c_str(), &z));
   int s = write_checkpoint(b, disk, z);
   int s2 = disco_npz_close(z);
   return s ? s : s2;
}

/* ------------------------------------------------------------ ascii */

extern "C" int disco_batch_write_ascii(disco_batch *b, int disk, const char *filestart){
   if( !b || !filestart || disk < 0 || disk >= b->ndisk ) return DISCO_ERR_ARG;
   if( !b->have_cells ) return DISCO_ERR_STATE;
   const DiskParams &D = b->dparams[disk];
   const disco_params &p = b->params[disk];
   const int Nr = b->disk_Nr[disk], Nz = b->disk_Nz[disk], Q = b->Q, ncol = Q + 2;
   size_t c0, n;
   disk_cells(b, disk, &c0, &n);
   std::vector<double> rows(n*ncol);
   size_t at = 0;
   CKS(stream_rows(b, c0, n, 0, ROWS_ASCII, [&](const double *r, size_t m){
      memcpy(rows.data() + at*ncol, r, m*ncol*sizeof(double));
      at += m;
      return DISCO_OK;
   }));
   const double *r_jph = b->rj.data() + D.rj0 + 1;
   const double *z_kph = b->zk.data() + D.zk0 + 1;
   int k_min = p.Z_Periodic ? NUM_G_GHOSTS : 0;
   int k_max = p.Z_Periodic ? Nz - NUM_G_GHOSTS : Nz;
   std::string path = std::string(filestart) + ".dat";
   FILE *f = fopen(path.c_str(), "w");
   if( !f ) return DISCO_ERR_IO;
   std::vector<char> fbuf(1 << 22);
   setvbuf(f, fbuf.data(), _IOFBF, fbuf.size());
   for( int j=0 ; j<Nr ; ++j ){
      double r = .5*(r_jph[j] + r_jph[j-1]);
      double dr = r_jph[j] - r_jph[j-1];
      for( int k=k_min ; k<k_max ; ++k ){
         double z = .5*(z_kph[k] + z_kph[k-1]);
         double dz = z_kph[k] - z_kph[k-1];
         int a = D.ann0 + j + Nr*k;
         size_t o = (size_t)b->ann_off[a] - c0;
         for( int i=0 ; i<b->ann_np[a] ; ++i ){
            const double *row = rows.data() + (o + i)*ncol;
            double piph = row[Q], dphi = row[Q+1];
            double phi = piph - .5*dphi;
            fprintf(f, "%e %e %e ", r, phi, z);
            fprintf(f, "%e %e %e ", dr, dphi, dz);
            for( int q=0 ; q<Q ; ++q ) fprintf(f, "%e ", row[q]);
            fprintf(f, "\n");
         }
      }
   }
   int bad = ferror(f);
   if( fclose(f) != 0 || bad ) return DISCO_ERR_IO;
   return DISCO_OK;
}

/* ------------------------------------------------------------ restart */

static int read_exact(disco_npz *z, const char *name, const char *descr, int ndim,
                      const int64_t *shape, void *dst){
   char d[16];
   int nd;
   int64_t sh[8];
   CKS(disco_npz_info(z, name, d, &nd, sh));
   if( strcmp(d, descr) || nd != ndim ) return DISCO_ERR_IO;
   size_t count = 1;
   for( int i=0 ; i<ndim ; ++i ){
      if( sh[i] != shape[i] ) return DISCO_ERR_ARG;
      count *= (size_t)sh[i];
   }
   return disco_npz_read(z, name, 0, dst, count*(strcmp(descr, "<i4") ? 8 : 4));
}

/* restart() for one disk (h5in.c:100-354, serial): checks the grid, reads
 * T and the planets, and places the disk's cells into the batch arrays */
static int read_disk(disco_batch *b, int disk, disco_npz *z, double *prim, double *Phi,
                     double *piph, double *T, std::vector<double> &pl){
   const DiskParams &D = b->dparams[disk];
   const int Nr = b->disk_Nr[disk], Nz = b->disk_Nz[disk], na = Nr*Nz, a0 = D.ann0;
   const int Q = b->Q, F = num_faces(b->mods.ct_mode), ncol = Q + F + 1;
   int64_t one = 1, sh2[2] = {Nz, Nr}, shr = Nr + 1, shz = Nz + 1;
   CKS(read_exact(z, "Grid/T", "<f8", 1, &one, T));
   std::vector<double> rj(Nr + 1), zk(Nz + 1);
   CKS(read_exact(z, "Grid/r_jph", "<f8", 1, &shr, rj.data()));
   CKS(read_exact(z, "Grid/z_kph", "<f8", 1, &shz, zk.data()));
   if( memcmp(rj.data(), b->rj.data() + D.rj0, rj.size()*sizeof(double)) ||
       memcmp(zk.data(), b->zk.data() + D.zk0, zk.size()*sizeof(double)) ) return DISCO_ERR_ARG;
   std::vector<int> Index(na), Np(na);
   CKS(read_exact(z, "Grid/Np", "<i4", 2, sh2, Np.data()));
   CKS(read_exact(z, "Grid/Index", "<i4", 2, sh2, Index.data()));
   for( int jk=0 ; jk<na ; ++jk ) if( Np[jk] != b->ann_np[a0 + jk] ) return DISCO_ERR_ARG;
   char d[16];
   int nd;
   int64_t sh[8];
   CKS(disco_npz_info(z, "Data/Cells", d, &nd, sh));
   if( strcmp(d, "<f8") || nd != 2 ) return DISCO_ERR_IO;
   if( sh[1] != ncol ) return DISCO_ERR_ARG;              /* h5in.c:324 */
   const int64_t Nc = sh[0];
   std::vector<double> track;
   for( int jk=0 ; jk<na ; ++jk ){                        /* h5in.c:270-289 */
      int np = Np[jk];
      if( Index[jk] < 0 || (int64_t)Index[jk] + np > Nc ) return DISCO_ERR_IO;
      track.resize((size_t)np*ncol);
      CKS(disco_npz_read(z, "Data/Cells", (uint64_t)Index[jk]*ncol*sizeof(double), track.data(),
                         track.size()*sizeof(double)));
      size_t c = (size_t)b->ann_off[a0 + jk];
      for( int i=0 ; i<np ; ++i, ++c ){                   /* Doub2Cell, h5in.c:72-77 */
         const double *row = track.data() + (size_t)i*ncol;
         memcpy(prim + c*Q, row, Q*sizeof(double));
         if( Phi ) memcpy(Phi + c*F, row + Q, F*sizeof(double));
         piph[c] = row[Q + F];
      }
   }
   /* Planets: the module's count of rows; a type column is optional
    * (h5in.c:291-318) */
   CKS(disco_npz_info(z, "Data/Planets", d, &nd, sh));
   if( strcmp(d, "<f8") || nd != 2 || sh[1] < 6 ) return DISCO_ERR_IO;
   if( sh[0] != D.npl ) return DISCO_ERR_ARG;
   std::vector<double> raw((size_t)sh[0]*sh[1]);
   CKS(disco_npz_read(z, "Data/Planets", 0, raw.data(), raw.size()*sizeof(double)));
   pl.assign((size_t)D.npl*DISCO_PLANET_COLS, 0.0);
   for( int q=0 ; q<D.npl ; ++q ){
      for( int col=0 ; col<DISCO_PLANET_COLS && col<sh[1] ; ++col )
         pl[(size_t)q*DISCO_PLANET_COLS + col] = raw[(size_t)q*sh[1] + col];
      if( pl[(size_t)q*DISCO_PLANET_COLS + 6] != 0.0 ) return DISCO_ERR_UNSUPPORTED;  /* PLPOINTMASS */
   }
   return DISCO_OK;
}

extern "C" int disco_batch_restart(disco_batch *b, const char *const *paths){
   if( !b || !paths ) return DISCO_ERR_ARG;
   for( int d=0 ; d<b->ndisk ; ++d ) if( !paths[d] ) return DISCO_ERR_ARG;
   const size_t N = (size_t)b->ncell;
   const int F = num_faces(b->mods.ct_mode);
   std::vector<double> prim(N*b->Q), piph(N), Phi(F ? N*F : 0);
   std::vector<double> T(b->ndisk);
   std::vector<std::vector<double>> pl(b->ndisk);
   for( int d=0 ; d<b->ndisk ; ++d ){
      disco_npz *z = NULL;
      CKS(disco_npz_open(paths[d], &z));
      int s = read_disk(b, d, z, prim.data(), F ? Phi.data() : NULL, piph.data(), &T[d], pl[d]);
      disco_npz_close(z);
      if( s ) return s;
   }
   /* setupCells adds noise on restart as well (domain.c:202-203): the same
    * draws as at the start, from glibc's rand() stream */
   bool any_noise = false;
   for( int d=0 ; d<b->ndisk ; ++d ) any_noise = any_noise || b->dparams[d].noise_type;
   if( any_noise ){
      std::vector<double> nz((size_t)4*N, 0.0);
      for( int d=0 ; d<b->ndisk ; ++d ){
         if( !b->dparams[d].noise_type ) continue;
         const DiskParams &D = b->dparams[d];
         int Ng[4] = {D.NgRa, D.NgRb, D.NgZa, D.NgZb};
         size_t c0, n;
         disk_cells(b, d, &c0, &n);
         CKS(disco_setup_noise(&b->params[d], D.Nr, D.Nz, Ng, b->ann_np.data() + D.ann0,
                               nz.data() + 4*c0));
      }
      CKS(disco_batch_set_noise(b, nz.data()));
   }
   for( int d=0 ; d<b->ndisk ; ++d ){
      CKS(disco_batch_set_time(b, d, T[d]));
      CKS(disco_batch_set_planets(b, d, pl[d].data(), b->dparams[d].npl));
   }
   /* the batch keeps nfs == NUM_FACES slots under constrained transport */
   return disco_batch_restart_cells(b, prim.data(), F ? Phi.data() : NULL, piph.data());
}
