/*
 * disco_b200 host side (C): the parts of Disco's start-up that stay on the
 * host -- in.par and Makefile_opt.in parsing, grid construction and the
 * per-annulus phi offsets -- restated so a batch can be built without the
 * reference tree.  Each function names the reference routine it replaces.
 */
#ifndef DISCO_HOST_H
#define DISCO_HOST_H

#include "disco_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/*
 * Parse an in.par file (readpar.c:6-42 readvar, :44-188 read_par_file).
 * Same key names, same "first matching line wins" rule, same separators
 * ("\t :=>_"), same 2*pi / pi scalings of T_*, Phi_Max and Z_* (:162-172).
 * Missing keys keep their zero value, as in the reference (main.c:31 zero-
 * initialises the domain); *nmissing receives how many were absent.
 */
int disco_read_par(const char *path, disco_params *p, int *nmissing);

/*
 * Parse a Makefile_opt.in module selection (INITIAL, HYDRO, BOUNDARY,
 * PLANETS, ANALYSIS, NUM_C, NUM_N, CT_MODE; Makefile:11-26).  Unknown module
 * names give DISCO_ERR_UNSUPPORTED, except INITIAL: a module other than
 * kepler_noise / mhd_shear_noise reads as DISCO_IC_HOST (its state must be
 * uploaded, disco_batch_setup_cells refuses it).
 */
int disco_read_opt(const char *path, disco_modules *m);

/*
 * setupGrid (gridsetup.c:15-142) for the serial single-rank case: fills
 * Nr, Nz (annuli incl. ghosts), Ng[4] = {NgRa, NgRb, NgZa, NgZb}, and, when
 * the pointers are non-NULL, Np[Nr*Nz], r_jph[Nr+1], z_kph[Nz+1] (element 0
 * is index -1 of the reference's arrays).  Call once with NULL arrays to
 * get the sizes.
 */
int disco_setup_grid(const disco_params *p, int *Nr, int *Nz, int *Ng,
                     int *Np, double *r_jph, double *z_kph);

/*
 * The per-annulus phi offsets of setupDomain (domain.c:172-233): glibc
 * srand(314159), one discarded rand(), then p0 = Pmax*rand()/RAND_MAX per
 * annulus, piph_i = p0 + i*Pmax/Np (wrapped once), and dphi from calc_dp
 * (misc.c:271-288) as setupCells does first (domain.c:290).  Also sets
 * real[] (1 for cells outside the ghost annuli, domain.c:307-351).
 */
int disco_setup_phi(const disco_params *p, int Nr, int Nz, const int *Ng,
                    const int *Np, double *piph, double *dphi, int *real);

/*
 * The random numbers addNoise (noise.c:15-50) draws for Noise_Type 1, 2 or
 * 3: glibc's rand() stream of disco_setup_phi continued, in setupCells'
 * cell order (domain.c:183-205, real cells only), each 2*rand()/RAND_MAX-1.
 * noise[4*c + m] for cell c (annulus order), m < 4 (2 for type 2); zero
 * elsewhere.  Upload with disco_batch_set_noise before set-up or restart.
 */
int disco_setup_noise(const disco_params *p, int Nr, int Nz, const int *Ng,
                      const int *Np, double *noise);

/* sizeof(disco_params) for which = 0, sizeof(disco_modules) for 1: lets a
 * foreign-language mirror of the structs check its layout. */
int disco_sizeof(int which);

/*
 * The checkpoint container (disco_npz.c): a NumPy .npz archive -- an
 * uncompressed ZIP64 archive of .npy arrays -- standing in for the HDF5 file
 * of Output/h5out.c and Restart/h5in.c, which this build has no library for.
 * A member is named by the reference's dataset path ("Grid/T",
 * "Data/Cells", ...); numpy.load(path)[name] reads it.  descr is a NumPy
 * type string: "<f8", "<i4", "|S<n>".  All calls return a disco_status;
 * DISCO_ERR_IO for a file that cannot be opened, written or parsed.
 *
 * Writing: disco_npz_create, then per member disco_npz_put (whole array) or
 * disco_npz_begin / disco_npz_append (any number of pieces, exactly the
 * array's bytes in total) / disco_npz_end, then disco_npz_close.  Reading:
 * disco_npz_open, disco_npz_info (descr, ndim <= 8, shape), disco_npz_read
 * (a byte range of the array data, C order), disco_npz_close.  Compressed
 * members (numpy.savez_compressed) are refused with DISCO_ERR_UNSUPPORTED.
 */
typedef struct disco_npz disco_npz;
int disco_npz_create(const char *path, disco_npz **z);
int disco_npz_begin(disco_npz *z, const char *name, const char *descr, int ndim,
                    const int64_t *shape);
int disco_npz_append(disco_npz *z, const void *data, size_t nbytes);
int disco_npz_end(disco_npz *z);
int disco_npz_put(disco_npz *z, const char *name, const char *descr, int ndim,
                  const int64_t *shape, const void *data);
int disco_npz_open(const char *path, disco_npz **z);
int disco_npz_info(disco_npz *z, const char *name, char *descr, int *ndim, int64_t *shape);
int disco_npz_read(disco_npz *z, const char *name, uint64_t offset, void *dst, size_t nbytes);
int disco_npz_close(disco_npz *z);

#ifdef __cplusplus
}
#endif
#endif
