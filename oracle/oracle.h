/*
 * ORACLE TEST INFRASTRUCTURE -- not part of the product.
 *
 * CPU restatement (plain C, FP64, single thread) of the reference Disco
 * serial timestep hot path, used only by tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg as the checker.  Each function cites the
 * reference file:line it restates.  It is pinned bit-for-bit against the
 * reference itself, compiled from its own sources into oracle/_ref/ by
 * oracle/Makefile (tests/test_oracle_pin.py).
 *
 * The oracle does the step only (timestep/onestep/getmindt); the state it
 * starts from is uploaded as plain arrays, so the same starting state can
 * be handed to the reference dump, this oracle and the GPU.
 */
#ifndef DISCO_ORACLE_H
#define DISCO_ORACLE_H
#include "disco_b200.h"

typedef struct orc_domain orc_domain;

orc_domain *orc_create(const disco_params *p, const disco_modules *m,
                       int Nr, int Nz, const int *Ng, const int *Np,
                       const double *r_jph, const double *z_kph);
void   orc_destroy(orc_domain *d);
int    orc_ncell(const orc_domain *d);
void   orc_set_cells(orc_domain *d, const double *prim, const double *cons,
                     const double *piph, const double *dphi, const double *wiph,
                     const int *real);
void   orc_get_cells(const orc_domain *d, double *prim, double *cons,
                     double *piph, double *dphi, double *wiph);
double orc_mindt(orc_domain *d);
void   orc_timestep(orc_domain *d, double dt);
double orc_time(const orc_domain *d);
int    orc_get_faces(orc_domain *d, int dim, int *fIndex, int *iL, int *iR,
                     int *LRtype, double *geom);
void   orc_get_diagnostics(const orc_domain *d, double *Qrz, double *t_avg);

/* Lock-step hooks: run one stage of onestep() on the current state, so a
 * test can compare one GPU kernel at a time.  stage names:
 *   "wcell", "adjust_rk", "plm_phi", "faces_r", "plm_r", "flux_phi",
 *   "flux_r", "source", "move", "clean_dp", "c2p", "boundary" */
int    orc_stage(orc_domain *d, const char *stage, double RK, double dt);
/* gradp / gradr / gradz (which = 0,1,2), cell-major Q doubles per cell */
void   orc_get_grad(const orc_domain *d, int which, double *out);

#endif
