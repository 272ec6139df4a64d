/*
 * CPU oracle for the SPECFEM2D time-marching hot path -- TEST INFRASTRUCTURE.
 *
 * This library is the checker for the CUDA path and the timed CPU baseline.
 * It is a restatement of the reference's CPU Fortran routines (cited per
 * function in sf2d_oracle.cpp).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it; the product never calls it.
 *
 * Parity pin: seismograms of the reference's EXAMPLES/Tromp2005_kernel run
 * (REF_SEIS/AA.S0001.BX?.semd) are reproduced by setup + this oracle (see
 * tests/test_oracle_golden.py).  The reference binary itself cannot be built
 * (no Fortran compiler), so 1e-5-level parity to xspecfem2D is unpinned.
 *
 * All arrays use the solver layout: per-element GLL arrays [ispec][j][i]
 * (25 values per element), global vectors [iglob][component], 0-based ids.
 */
#ifndef SF2D_ORACLE_H
#define SF2D_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nspec, nglob;
  const int *ibool;                                       /* nspec*25 */
  const double *xix, *xiz, *gammax, *gammaz, *jacobian;   /* nspec*25 */
  const double *rhostore, *kappastore, *mustore, *rho_vpstore, *rho_vsstore;
  const double *rmass_inverse;                            /* nglob*2 */
  const double *hprime, *hprimewgll;                      /* 5x5 [i2][i1] */
  const double *wxgll, *wzgll;                            /* 5 */
  /* Stacey, one entry per absorbing GLL point, reference order */
  int nstacey;
  const int *st_iglob;
  const double *st_nx, *st_nz, *st_w, *st_rvp, *st_rvs;
  /* sources */
  int nsrc;
  const int *src_ispec;
  const double *sourcearrays;                             /* nsrc*25*2 */
  const double *stf;                                      /* nsrc*nstep_total*nstage */
  int nstep_total, nstage;
  /* receivers */
  int nrec;
  const int *rec_ispec;
  const double *hxir, *hgammar;                           /* nrec*5 */
  double cosrot, sinrot;
  int seismotype;                                         /* 1 displ, 2 veloc, 3 accel */
  double deltat, deltatover2, deltatsquareover2;
  /* anisotropy (may be NULL): per-element flag and c11,c13,c15,c33,c35,c55 */
  const int *ispec_is_anisotropic;
  const double *c11, *c13, *c15, *c33, *c35, *c55;
} sf2d_oracle_db;

/* Runs `nstep` Newmark steps starting at step index `it0` (0-based) on the
 * fields in/out (displ, veloc, accel: nglob*2 each, caller-owned, same
 * precision as `precision`: 4 -> float, 8 -> double).  Seismograms are
 * written to seis (nrec*nstep*2 doubles, [irec][it][comp]).  nthreads <= 0
 * uses all host threads (or SF2D_ORACLE_THREADS).  Returns 0 on success, <0 on bad arguments. */
int sf2d_oracle_newmark_elastic(const sf2d_oracle_db *db, int precision, int it0, int nstep,
                                void *displ, void *veloc, void *accel, double *seis,
                                int nthreads);

/* Number of host threads the oracle uses by default. */
int sf2d_oracle_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
