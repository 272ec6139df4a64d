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
 * (no Fortran compiler), so parity to xspecfem2D is pinned through its golden
 * outputs only.
 *
 * All arrays use the solver layout: per-element GLL arrays [ispec][j][i]
 * (25 values per element), global vectors [iglob][component], attenuation
 * arrays [ispec][j][i][i_sls] with N_SLS = 3, 0-based ids.
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
  int seismotype;                                         /* 1 displ, 2 veloc, 3 accel, 4 pressure, 6 potential */
  double deltat, deltatover2, deltatsquareover2;
  /* anisotropy (may be NULL): per-element flag and c11,c13,c15,c33,c35,c55 */
  const int *ispec_is_anisotropic;
  const double *c11, *c13, *c15, *c33, *c35, *c55;
  /* time scheme: 1 Newmark, 2 LDDRK (6 stages, coefficients in CUSTOM_REAL) */
  int time_scheme;
  const double *alpha_lddrk, *beta_lddrk;                 /* 6 each */
  /* viscoelastic 3-SLS (may be NULL): Newmark recursive-convolution
   * coefficients A/B (prepare_attenuation.f90:378-396) and the LDDRK
   * inverse relaxation times and weights (attenuation_model.f90:114-125).
   * All zero at a point means no attenuation there. */
  const double *att_a1, *att_b1, *att_a2, *att_b2;        /* nspec*25*3 */
  const double *att_itau1, *att_phi1, *att_itau2, *att_phi2;
  /* adjoint simulation (SIMULATION_TYPE = 3): when adj_src is not NULL the
   * force sources are replaced by the adjoint sources at the receivers,
   * adj_src[irec][it][comp] in time order, injected time-reversed
   * (compute_add_sources_viscoelastic.f90:351-405; in a fluid element comp 0
   * into chi_dot_dot, compute_add_sources_acoustic.f90:247-290).  With fluid
   * elements (Newmark only) the solid step runs first, the solid takes the
   * fluid potential and the fluid minus the solid acceleration as coupling
   * terms (iterate_time.F90:298-327, compute_coupling_*.f90 SIMULATION_TYPE 3) */
  const double *adj_src;
  /* acoustic (fluid) domain, potential formulation u = grad(chi)/rho (may be
   * NULL = no acoustic element): compute_forces_viscoacoustic.f90:34-417,
   * compute_stacey_acoustic.f90:34-199, enforce_acoustic_free_surface.f90:35-96,
   * compute_coupling_acoustic_el.f90:36-283 (acoustic side) and
   * compute_coupling_viscoelastic_ac.f90:36-258 (elastic side) */
  const int *ispec_is_acoustic;                           /* nspec (kappastore above is used) */
  const double *rmass_inverse_acoustic;                   /* nglob */
  int nstacey_ac;                                         /* acoustic absorbing points, reference order */
  const int *st_ac_iglob;
  const double *st_ac_w, *st_ac_rvp;                      /* jacobian1D*w, rho*vp */
  int nfree_ac;                                           /* free-surface points (zeroed) */
  const int *free_ac_iglob;
  int ncpl_ac;                                            /* coupling points, acoustic side */
  const int *cpl_ac_iglob;
  const double *cpl_ac_nx, *cpl_ac_nz, *cpl_ac_w;
  int ncpl_el;                                            /* coupling points, elastic side */
  const int *cpl_el_iglob;
  const double *cpl_el_nx, *cpl_el_nz, *cpl_el_w;
  int use_trick;                                          /* USE_TRICK_FOR_BETTER_PRESSURE: p = -chi */
  /* CPML layers (pml_region NULL = none): pml_compute_memory_variables.f90,
   * pml_compute_accel_contribution.f90, pml_compute.f90 (l/lik parameters,
   * convolution coefficients, outer-edge zeroing) */
  const int *pml_region;                                  /* nspec: 0 none, 1 X only, 2 Z only, 3 XZ */
  const double *pml_K_x, *pml_K_z, *pml_d_x, *pml_d_z, *pml_alpha_x, *pml_alpha_z;  /* nspec*25 */
  int npml_bnd_el, npml_bnd_ac;                           /* outer PML edge points zeroed every step */
  const int *pml_bnd_el, *pml_bnd_ac;
  const int *cpl_ac_elpt, *cpl_el_acpt;                   /* other-domain element point per coupling entry */
  double DT;                                              /* time step in double (PML coefficients) */
  /* CPML in attenuating solids, Newmark only (pml_compute_memory_variables.f90:546-894):
   * pml_visco[e] = 1 for a layer element whose largest Qkappa and Qmu are both below
   * 9998.999 (compute_forces_viscoelastic.F90:249-267), NULL = none; for them the Zener
   * strain relaxation times tau_epsilon_nu1/2 (nspec*25*3) and Mu_nu1/2 (nspec*25) of
   * attenuation_model.f90:147-160, with att_itau and att_phi above */
  const int *pml_visco;
  const double *att_teps1, *att_teps2;
  const double *att_mu1, *att_mu2;
} sf2d_oracle_db;

/* Fields addressed by sf2d_oracle_get/set. */
enum {
  SF2D_OR_DISPL = 0, SF2D_OR_VELOC = 1, SF2D_OR_ACCEL = 2,
  SF2D_OR_DISPL_LDDRK = 3, SF2D_OR_VELOC_LDDRK = 4,
  SF2D_OR_E1 = 5, SF2D_OR_E11 = 6, SF2D_OR_E13 = 7,
  SF2D_OR_ATT_OLD = 8,                                   /* nspec*25*3: dux_dxl, duz_dzl, dux_dzl+duz_dxl of the last step */
  SF2D_OR_RHO_KL = 9, SF2D_OR_KAPPA_KL = 10, SF2D_OR_MU_KL = 11,  /* nspec*25, unscaled sums */
  SF2D_OR_POT = 12, SF2D_OR_POT_DOT = 13, SF2D_OR_POT_DOT_DOT = 14, /* nglob: chi, chi_dot, chi_dot_dot */
  SF2D_OR_POT_LDDRK = 15, SF2D_OR_POT_DOT_LDDRK = 16,
  SF2D_OR_HESS1 = 17, SF2D_OR_HESS2 = 18,                         /* nspec*25: approximate Hessian sums */
  SF2D_OR_RHO_AC_KL = 19, SF2D_OR_KAPPA_AC_KL = 20                /* nspec*25: fluid kernels, deltat included */
};

/* Creates an oracle state (fields zero).  precision: 4 -> float, 8 -> double.
 * Returns NULL on bad arguments. */
void *sf2d_oracle_create(const sf2d_oracle_db *db, int precision);

/* Advances nstep time steps.  seis (may be NULL): nrec*nstep*2 doubles,
 * [irec][it][comp]; seismotype 4 (pressure) fills comp 0 and zeroes comp 1.  nthreads <= 0 uses all host threads (or
 * SF2D_ORACLE_THREADS).  Returns 0 on success. */
int sf2d_oracle_run(void *h, int nstep, double *seis, int nthreads);

/* Copy a field out of / into the state, in the state's precision.  Sizes:
 * DISPL..VELOC_LDDRK nglob*2, E1..E13 nspec*25*3. */
int sf2d_oracle_get(void *h, int which, void *out);
int sf2d_oracle_set(void *h, int which, const void *in);

/* Adds, at every element GLL point, the sensitivity-kernel integrands of the
 * state's (adjoint) displacement and acceleration against the forward
 * displacement b_displ (nglob*2, state precision): compute_kernels.f90:75-292. */
int sf2d_oracle_accumulate_kernels(void *h, const void *b_displ);

/* Adds the fluid-element kernel integrands of the state's (adjoint) potential
 * against the forward potential b_pot (nglob, state precision):
 * compute_kernels.f90:293-449.  Solid elements are left to
 * sf2d_oracle_accumulate_kernels. */
int sf2d_oracle_accumulate_kernels_acoustic(void *h, const void *b_pot);

/* Adds the approximate-Hessian integrands (compute_kernels.f90:749-800,
 * elastic): at every point |b_accel|^2 and accel . b_accel of the state's
 * (adjoint) acceleration against the forward acceleration b_accel, times
 * deltat, into HESS1 and HESS2 of the element points. */
int sf2d_oracle_accumulate_hessian(void *h, const void *b_accel);

/* Gaussian smoothing of per-element-point fields, the CPU loop of
 * smooth_sem.F90:63-467 (every pair of points, no cutoff, CUSTOM_REAL = float).
 * x, z, jacobian: nspec*25; wgll_sq: 25; fields, out: nfields*nspec*25. */
int sf2d_oracle_smooth(int nspec, int nglob, const int *ibool, const float *x, const float *z,
                       const float *jacobian, const float *wgll_sq, int nfields, const float *fields,
                       float sigma_h, float sigma_v, float *out);

/* Sets the number of steps done (the source time functions are indexed by it). */
int sf2d_oracle_set_step(void *h, int it);

void sf2d_oracle_destroy(void *h);

/* Number of host threads the oracle uses by default. */
int sf2d_oracle_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
