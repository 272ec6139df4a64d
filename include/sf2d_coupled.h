/*
 * sf2d_b200 -- coupled fluid-solid runs (acoustic + elastic domains).
 * Plain C ABI, same conventions as sf2d_b200.h (int status, 0 = OK).
 *
 * A mesh with acoustic (fluid) elements runs as two sub-meshes with their own
 * compact point numberings: the solid one described by an sf2d_elastic_desc
 * (only its elements, points, absorbing points, sources and receivers) and
 * the fluid one by an sf2d_acoustic_desc.  Interface points exist in both;
 * sf2d_coupling_desc lists them in both numberings.  Correspondence:
 *   sf2d_coupled_create   <- prepare_fields_acoustic_device
 *                            (src/gpu/prepare_mesh_constants_cuda.cu:319) with
 *                            the fluid parts of prepare_constants_device and
 *                            prepare_stacey_device
 *   sf2d_coupled_run      <- per step, in order: update_displacement_ac_cuda
 *                            (src/gpu/update_displacement_cuda.cu:133),
 *                            acoustic_enforce_free_surf_cuda
 *                            (src/gpu/enforce_acoustic_free_surface_cuda.cu:46),
 *                            compute_forces_acoustic_cuda
 *                            (src/gpu/compute_forces_acoustic_cuda.cu:248),
 *                            compute_stacey_acoustic_cuda
 *                            (src/gpu/compute_stacey_acoustic_cuda.cu:40),
 *                            compute_coupling_ac_el_cuda (src/gpu/compute_coupling_cuda.cu:47),
 *                            compute_add_sources_ac_cuda
 *                            (src/gpu/compute_add_sources_viscoacoustic_cuda.cu:46),
 *                            kernel_3_acoustic_cuda (src/gpu/update_displacement_cuda.cu:322),
 *                            then the solid step of sf2d_run with
 *                            compute_coupling_el_ac_cuda (src/gpu/compute_coupling_cuda.cu:125)
 *                            and compute_seismograms_cuda for both domains
 *   sf2d_coupled_get_fields / set_fields <- transfer_fields_el_{from,to}_device
 *                            and transfer_fields_ac_{from,to}_device
 *                            (src/gpu/transfer_fields_cuda.cu:53,69,223,274)
 */
#ifndef SF2D_COUPLED_H
#define SF2D_COUPLED_H

#include "sf2d_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct sf2d_coupled sf2d_coupled;

typedef struct {
  int nspec, nglob;                          /* fluid elements and their points (own 0-based numbering) */
  const int *ibool;                          /* nspec*25 */
  const float *xix, *xiz, *gammax, *gammaz;  /* nspec*25 */
  const float *jacobian, *rhostore, *kappastore;  /* nspec*25; J/rho is formed in FP32 */
  const float *rmass_inverse;                /* nglob: rmass_inverse_acoustic (invert_mass_matrix.F90) */
  const double *centroid_xz;                 /* nspec*2 element centres for tiling, may be NULL */
  int nfree;                                 /* free-surface points, zeroed every step */
  const int *free_iglob;
  int nstacey;                               /* fluid absorbing points in reference order */
  const int *st_iglob;
  const float *st_w, *st_rho_vp;             /* jacobian1D * w, rho * vp */
  int nsrc;                                  /* pressure sources in fluid elements */
  const int *src_ispec;
  const float *sourcearrays;                 /* nsrc*25 hlagrange values [isrc][j][i] */
  const float *stf;                          /* nsrc*nstep*nstage */
  int nrec;                                  /* receivers in fluid elements */
  const int *rec_ispec;
  const double *hxir, *hgammar;              /* nrec*5 */
  const int *rec_global;                     /* index of each in the run's receiver list */
  int tile_elems;                            /* 0 = 32 */
  /* CPML layer in the fluid (pml_region NULL = none), as in sf2d_elastic_desc;
   * edge points: pml_boundary_acoustic (pml_compute.f90:502-541) */
  const int *pml_region;
  const double *pml_K_x, *pml_K_z, *pml_d_x, *pml_d_z, *pml_alpha_x, *pml_alpha_z;
  int npml_edge;
  const int *pml_edge_iglob;
  double pml_dt;
  int threads_per_block;                     /* fluid tile kernel: 128, 250, 256 or 512; 0 = the solid's */
} sf2d_acoustic_desc;

typedef struct {
  int nrec_total;                            /* receivers of the run (solid + fluid) */
  const int *el_rec_global;                  /* index of each solid receiver in that list */
  int seismotype;                            /* 1-3 displacement/velocity/acceleration, 4 pressure (fluid only),
                                                6 potential (fluid; zero in the solid) */
  int use_trick;                             /* USE_TRICK_FOR_BETTER_PRESSURE: pressure = -chi */
  double cosrot, sinrot;
  /* fluid side (compute_coupling_acoustic_el.f90): chi_dd[ac] += w * (u_pred[el] . n) */
  int ncpl_ac;
  const int *cpl_ac_point, *cpl_ac_el_point; /* fluid point, the same point in the solid numbering */
  const float *cpl_ac_nx, *cpl_ac_nz, *cpl_ac_w;
  /* solid side (compute_coupling_viscoelastic_ac.f90): a[el] += w * n * (-chi_dd[ac]) */
  int ncpl_el;
  const int *cpl_el_point, *cpl_el_ac_point;
  const float *cpl_el_nx, *cpl_el_nz, *cpl_el_w;
  /* with CPML layers: the element GLL point (ispec*25 + j*5 + i, sub-mesh numbering)
   * of the solid element behind each fluid-side entry and of the fluid element behind
   * each solid-side entry; an entry whose element lies in a layer adds the layer's
   * memory terms (compute_coupling_acoustic_el.f90:78-140,
   * compute_coupling_viscoelastic_ac.f90:105-150) */
  const int *cpl_ac_el_elpt, *cpl_el_ac_elpt;
  /* 1: an adjoint run (SIMULATION_TYPE = 3, Newmark, no CPML): the solid step
   * runs first and accumulates the solid kernels, the solid takes the fluid's
   * predicted chi as its pressure term and the fluid minus the solid's new
   * acceleration as its displacement term (iterate_time.F90:298-327,
   * compute_coupling_viscoelastic_ac.f90:89-93, compute_coupling_acoustic_el.f90:89-95);
   * fluid sources add (hlagrange) stf to chi_dot_dot without 1/kappa
   * (compute_add_sources_acoustic.f90:247-290).  Used by sf2d_coupled_fwi_*. */
  int adjoint;
} sf2d_coupling_desc;

/* A solid description with nspec = 0 makes a fluid-only run (no coupling entries,
 * solid sources or solid receivers): only its time-stepping members (nstep,
 * deltat, deltatover2, deltatsquareover2, time_scheme, nstage, alpha_lddrk,
 * beta_lddrk, threads_per_block) and GLL arrays (hprime, hprimewgll, wxgll,
 * wzgll) are read. */
int sf2d_coupled_create(const sf2d_elastic_desc *solid, const sf2d_acoustic_desc *fluid,
                        const sf2d_coupling_desc *coupling, sf2d_coupled **out);
/* Advances nstep steps (fluid then solid per step or LDDRK stage); seismograms
 * (may be NULL): nrec_total*nstep*2 doubles [irec][it][comp]. */
int sf2d_coupled_run(sf2d_coupled *c, int nstep, double *seismograms);
/* The same steps queued without a host wait (CUDA graphs of fixed step
 * chunks on the solver's stream); sf2d_coupled_synchronize waits for them and
 * returns the stability status; sf2d_coupled_get_stream gives the stream. */
int sf2d_coupled_enqueue(sf2d_coupled *c, int nstep);
/* Traces of steps it0 .. it0+n-1 (0-based) of the run's receivers:
 * out nrec_total*n*2 [irec][k][comp]; waits for the queued steps. */
int sf2d_coupled_copy_seismograms(sf2d_coupled *c, int it0, int n, double *out);
int sf2d_coupled_prepare(sf2d_coupled *c);  /* as sf2d_prepare */
int sf2d_coupled_synchronize(sf2d_coupled *c);
int sf2d_coupled_get_stream(sf2d_coupled *c, void **stream);
/* Fields in the sub-mesh numberings: displ/veloc/accel solid nglob*2,
 * chi/chi_dot/chi_dot_dot fluid nglob.  NULL skips (get) or zeroes (set). */
int sf2d_coupled_get_fields(sf2d_coupled *c, float *displ, float *veloc, float *accel, float *chi,
                            float *chi_dot, float *chi_dot_dot);
int sf2d_coupled_set_fields(sf2d_coupled *c, const float *displ, const float *veloc, const float *accel,
                            const float *chi, const float *chi_dot, const float *chi_dot_dot);
/* Whole-mesh numbering of the two sub-meshes: solid_points[k] (fluid_points[k])
 * is the mesh point of the solid's (fluid's) point k, nglob_total points in
 * all (solid_points may be NULL for a fluid-only mesh).  Set once; afterwards
 * the _global transfers take whole-mesh arrays (displ/veloc/accel nglob_total*2,
 * chi/chi_dot/chi_dot_dot nglob_total) and permute on the device, so the host
 * touches no point twice.  get: points outside a field's domain read zero. */
int sf2d_coupled_set_global_numbering(sf2d_coupled *c, int nglob_total, const int *solid_points,
                                      const int *fluid_points);
int sf2d_coupled_set_fields_global(sf2d_coupled *c, const float *displ, const float *veloc, const float *accel,
                                   const float *chi, const float *chi_dot, const float *chi_dot_dot);
int sf2d_coupled_get_fields_global(sf2d_coupled *c, float *displ, float *veloc, float *accel, float *chi,
                                   float *chi_dot, float *chi_dot_dot);
/* Average ms per launch of the fluid tile, fluid shared-point, solid tile and
 * solid shared-point kernels (ms[0..3]) and per step (ms[4]); advances nstep steps. */
int sf2d_coupled_time_kernels(sf2d_coupled *c, int nstep, float *ms);
/* info[6]: fluid tiles, fluid shared points, max local points, shared bytes per CTA,
 * fluid interior points, partial-sum slots. */
int sf2d_coupled_layout_info(sf2d_coupled *c, long long *info);
/* sf2d_layout_info of the solid sub-solver. */
int sf2d_coupled_solid_layout_info(sf2d_coupled *c, long long *info8);
/* Kernel launches that sf2d_coupled_enqueue(c, nstep) issues. */
int sf2d_coupled_launch_count(sf2d_coupled *c, int nstep, long long *launches);
int sf2d_coupled_destroy(sf2d_coupled *c);

/* Sensitivity kernels of a coupled fluid-solid mesh (the kernel run of
 * SIMULATION_TYPE = 3 with fluid and solid elements), as sf2d_fwi_* for a
 * solid mesh: a forward run with a state checkpoint (solid u, v, a and fluid
 * chi, chi_dot, chi_dot_dot) every checkpoint_every steps, then an adjoint
 * sweep that recomputes each forward segment from its checkpoint (solid
 * displacement and fluid chi frames) while the adjoint field, driven by the
 * time-reversed adjoint sources at the receivers, accumulates
 *   solid: rho_kl, kappa_kl, mu_kl as sf2d_fwi_backward (compute_kernels.f90:75-292,
 *          save_adjoint_kernels.f90:134-141), over the solid sub-mesh's elements;
 *   fluid: rho_ac_kl = sum 1/rho grad(chi_adj) . grad(chi) dt and
 *          kappa_ac_kl = sum 1/kappa chi_adj_dd chi dt (compute_kernels.f90:293-449),
 *          over the fluid sub-mesh's elements.
 * Adjoint step it is paired with forward step NSTEP - it + 1 (iterate_time_undoatt.F90).
 * Newmark only, no CPML.  Replaces the GPU kernel run of
 * compute_kernels_acoustic_cuda / compute_kernels_elastic_cuda
 * (src/gpu/compute_kernels_cuda.cu) driven by iterate_time.F90. */
typedef struct sf2d_coupled_fwi sf2d_coupled_fwi;
/* solid_rhostore, solid_kappastore: nspec*25 of the solid sub-mesh (may be
 * NULL for a fluid-only mesh) */
int sf2d_coupled_fwi_create(const sf2d_elastic_desc *solid, const sf2d_acoustic_desc *fluid,
                            const sf2d_coupling_desc *coupling, const float *solid_rhostore,
                            const float *solid_kappastore, int checkpoint_every, sf2d_coupled_fwi **out);
/* forward run from rest; seismograms (may be NULL): nrec_total*nstep*2 [irec][it][comp] */
int sf2d_coupled_fwi_forward(sf2d_coupled_fwi *f, double *seismograms);
/* adj_src: nrec_total*nstep*2 in time order ([irec][it][comp]; a fluid receiver
 * uses comp 0).  Kernels in each sub-mesh's element order; solid arrays may be
 * NULL for a fluid-only mesh. */
int sf2d_coupled_fwi_backward(sf2d_coupled_fwi *f, const float *adj_src, float *rho_kl, float *kappa_kl,
                              float *mu_kl, float *rho_ac_kl, float *kappa_ac_kl);
/* receiver traces of the adjoint field of the last backward (nrec_total*nstep*2) */
int sf2d_coupled_fwi_adjoint_seismograms(sf2d_coupled_fwi *f, double *seismograms);
/* The solid kernel sums of the last backward before the scaling of
 * save_adjoint_kernels.f90:134-141 (solid sub-mesh element order): what the
 * reference's transfer_kernels_el_to_host hands to the host. */
int sf2d_coupled_fwi_kernel_sums(sf2d_coupled_fwi *f, float *rho_kl, float *kappa_kl, float *mu_kl);
/* The coupled run of the adjoint field (owned by f, valid until
 * sf2d_coupled_fwi_destroy) for reading its fields and norms after a backward
 * sweep (sf2d_coupled_get_fields*, sf2d_coupled_set_global_numbering).  Its
 * time loop belongs to f: do not enqueue steps on it. */
int sf2d_coupled_fwi_adjoint_run(sf2d_coupled_fwi *f, sf2d_coupled **adj);
int sf2d_coupled_fwi_destroy(sf2d_coupled_fwi *f);

#ifdef __cplusplus
}
#endif
#endif
