/*
 * sf2d_b200 -- B200-native (sm_100a) time-marching hot path of SPECFEM2D.
 *
 * Plain C ABI: pointers and sizes only, every call returns an int status
 * (SF2D_OK = 0, negative on error; sf2d_last_error() gives the message).
 * Nothing here exits the process.  Arrays use the reference solver layout:
 * per-element GLL arrays are [ispec][j][i] (the memory order of the
 * Fortran arrays (i,j,ispec)), global vectors [iglob][component]; indices
 * are 0-based.
 *
 * Correspondence with the reference's Fortran->GPU interface
 * (src/gpu/specfem2D_gpu_cuda_method_stubs.c lists all of them):
 *   sf2d_elastic_create   <- prepare_constants_device
 *                            (src/gpu/prepare_mesh_constants_cuda.cu:83),
 *                            prepare_fields_elastic_device (:527),
 *                            prepare_stacey_device (:926), plus the source
 *                            and receiver arrays of prepare_constants_device
 *   sf2d_set_fields       <- transfer_fields_el_to_device
 *                            (src/gpu/transfer_fields_cuda.cu:53)
 *   sf2d_get_fields       <- transfer_fields_el_from_device (:69)
 *   sf2d_run              <- one call per time step of, in order,
 *                            update_displacement_cuda
 *                            (src/gpu/update_displacement_cuda.cu:52),
 *                            compute_forces_viscoelastic_cuda
 *                            (src/gpu/compute_forces_viscoelastic_cuda.cu:327),
 *                            compute_stacey_viscoelastic_cuda
 *                            (src/gpu/compute_stacey_viscoelastic_cuda.cu:40),
 *                            compute_add_sources_el_cuda
 *                            (src/gpu/compute_add_sources_viscoelastic_cuda.cu:46),
 *                            kernel_3_a_cuda (src/gpu/update_displacement_cuda.cu:221),
 *                            compute_seismograms_cuda
 *                            (src/gpu/write_seismograms_cuda.cu:41),
 *                            fused into one tile-staged kernel per step
 *   sf2d_get_norm         <- get_norm_elastic_from_device
 *                            (src/gpu/check_fields_cuda.cu:358)
 *   sf2d_initialize_device <- initialize_cuda_device (src/gpu/initialize_cuda.cu:50)
 *   sf2d_destroy          <- prepare_cleanup_device
 *                            (src/gpu/prepare_mesh_constants_cuda.cu:1139)
 */
#ifndef SF2D_B200_H
#define SF2D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SF2D_OK 0
#define SF2D_ERR_INVALID (-1)
#define SF2D_ERR_CUDA (-2)
#define SF2D_ERR_OOM (-3)
#define SF2D_ERR_UNSTABLE (-4)
#define SF2D_ERR_TIMEOUT (-5)

typedef struct sf2d_solver sf2d_solver;

/* Elastic (isotropic) Newmark problem in reference layout. */
typedef struct {
  int nspec, nglob;
  const int *ibool;                          /* nspec*25, 0-based */
  const float *xix, *xiz, *gammax, *gammaz;  /* nspec*25 */
  const float *lambdastore, *mustore;        /* nspec*25: lambda = rho*cp*cp - 2*mu with
                                                cp = rho_vpstore/rhostore, in FP32
                                                (compute_forces_viscoelastic.F90:286-294) */
  const float *rmass_inverse;                /* nglob*2 */
  const float *hprime, *hprimewgll;          /* 25: [i2*5+i1] = l'_{i1}(xi_{i2}) (times w_{i2}) */
  const float *wxgll, *wzgll;                /* 5 */
  const double *centroid_xz;                 /* nspec*2 element centres for tiling, may be NULL */
  /* Stacey absorbing points, one entry per (edge, GLL point) in the order the
   * reference visits them (compute_stacey_elastic.f90:116-980) */
  int nstacey;
  const int *st_iglob;
  const float *st_nx, *st_nz, *st_w, *st_rho_vp, *st_rho_vs;
  /* sources: element, sourcearrays[isrc][j][i][comp], stf[isrc][it] */
  int nsrc;
  const int *src_ispec;
  const float *sourcearrays;
  const float *stf;
  /* receivers: element, Lagrange weights hxir[irec][i], hgammar[irec][j] */
  int nrec;
  const int *rec_ispec;
  const double *hxir, *hgammar;
  double cosrot, sinrot;
  int seismotype;                            /* 1 displacement, 2 velocity, 3 acceleration */
  /* time stepping */
  int nstep;                                 /* length of stf and of the seismogram buffer */
  float deltat, deltatover2, deltatsquareover2;
  int tile_elems;                            /* elements per tile, 0 = default (64) */
  int threads_per_block;                     /* 128, 250, 256 or 512; 0 = default (256); 250 keeps
                                                each thread on one GLL position of every element */
  /* time scheme: 1 (or 0) Newmark, 2 LDDRK with 6 stages (update_displacement_LDDRK.F90);
   * stf holds nstage values per step: stf[isrc][it][stage] */
  int time_scheme;
  int nstage;
  const float *alpha_lddrk, *beta_lddrk;     /* 6 each (ALPHA_LDDRK, BETA_LDDRK) */
  /* anisotropy (NULL = isotropic): per-element flag, c11 c13 c15 c33 c35 c55 per GLL point */
  const int *ispec_is_anisotropic;
  const float *c11, *c13, *c15, *c33, *c35, *c55;
  /* viscoelastic 3 SLS (NULL = elastic), nspec*25*3 [ispec][j][i][sls]; all zero at a
   * point = no attenuation there.  Newmark: A/B recursive-convolution coefficients
   * (prepare_attenuation.f90:378-396); LDDRK: 1/tau_sigma and phi (attenuation_model.f90). */
  const float *att_a1, *att_b1, *att_a2, *att_b2;
  const float *att_itau1, *att_phi1, *att_itau2, *att_phi2;
  /* CPML absorbing layer (pml_region NULL = none), the arrays of prepare_pml.f90 /
   * pml_init.F90: region per element, 0 outside the layer, 1 CPML_X_ONLY, 2 CPML_Z_ONLY,
   * 3 CPML_XZ; damping profiles K, d, alpha per element GLL point (nspec*25, read in
   * the layer); rho and the Jacobian per element GLL point (nspec*25) for the layer's
   * acceleration terms; the points of the layer's outer edge, zeroed every step
   * (pml_boundary_elastic, pml_compute.f90:545-574); DT in double for the
   * convolution coefficients.  Isotropic forward runs only, not together with
   * Stacey conditions (read_parameter_file.F90:1495); with attenuation, Newmark only
   * (pml_compute_memory_variables.f90:736-741). */
  const int *pml_region;
  const double *pml_K_x, *pml_K_z, *pml_d_x, *pml_d_z, *pml_alpha_x, *pml_alpha_z;
  const float *rhostore, *jacobian;
  int npml_edge;
  const int *pml_edge_iglob;
  double pml_dt;
  /* CPML in attenuating solids (pml_compute_memory_variables_viscoelastic,
   * pml_compute_memory_variables.f90:546-894): pml_visco[e] = 1 for a layer element
   * whose largest Qkappa and Qmu are both below 9998.999 (those elements take the
   * viscoelastic update, compute_forces_viscoelastic.F90:249-267; NULL = none).  They
   * need att_itau1/2 and att_phi1/2 above (also under Newmark), the strain relaxation
   * times tau_epsilon_nu1/2 (nspec*25*3) and Mu_nu1/2 (nspec*25) of
   * attenuation_model.f90:147-160. */
  const int *pml_visco;
  const float *att_teps1, *att_teps2;
  const float *att_mu1, *att_mu2;
  /* tiles of the CPML layer: elements per tile and threads per CTA (128, 250, 256
   * or 512) of their kernel; 0 = tile_elems and threads_per_block */
  int pml_tile_elems;
  int pml_threads_per_block;
} sf2d_elastic_desc;

/* Makes device rank % (visible devices) current for the calling thread, as
 * initialize_cuda_device (src/gpu/initialize_cuda.cu:50-125) does for each MPI
 * rank; *ndevices (may be NULL) gets the number of visible devices.  Every
 * later call of this library on the thread uses that device.  The library
 * links its own CUDA runtime, so a host that selected a device through another
 * runtime (torch.cuda.set_device, say) calls this with the same rank.
 * SF2D_ERR_CUDA when no device is visible. */
int sf2d_initialize_device(int rank, int *ndevices);

/* Builds the tiled device layout and uploads everything (fields start at 0). */
int sf2d_elastic_create(const sf2d_elastic_desc *desc, sf2d_solver **out);

/* Host <-> device copies of the wavefields, nglob*2 floats each in the
 * original global numbering.  NULL pointers are skipped (set: zero-filled). */
int sf2d_set_fields(sf2d_solver *s, const float *displ, const float *veloc, const float *accel);
int sf2d_get_fields(sf2d_solver *s, float *displ, float *veloc, float *accel);

/* Advances nstep time steps on the device.  When `seismograms` is not NULL
 * the receiver traces of these steps are copied to it (nrec*nstep*2 doubles,
 * [irec][it][comp], rotated by cosrot/sinrot) before returning.  Returns
 * SF2D_ERR_UNSTABLE if a displacement became NaN or exceeded 1e25 (the check
 * of check_stability.F90:95-98), after finishing the steps. */
int sf2d_run(sf2d_solver *s, int nstep, double *seismograms);

/* Same without a host sync or copy: the steps are queued on the solver's
 * stream (CUDA graphs of fixed step chunks).  sf2d_synchronize waits (with a
 * timeout in seconds, <= 0 meaning none) and returns the stability status. */
int sf2d_enqueue(sf2d_solver *s, int nstep);
/* (sf2d_synchronize returns SF2D_ERR_TIMEOUT when the steps have not finished
 * within timeout_s; they keep running and a later call waits for them.) */
/* Builds and uploads the CUDA graph of one step chunk now (capture runs
 * nothing), so that a later sf2d_enqueue starts without that host work. */
int sf2d_prepare(sf2d_solver *s);
int sf2d_synchronize(sf2d_solver *s, double timeout_s);

/* Packed batches (several independent meshes in one solver, the GPU form of
 * NUMBER_OF_SIMULTANEOUS_RUNS, src/shared/parallel.F90:40-50): elem_member
 * (nspec values in [0, nmembers)) names the member of every element.  From
 * then on a member whose displacement becomes NaN or exceeds 1e25 is masked:
 * its tiles and points keep their last values and stop advancing, the other
 * members run on, and the run does not return SF2D_ERR_UNSTABLE for it.  The
 * reference instead aborts all runs and leaves a runXXXX_failed marker
 * (parallel.F90:190-214).  A tile or point may not mix members
 * (SF2D_ERR_INVALID).  Clears every member's status. */
int sf2d_set_members(sf2d_solver *s, const int *elem_member, int nmembers);
/* status (nmembers ints): 0 running, 1 masked because its field blew up. */
int sf2d_member_status(sf2d_solver *s, int *status);

/* Copies receiver traces [it0, it0+nstep) already recorded on the device. */
int sf2d_copy_seismograms(sf2d_solver *s, int it0, int nstep, double *out);

/* Maximum displacement norm over all points (check_stability.F90). */
int sf2d_get_norm(sf2d_solver *s, float *max_norm);

/* Steps done since creation. */
int sf2d_step_index(sf2d_solver *s, int *it);

/* The cudaStream_t the solver launches on (as void*). */
int sf2d_get_stream(sf2d_solver *s, void **stream);

/* Times `nstep` steps launched one kernel at a time with CUDA events around
 * each launch; writes the average milliseconds per launch of the element
 * kernel (ms[0]), the shared-point kernel (ms[1]) and their sum per time step
 * (ms[2], all LDDRK stages).  The steps advance the wavefield like sf2d_run. */
int sf2d_time_kernels(sf2d_solver *s, int nstep, float *ms);

/* Layout statistics: [ntiles, nshared points, max local points, max elements
 * per tile, device bytes, dynamic shared memory per CTA, threads per CTA,
 * partial-sum slots]. */
int sf2d_layout_info(sf2d_solver *s, long long *info8);

/* Kernel launches that sf2d_enqueue(s, nstep) issues (all stages, receiver
 * kernels included), for launch accounting. */
int sf2d_launch_count(sf2d_solver *s, int nstep, long long *launches);

int sf2d_destroy(sf2d_solver *s);

const char *sf2d_last_error(void);

/* ---- misfit gradient (forward/backward pair) ----
 * sf2d_fwi_create builds a forward and an adjoint solver for one medium and
 * source (Newmark only) and reserves checkpoint_every displacement frames plus
 * one state checkpoint per checkpoint_every steps in device memory.
 * rhostore/kappastore (nspec*25) are used for the final kernel scaling.
 * Replaces the reference's SIMULATION_TYPE = 3 path with undo_attenuation
 * checkpointing (iterate_time_undoatt.F90:35-653, compute_kernels.f90:75-292,
 * save_adjoint_kernels.f90:79-141). */
typedef struct sf2d_fwi sf2d_fwi;
int sf2d_fwi_create(const sf2d_elastic_desc *desc, const float *rhostore, const float *kappastore,
                    int checkpoint_every, sf2d_fwi **out);
/* Forward run from rest over desc->nstep steps, saving the checkpoints;
 * seismograms (may be NULL): nrec*nstep*2 doubles. */
int sf2d_fwi_forward(sf2d_fwi *f, double *seismograms);
/* Adjoint sweep with adjoint source adj_src[irec][it][comp] (nrec*nstep*2,
 * time order; the residual for an L2 waveform misfit).  Writes the scaled
 * kernels rho_kl, kappa_kl, mu_kl (nspec*25 each, [ispec][j][i]):
 * rho_kl = -rho dt sum(a_adj . u), kappa_kl = -kappa dt sum(div div),
 * mu_kl = -2 mu dt sum(eps:eps - 1/3 div div). */
int sf2d_fwi_backward(sf2d_fwi *f, const float *adj_src, float *rho_kl, float *kappa_kl, float *mu_kl);
/* The approximate Hessian of the kernel run (APPROXIMATE_HESS_KL,
 * compute_kernels.f90:749-800, elastic part): the forward sweep also keeps the
 * forward accelerations of each segment (one more frame buffer) and the adjoint
 * sweep sums |b_accel|^2 and accel . b_accel at every point.  Call before
 * sf2d_fwi_forward.  sf2d_fwi_hessian then writes rhorho_el_Hessian_final1 and
 * _final2 (nspec*25 each, [ispec][j][i]) of the last backward sweep, scaled by
 * dt as the reference accumulates them. */
int sf2d_fwi_enable_hessian(sf2d_fwi *f);
int sf2d_fwi_hessian(sf2d_fwi *f, float *hess1, float *hess2);
/* Receiver traces of the adjoint wavefield of the last sf2d_fwi_backward, in
 * the adjoint run's own time order (nrec*nstep*2 doubles, [irec][it][comp]):
 * the seismograms a kernel run writes (write_seismograms.F90:36-150 records
 * the adjoint field when SIMULATION_TYPE = 3). */
int sf2d_fwi_adjoint_seismograms(sf2d_fwi *f, double *seismograms);
/* The kernel integrand sums of the last sf2d_fwi_backward before the scaling of
 * save_adjoint_kernels.f90:134-141 (nspec*25 each, element order): rho_kl =
 * sum a_adj . b_u, kappa_kl = sum div u_adj div b_u, mu_kl = sum of the
 * deviatoric strain products (compute_kernels.f90:75-292), as the reference's
 * transfer_kernels_el_to_host hands them to the host. */
int sf2d_fwi_kernel_sums(sf2d_fwi *f, float *rho_kl, float *kappa_kl, float *mu_kl);
/* The adjoint wavefield at the end of the last sf2d_fwi_backward (each
 * 2*nglob, may be NULL): displ_elastic, veloc_elastic and accel_elastic of a
 * kernel run, as transfer_fields_el_from_device hands them to the host at its
 * end (iterate_time.F90:462-504). */
int sf2d_fwi_adjoint_fields(sf2d_fwi *f, float *displ, float *veloc, float *accel);
int sf2d_fwi_destroy(sf2d_fwi *f);

/* ---- batches of shots and models (one launch per step for all) ----
 * The GPU counterpart of NUMBER_OF_SIMULTANEOUS_RUNS (src/shared/parallel.F90:
 * 40-50, 1714), which runs independent simulations as separate MPI groups.
 * A batch packs its members into one disconnected mesh: a member is a shot on
 * one of the models, with the model's arrays and the shot's sources; its
 * elements, points, absorbing points, sources and receivers are appended with
 * offsets, and its element centres are moved 1e8 m apart along x so that no
 * tile mixes members.  Models must share nstep, the time step, the time scheme,
 * the seismogram type and rotation, and their physics (anisotropy and
 * attenuation present in all or none); CPML layers are not packed.  Receivers,
 * seismograms and adjoint sources are in member order (each member's
 * receivers in its model's order). */
typedef struct {
  int model;                 /* 0-based index into the models array */
  int nsrc;                  /* the shot's sources, in place of the model's */
  const int *src_ispec;      /* nsrc elements of the model */
  const float *sourcearrays; /* nsrc*25*2 [isrc][j][i][comp] */
  const float *stf;          /* nsrc*nstep*nstage */
} sf2d_shot;
typedef struct sf2d_batch sf2d_batch;
/* nshots = 0: one member per model with its own sources.  checkpoint_every >
 * 0 makes a gradient batch (Newmark only): rhostore/kappastore then hold one
 * nspec*25 array per model for the kernel scaling, as in sf2d_fwi_create;
 * checkpoint_every = 0 makes a forward batch (rhostore/kappastore unused), whose
 * members are masked one by one if their field blows up (sf2d_set_members). */
int sf2d_batch_create(const sf2d_elastic_desc *models, int nmodels, const sf2d_shot *shots, int nshots,
                      const float *const *rhostore, const float *const *kappastore, int checkpoint_every,
                      sf2d_batch **out);
/* [members, total elements, total points, total receivers] */
int sf2d_batch_info(sf2d_batch *b, long long *info4);
/* Forward run of every member from rest over nstep steps; seismograms (may be
 * NULL): nrec_total*nstep*2 doubles.  A gradient batch keeps its checkpoints. */
int sf2d_batch_run_forward(sf2d_batch *b, double *seismograms);
/* Gradient batch: adjoint sweep with adj_src (nrec_total*nstep*2, time order);
 * the kernels rho_kl, kappa_kl, mu_kl of each model, summed over its shots
 * (each array: the models' nspec*25 one after the other, scaled as
 * sf2d_fwi_backward scales them). */
int sf2d_batch_run_adjoint(sf2d_batch *b, const float *adj_src, float *rho_kl, float *kappa_kl, float *mu_kl);
/* Forward batch: per member 0 running, 1 masked (blew up). */
int sf2d_batch_member_status(sf2d_batch *b, int *status);
int sf2d_batch_destroy(sf2d_batch *b);

/* ---- kernel smoothing (post-gradient step) ----
 * Gaussian smoothing of per-element-point fields, as
 * src/tomography/postprocess_sensitivity_kernels/smooth_sem.F90:63-467 does to
 * sensitivity kernels (its GPU path: src/gpu/smooth_cuda.cu, kernels/process_smooth.cu):
 * out_k(i) = sum_j G J_j w_j f_k(j) / sum_j G J_j w_j with
 * G = exp(-dx^2 / (2 sigma_h^2) - dz^2 / (2 sigma_v^2)) over every element GLL
 * point j.  x, z, jacobian, fields and out are host arrays of nspec*25 values
 * per field ([ispec][j][i]; fields and out [field][ispec][j][i]); wgll_sq the
 * 25 products wxgll(i) wzgll(j) [j][i].  Points farther than `cutoff` standard
 * deviations (the ellipse (dx/sigma_h)^2 + (dz/sigma_v)^2 <= cutoff^2) are
 * left out: their weights are below exp(-cutoff^2/2) of the largest (6: 1.5e-8).
 * The reference's CPU program sums over every pair; its GPU kernel leaves out
 * element pairs whose first points are farther than 3 sigma + max(sigma)/2.
 * Sums in double.  Returns after the results are in `out`. */
#define SF2D_SMOOTH_MAX_FIELDS 4
int sf2d_smooth(int nspec, const float *x, const float *z, const float *jacobian, const float *wgll_sq,
                int nfields, const float *fields, float sigma_h, float sigma_v, float cutoff, float *out,
                void *stream);

/* Host-only diagnostic, no GPU needed: builds the tiling of a mesh and checks
 * its invariants (one device id per point, local ibool consistent with
 * ibool, colours conflict-free, shared-point slots complete and in tile
 * order).  out8 = [ntiles, nshared, max local points, max elements per tile,
 * max colours, interior points, partial-sum slots, 0].  Returns 0 when every
 * invariant holds, a negative code naming the first that fails otherwise.
 * No reference counterpart (the reference assembles with atomics). */
int sf2d_tiling_stats(int nspec, int nglob, const int *ibool, const double *centroid_xz, int tile_elems,
                      long long *out8);

/* Largest member count sf2d_member_norms_noalloc accepts (its static scratch). */
#define SF2D_NOALLOC_MAX_MEMBERS 4096

/* Maximum displacement norm per member of a batch, with no device allocation.
 * No counterpart in the reference: its get_norm_elastic_from_device
 * (src/gpu/check_fields_cuda.cu:358) allocates and frees its per-block maxima
 * on every call and takes one field.  This one serves callers that own all
 * of their device memory (a host code that plans it before the time loop, or
 * a pooling allocator that holds the GPU's free memory), where a cudaMalloc
 * can fail and a cudaFree waits for the whole device.
 *
 * d_field: caller-owned device array of (ux, uz) float pairs, 8-byte aligned,
 * on the current device.  Member m covers the points
 * [offsets[m], offsets[m+1]); offsets (host, nmembers+1 values) start at
 * >= 0 and never decrease, and must stay inside the field's allocation
 * (checked).  max_norm (host, nmembers floats) receives
 * max sqrt(ux^2 + uz^2) per member, +inf where a NaN occurs, 0 for an empty
 * member.  1 <= nmembers <= SF2D_NOALLOC_MAX_MEMBERS, else SF2D_ERR_INVALID.
 * stream: cudaStream_t (NULL = default stream); the call returns after the
 * stream has finished the reduction.
 *
 * Intermediates live in one static device array (49,160 bytes per device).
 * The first call on each device looks its address up with that device
 * current, so make that first call before any stream capture.  Calls that
 * overlap on one device (from several host threads) race on that array:
 * serialise them. */
int sf2d_member_norms_noalloc(const float *d_field, const int64_t *offsets, int nmembers, float *max_norm,
                              void *stream);

#ifdef __cplusplus
}
#endif
#endif
