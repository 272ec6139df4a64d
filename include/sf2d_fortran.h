/*
 * sf2d_fortran.h -- the reference's Fortran-to-GPU interface, provided by
 * libsf2d_b200.so so that the SPECFEM2D Fortran host links against this
 * library in place of its src/gpu objects with no change at its call sites.
 *
 * Every entry point has the name, argument list and argument meaning of the
 * reference's src/gpu routine of the same name (the complete list is
 * src/gpu/specfem2D_gpu_cuda_method_stubs.c:51-724).  gfortran calls
 * `call name(args)` as the C symbol name_ with every argument by reference;
 * arrays are Fortran column-major, ibool and element/receiver indices are
 * 1-based, logicals arrive as int (nonzero = true).  Mesh_pointer is the
 * Fortran integer(kind=8) handle that prepare_constants_device fills.
 *
 * Errors behave as the reference's do (exit_on_error, helper_functions.cu):
 * the message goes to stderr and the process exits with EXIT_FAILURE.
 *
 * Provided: the elastic forward path (SIMULATION_TYPE = 1, Newmark, isotropic,
 * anisotropic and viscoelastic elements, Stacey conditions, force and moment
 * tensor sources, displacement, velocity or acceleration seismograms, one
 * process).  The reference splits one time step over several calls
 * (update_displacement_cuda, compute_forces_viscoelastic_cuda for the outer
 * and inner phases, compute_stacey_viscoelastic_cuda,
 * compute_add_sources_el_cuda, kernel_3_a_cuda); this library advances the
 * whole step in its fused tile kernels when kernel_3_a_cuda, the last call of
 * the step, arrives, and the earlier calls only check the sequence.
 * compute_seismograms_cuda does not synchronise the device each step: it hands
 * the traces over when the host's seismogram buffer is full or at the last
 * step, as the reference copies them.
 *
 * Not provided (the call prints which entry point of include/sf2d_b200.h or
 * include/sf2d_coupled.h covers it and exits): fluid domains, CPML, kernel
 * (SIMULATION_TYPE = 3) runs with backward reconstruction, MPI halo buffers,
 * moving sources, smoothing, the Hessian and the debug helpers.
 */
#ifndef SF2D_FORTRAN_H
#define SF2D_FORTRAN_H

#ifdef __cplusplus
extern "C" {
#endif

typedef float realw; /* CUSTOM_REAL = 4 */

/* --- device and memory --- */
void initialize_cuda_device_(int* myrank_f, int* ncuda_devices);
void initialize_cuda_aware_mpi_();
void pause_for_debug_();
void output_free_device_memory_(int* myrank_f);
void get_free_device_memory_(realw* free, realw* used, realw* total);

/* --- set-up and clean-up --- */
void prepare_constants_device_(long* Mesh_pointer, int* h_NGLLX, int* NSPEC_AB, int* NGLOB_AB, realw* h_xix, realw* h_xiz, realw* h_gammax, realw* h_gammaz, realw* h_kappav, realw* h_muv, int* h_ibool, int* num_interfaces_ext_mesh, int* max_nibool_interfaces_ext_mesh, int* h_nibool_interfaces_ext_mesh, int* h_ibool_interfaces_ext_mesh, realw* h_hprime_xx, realw* h_hprimewgll_xx, realw* h_wxgll, int* STACEY_BOUNDARY_CONDITIONS, int* PML_BOUNDARY_CONDITIONS, int* h_ispec_is_inner, int* nsources_local_f, realw* h_sourcearrays, realw* h_source_time_function, int* NSTEP, int* h_ispec_selected_source, int* h_ispec_selected_rec_loc, int* nrec_local, realw* h_cosrot, realw* h_sinrot, int* SIMULATION_TYPE, int* P_SV, int* nspec_acoustic, int* nspec_elastic, int* ispec_is_acoustic, int* ispec_is_elastic, int* h_myrank, int* SAVE_FORWARD, realw* h_xir_store, realw* h_gammar_store, int* h_NSIGTYPE, int* h_seismotypeVec, int* nlength_seismogram);
void prepare_fields_elastic_device_(long* Mesh_pointer, realw* rmassx, realw* rmassz, int* num_phase_ispec_elastic, int* phase_ispec_inner_elastic, int* ispec_is_anisotropic, int* ANISOTROPY, realw* c11store, realw* c12store, realw* c13store, realw* c15store, realw* c23store, realw* c25store, realw* c33store, realw* c35store, realw* c55store, int* h_ninterface_elastic, int* h_inum_interfaces_elastic, int* ATTENUATION_VISCOELASTIC, realw* h_A_newmark_mu, realw* h_B_newmark_mu, realw* h_A_newmark_kappa, realw* h_B_newmark_kappa);
void prepare_stacey_device_(long* Mesh_pointer, int* ACOUSTIC_SIMULATION, int* ELASTIC_SIMULATION, realw* rho_vp, realw* rho_vs, int* h_nspec_bottom, int* h_nspec_left, int* h_nspec_right, int* h_nspec_top, int* h_abs_boundary_ispec, int* h_abs_boundary_ij, realw* h_abs_boundary_normal, realw* h_abs_boundary_jacobian1Dw, int* h_num_abs_boundary_faces, int* h_edge_abs, int* h_ib_bottom, int* h_ib_left, int* h_ib_right, int* h_ib_top);
void prepare_cleanup_device_(long* Mesh_pointer, int* ACOUSTIC_SIMULATION, int* ELASTIC_SIMULATION, int* ANISOTROPY, int* APPROXIMATE_HESS_KL, int* ATTENUATION_VISCOACOUSTIC, int* ATTENUATION_VISCOELASTIC, int* NO_BACKWARD_RECONSTRUCTION, realw* h_no_backward_acoustic_buffer);

/* --- one elastic time step, in the order of compute_gpu_elastic.f90 and write_seismograms.F90 --- */
void update_displacement_cuda_(long* Mesh_pointer, realw* deltat_F, realw* deltatsqover2_F, realw* deltatover2_F, realw* b_deltat_F, realw* b_deltatsqover2_F, realw* b_deltatover2_F);
void compute_forces_viscoelastic_cuda_(long* Mesh_pointer, int* iphase, realw* deltat, int* nspec_outer_elastic, int* nspec_inner_elastic, int* ANISOTROPY, int* ATTENUATION_VISCOELASTIC, int* compute_wavefield_1, int* compute_wavefield_2);
void compute_stacey_viscoelastic_cuda_(long* Mesh_pointer, int* iphasef, realw* h_b_absorb_elastic_left, realw* h_b_absorb_elastic_right, realw* h_b_absorb_elastic_top, realw* h_b_absorb_elastic_bottom, int* compute_wavefield_1, int* compute_wavefield_2, int* UNDO_ATTENUATION_AND_OR_PML);
void compute_add_sources_el_cuda_(long* Mesh_pointer, int* iphasef, int* itf);
void kernel_3_a_cuda_(long* Mesh_pointer, realw* deltatover2_F, realw* b_deltatover2_F, int* compute_wavefield_1, int* compute_wavefield_2);
void compute_seismograms_cuda_(long* Mesh_pointer_f, int* i_sigf, double* sisux, double* sisuz, int* seismo_currentf, int* nlength_seismogramf, int* ELASTIC_SIMULATION, int* ACOUSTIC_SIMULATION, int* USE_TRICK_FOR_BETTER_PRESSURE, int* ATTENUATION_VISCOELASTIC, int* itf, int* it_endf);
void get_norm_elastic_from_device_(realw* norm, long* Mesh_pointer, const int* FORWARD_OR_ADJOINT);

/* --- wavefield transfers --- */
void transfer_fields_el_to_device_(int* size, realw* displ, realw* veloc, realw* accel, long* Mesh_pointer);
void transfer_fields_el_from_device_(int* size, realw* displ, realw* veloc, realw* accel, long* Mesh_pointer);
void transfer_displ_from_device_(int* size, realw* displ, long* Mesh_pointer);
void transfer_accel_from_device_(int* size, realw* accel, long* Mesh_pointer);
void transfer_accel_to_device_(int* size, realw* accel, long* Mesh_pointer);

/* --- not provided: each prints which interface covers it and exits --- */
void transfer_boun_pot_from_device_(long* Mesh_pointer, realw* h_send_potential_dot_dot_buffer, const int* FORWARD_OR_ADJOINT);
void transfer_asmbl_pot_to_device_(long* Mesh_pointer, realw* h_buffer_recv_scalar_gpu, const int* FORWARD_OR_ADJOINT);
void transfer_boun_accel_from_device_(long* Mesh_pointer, realw* h_send_accel_buffer, const int* FORWARD_OR_ADJOINT);
void transfer_boundary_from_device_a_(long* Mesh_pointer);
void prepare_boundary_on_device_(long* Mesh_pointer);
void transfer_boundary_to_device_a_(long* Mesh_pointer, realw* buffer_recv_vector_gpu, const int* max_nibool_interfaces_ext_mesh);
void transfer_asmbl_accel_to_device_(long* Mesh_pointer, realw* buffer_recv_vector_gpu, const int* max_nibool_interfaces_ext_mesh, const int* nibool_interfaces_ext_mesh, const int* ibool_interfaces_ext_mesh, const int* FORWARD_OR_ADJOINT);
void sync_copy_from_device_(long* Mesh_pointer, int* iphase, realw* send_buffer);
void get_norm_acoustic_from_device_(realw* norm, long* Mesh_pointer, const int* FORWARD_OR_ADJOINT);
void get_max_accel_(int* itf, int* sizef, long* Mesh_pointer);
void check_max_norm_displ_gpu_(int* size, realw* displ, long* Mesh_pointer, int* announceID);
void check_max_norm_vector_(int* size, realw* vector1, int* announceID);
void check_max_norm_displ_(int* size, realw* displ, int* announceID);
void check_max_norm_b_displ_gpu_(int* size, realw* b_displ, long* Mesh_pointer, int* announceID);
void check_max_norm_b_accel_gpu_(int* size, realw* b_accel, long* Mesh_pointer, int* announceID);
void check_max_norm_b_veloc_gpu_(int* size, realw* b_veloc, long* Mesh_pointer, int* announceID);
void check_max_norm_b_displ_(int* size, realw* b_displ, int* announceID);
void check_max_norm_b_accel_(int* size, realw* b_accel, int* announceID);
void check_error_vectors_(int* sizef, realw* vector1, realw* vector2);
void compute_add_sources_ac_cuda_(long* Mesh_pointer, int* iphasef, int* itf);
void compute_add_sources_ac_s3_cuda_(long* Mesh_pointer, int* iphasef, int* itf);
void compute_add_moving_sources_ac_cuda_(long* Mesh_pointer, int* iphase_f, int* nsources_local_moving, int* itf, int* NSTEP_f, int* nsources_f);
void add_sources_ac_sim_2_or_3_cuda_(long* Mesh_pointer, int* iphasef, int* itf, int* nadj_rec_local, int* NSTEP);
void compute_add_sources_el_s3_cuda_(long* Mesh_pointer, int* iphasef, int* itf);
void add_sources_el_sim_type_2_or_3_(long* Mesh_pointer, int* iphasef, int* itf, int* nadj_rec_local, int* NSTEP);
void compute_coupling_ac_el_cuda_(long* Mesh_pointer, int* iphasef, int* num_coupling_ac_el_facesf, int* FORWARD_OR_ADJOINT);
void compute_coupling_el_ac_cuda_(long* Mesh_pointer, int* iphasef, int* num_coupling_ac_el_facesf, int* FORWARD_OR_ADJOINT);
void compute_forces_acoustic_cuda_(long* Mesh_pointer, int* iphase, int* nspec_outer_acoustic, int* nspec_inner_acoustic, int* ATTENUATION_VISCOACOUSTIC, int* compute_wavefield_1, int* compute_wavefield_2);
void compute_kernels_elastic_cuda_(long* Mesh_pointer, realw* deltat);
void compute_kernels_acoustic_cuda_(long* Mesh_pointer, realw* deltat);
void compute_kernels_hess_cuda_(long* Mesh_pointer, int* ELASTIC_SIMULATION, int* ACOUSTIC_SIMULATION);
void compute_stacey_acoustic_cuda_(long* Mesh_pointer, int* iphasef, realw* h_b_absorb_potential_left, realw* h_b_absorb_potential_right, realw* h_b_absorb_potential_top, realw* h_b_absorb_potential_bottom, int* compute_wavefield_1, int* compute_wavefield_2, int* UNDO_ATTENUATION_AND_OR_PML);
void acoustic_enforce_free_surf_cuda_(long* Mesh_pointer, int* compute_wavefield_1, int* compute_wavefield_2);
void pml_boundary_acoustic_cuda_(long* Mesh_pointer, int* compute_wavefield_1, int* compute_wavefield_2);
void prepare_fields_acoustic_device_(long* Mesh_pointer, realw* rmass_acoustic, realw* rhostore, realw* kappastore, int* num_phase_ispec_acoustic, int* phase_ispec_inner_acoustic, int* num_free_surface_faces, int* free_surface_ispec, int* free_surface_ijk, int* ELASTIC_SIMULATION, int* num_coupling_ac_el_faces, int* coupling_ac_el_ispec, int* coupling_ac_el_ijk, realw* coupling_ac_el_normal, realw* coupling_ac_el_jacobian2Dw, int* h_ninterface_acoustic, int* h_inum_interfaces_acoustic, int* ATTENUATION_VISCOACOUSTIC, realw* h_A_newmark, realw* h_B_newmark, int* NO_BACKWARD_RECONSTRUCTION, realw* h_no_backward_acoustic_buffer);
void prepare_fields_acoustic_adj_dev_(long* Mesh_pointer, int* APPROXIMATE_HESS_KL, int* ATTENUATION_VISCOACOUSTIC, int* NO_BACKWARD_RECONSTRUCTION);
void prepare_fields_elastic_adj_dev_(long* Mesh_pointer, int* size_f, int* APPROXIMATE_HESS_KL, int* ATTENUATION_VISCOELASTIC, int* NO_BACKWARD_RECONSTRUCTION);
void prepare_sim2_or_3_const_device_(long* Mesh_pointer, int* nadj_rec_local, realw* h_source_adjoint, int* NSTEP);
void prepare_pml_device_(long* Mesh_pointer, int* NSPEC_PML, int* NSPEC_PML_X, int* NSPEC_PML_Z, int* NSPEC_PML_XZ, int* h_spec_to_pml, realw* h_abs_normalized, realw* ALPHA_MAX_PML, realw* d0_max, realw* deltat, realw* h_alphax_store, realw* h_alphaz_store, realw* h_betax_store, realw* h_betaz_store, int* PML_nglob_abs_acoustic_f, int* h_PML_abs_points_acoustic);
void prepare_moving_sources_cuda_(long* Mesh_pointer, int* h_nsources_local_f_moving, int* NSOURCES, realw* h_sourcearrays_moving, int* h_ispec_selected_source_moving, int* NSTEP, realw* h_source_time_function_moving);
void prepare_arrays_gpu_(long* Container, realw* xstore_me, realw* zstore_me, realw* sigma_h2_inv, realw* sigma_v2_inv, realw* h_criterion, realw* v_criterion, int* nspec_me, int* nker, realw* wgll_sq);
void compute_smooth_(long* smooth_pointer, realw* jacobian, realw* xstore_other, realw* zstore_other, realw* data_other, const int* nspec_other);
void get_smooth_(long* smooth_pointer, realw* data_smooth);
void transfer_b_fields_to_device_(int* size, realw* b_displ, realw* b_veloc, realw* b_accel, long* Mesh_pointer);
void transfer_b_fields_from_device_(int* size, realw* b_displ, realw* b_veloc, realw* b_accel, long* Mesh_pointer);
void transfer_b_accel_from_device_(int* size, realw* b_accel, long* Mesh_pointer);
void transfer_b_displ_from_device_(int* size, realw* displ, long* Mesh_pointer);
void transfer_kernels_el_to_host_(long* Mesh_pointer, realw* h_rho_kl, realw* h_mu_kl, realw* h_kappa_kl, int* NSPEC_AB);
void transfer_fields_ac_to_device_(int* size, realw* potential_acoustic, realw* potential_dot_acoustic, realw* potential_dot_dot_acoustic, long* Mesh_pointer);
void transfer_b_fields_ac_to_device_(int* size, realw* b_potential_acoustic, realw* b_potential_dot_acoustic, realw* b_potential_dot_dot_acoustic, long* Mesh_pointer);
void transfer_fields_ac_from_device_(int* size, realw* potential_acoustic, realw* potential_dot_acoustic, realw* potential_dot_dot_acoustic, long* Mesh_pointer);
void transfer_b_fields_ac_from_device_(int* size, realw* b_potential_acoustic, realw* b_potential_dot_acoustic, realw* b_potential_dot_dot_acoustic, long* Mesh_pointer);
void transfer_b_potential_ac_from_device_(int* size, realw* b_potential_acoustic, long* Mesh_pointer);
void transfer_b_potential_ac_to_device_(int* size, realw* b_potential_acoustic, long* Mesh_pointer);
void transfer_dot_dot_from_device_(int* size, realw* potential_dot_dot_acoustic, long* Mesh_pointer);
void transfer_b_dot_dot_from_device_(int* size, realw* b_potential_dot_dot_acoustic, long* Mesh_pointer);
void transfer_kernels_ac_to_host_(long* Mesh_pointer, realw* h_rho_ac_kl, realw* h_kappa_ac_kl, int* NSPEC_AB);
void transfer_kernels_hess_el_tohost_(long* Mesh_pointer, realw* h_hess_kl, int* NSPEC_AB);
void transfer_kernels_hess_ac_tohost_(long* Mesh_pointer, realw* h_hess_ac_kl, int* NSPEC_AB);
void transfer_viscoacoustic_b_var_to_device_(int* size, realw* b_e1_acous_sf, realw* b_sum_forces_old, long* Mesh_pointer);
void transfer_viscoacoustic_var_from_device_(int* size, realw* e1_acous_sf, realw* sum_forces_old, long* Mesh_pointer);
void transfer_viscoelastic_b_var_to_device_(int* size, realw* b_e1, realw* b_e11, realw* b_e13, realw* b_dux_dxl_old, realw* b_duz_dzl_old, realw* b_dux_dzl_plus_duz_dxl_old, long* Mesh_pointer);
void transfer_viscoelastic_var_from_device_(int* size, realw* e1, realw* e11, realw* e13, realw* dux_dxl_old, realw* duz_dzl_old, realw* dux_dzl_plus_duz_dxl_old, long* Mesh_pointer);
void transfer_async_pot_ac_from_device_(realw* pot_buffer, long* Mesh_pointer);
void transfer_async_pot_ac_to_device_(realw* pot_buffer, long* Mesh_pointer);
void transfer_compute_kernel_answers_from_device_(long* Mesh_pointer, realw* rho_kl, int* size_rho, realw* mu_kl, int* size_mu, realw* kappa_kl, int* size_kappa);
void transfer_compute_kernel_fields_from_device_(long* Mesh_pointer, realw* accel, int* size_accel, realw* b_displ, int* size_b_displ, realw* epsilondev_xx, realw* epsilondev_yy, realw* epsilondev_xy, realw* epsilondev_xz, realw* epsilondev_yz, int* size_epsilondev, realw* b_epsilondev_xx, realw* b_epsilondev_yy, realw* b_epsilondev_xy, realw* b_epsilondev_xz, realw* b_epsilondev_yz, int* size_b_epsilondev, realw* rho_kl, int* size_rho, realw* mu_kl, int* size_mu, realw* kappa_kl, int* size_kappa, realw* epsilon_trace_over_3, realw* b_epsilon_trace_over_3, int* size_epsilon_trace_over_3);
void update_displacement_ac_cuda_(long* Mesh_pointer, realw* deltat_F, realw* deltatsqover2_F, realw* deltatover2_F, realw* b_deltat_F, realw* b_deltatsqover2_F, realw* b_deltatover2_F, int* compute_b_wavefield, int* UNDO_ATTENUATION_AND_OR_PML);
void kernel_3_b_cuda_(long* Mesh_pointer, realw* deltatover2_F, realw* b_deltatover2_F);
void kernel_3_acoustic_cuda_(long* Mesh_pointer, realw* deltatover2, realw* b_deltatover2, int* compute_wavefield_1, int* compute_wavefield_2);

#ifdef __cplusplus
}
#endif
#endif
