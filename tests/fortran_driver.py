"""Drives libsf2d_b200.so through the reference's Fortran-to-GPU entry points
(include/sf2d_fortran.h) in the order the SPECFEM2D Fortran host calls them,
with arguments passed by reference as gfortran passes them:

* prepare_GPU (src/specfem2D/prepare_gpu.f90:34-320): initialize_cuda_device,
  prepare_constants_device, prepare_fields_acoustic_device (fluid elements),
  prepare_fields_elastic_device (solid elements), prepare_Stacey_device,
  transfer_fields_el_to_device / transfer_fields_ac_to_device;
* with CPML layers (fluid-only meshes) prepare_PML_device, and
  pml_boundary_acoustic_cuda after each fluid forces call;
* each time step it = 1..NSTEP (iterate_time.F90:146-260):
  update_displacement_ac_cuda and update_displacement_cuda
  (update_displacement_Newmark.F90:150-240, 500-549); with fluid elements
  compute_forces_viscoacoustic_GPU (compute_gpu_acoustic.f90:36-180): the
  free-surface call, forces for iphase 1 with Stacey, coupling and sources,
  forces for iphase 2, kernel_3_acoustic_cuda, the free-surface call again;
  with solid elements compute_forces_viscoelastic_GPU (compute_gpu_elastic.f90:36-215):
  forces for iphase 1 with Stacey, coupling and sources, forces for iphase 2,
  kernel_3_a_cuda; then write_seismograms (write_seismograms.F90:199-205) and,
  every `check_every` steps, check_stability's get_norm_*_from_device;
* prepare_cleanup_device.

`run_kernel` drives a kernel run (SIMULATION_TYPE = 3) of a solid mesh the
same way: prepare_fields_elastic_adj_dev and prepare_sim2_or_3_const_device at
set-up, both wavefields in each step (compute_wavefield_1 and _2), the adjoint
sources add_sources_el_sim_type_2_or_3 and the replayed source
compute_add_sources_el_s3_cuda at it_tmp = NSTEP - it + 1
(compute_gpu_elastic.f90:283-311), transfer_b_fields_to_device after step 1
(read_forward_arrays.f90), compute_kernels_elastic_cuda every step, and
transfer_kernels_el_to_host at the end (iterate_time.F90:462-504).
"""
from __future__ import annotations

import ctypes

import numpy as np

from specfem2d_b200.setup.fortran_host import gpu_arrays


def _lib():
    from specfem2d_b200.runtime import load_library

    return load_library()


class _Refs:
    """Keeps the by-reference scalars and arrays of the calls alive."""

    def __init__(self):
        self.keep = []

    def i(self, v):
        x = ctypes.c_int(int(v))
        self.keep.append(x)
        return ctypes.byref(x)

    def f(self, v):
        x = ctypes.c_float(float(v))
        self.keep.append(x)
        return ctypes.byref(x)

    def a(self, arr):
        self.keep.append(arr)
        return arr.ctypes.data_as(ctypes.c_void_p)


def run_forward(db, nstep=None, check_every=1000, nlength_seismogram=None, save_forward=False):
    """Returns (seismograms (nrec, nstep, 2) float64, final displacement (nglob, 2), norms);
    with fluid elements the norms are (solid, fluid) pairs and the final potential
    follows as a fourth value."""
    return _drive(db, nstep, check_every, nlength_seismogram, None, save_forward)


def run_kernel(db, adj_src, check_every=1000, nlength_seismogram=None):
    """Kernel run with adjoint sources adj_src (nrec, nstep, 2) in forward time
    order (a fluid receiver's in component 0).  Returns (adjoint seismograms,
    final adjoint displacement, norms, kernels): the norms are (forward/adjoint,
    backward) pairs, one per domain (solid first); the kernels (nspec, 5, 5) are
    the solid sums rho, mu, kappa as transfer_kernels_el_to_host gives them, the
    fluid rho_ac, kappa_ac of transfer_kernels_ac_to_host and, with fluid
    elements, the final adjoint potential "pot"."""
    return _drive(db, None, check_every, nlength_seismogram, np.asarray(adj_src, np.float32), False)


def _drive(db, nstep, check_every, nlength_seismogram, adj_src, save_forward):
    lib = _lib()
    kernel = adj_src is not None
    A = gpu_arrays(db, nlength_seismogram)
    nstep = int(nstep or A["nstep"])
    nlen = A["nlength_seismogram"]
    r = _Refs()
    mesh = ctypes.c_long(0)
    M = ctypes.byref(mesh)
    ndev = ctypes.c_int(0)
    lib.initialize_cuda_device_(r.i(0), ctypes.byref(ndev))
    dummy_i = np.zeros(1, np.int32)
    dummy_f = np.zeros(1, np.float32)
    fluid = "ispec_is_acoustic" in A
    nac = A["nspec_acoustic"] if fluid else 0
    is_ac = A["ispec_is_acoustic"] if fluid else np.zeros(A["nspec"], np.int32)
    elastic = nac < A["nspec"]
    lib.prepare_constants_device_(
        M, r.i(5), r.i(A["nspec"]), r.i(A["nglob"]),
        r.a(A["xix"]), r.a(A["xiz"]), r.a(A["gammax"]), r.a(A["gammaz"]),
        r.a(A["kappastore"]), r.a(A["mustore"]), r.a(A["ibool"]),
        r.i(0), r.i(0), r.a(dummy_i), r.a(dummy_i),
        r.a(A["hprime_xx"]), r.a(A["hprimewgll_xx"]), r.a(A["wxgll"]),
        r.i(1 if A["stacey"] else 0), r.i(1 if "pml" in A else 0), r.a(np.ones(A["nspec"], np.int32)),
        r.i(A["nsrc"]), r.a(A["sourcearrays"]), r.a(A["source_time_function"]),
        r.i(A["nstep"]), r.a(A["ispec_selected_source"]), r.a(A["ispec_selected_rec_loc"]),
        r.i(A["nrec"]), r.a(A["cosrot"]), r.a(A["sinrot"]),
        r.i(3 if kernel else 1), r.i(1), r.i(nac), r.i(A["nspec"] - nac),
        r.a(is_ac), r.a((1 - is_ac).astype(np.int32)),
        r.i(0), r.i(int(save_forward)),
        r.a(A["xir_store"]), r.a(A["gammar_store"]),
        r.i(1), r.a(np.array([A["seismotype"]], np.int32)), r.i(nlen))
    if fluid:
        lib.prepare_fields_acoustic_device_(
            M, r.a(A["rmass_acoustic"]), r.a(A["rhostore"]), r.a(A["kappastore"]),
            r.i(nac), r.a(np.concatenate([np.zeros(nac, np.int32), np.flatnonzero(is_ac).astype(np.int32) + 1])),
            r.i(A["nfree"]), r.a(A["free_ac_ispec"]), r.a(A["free_surface_ij"]),
            r.i(int(elastic)), r.i(A["ncoupling"]), r.a(A["coupling_ac_el_ispec"]), r.a(A["coupling_ac_el_ij"]),
            r.a(A["coupling_ac_el_normal"]), r.a(A["coupling_ac_el_jacobian1Dw"]),
            r.i(0), r.a(dummy_i), r.i(0), r.a(dummy_f), r.a(dummy_f), r.i(0), r.a(dummy_f))
        if kernel:
            lib.prepare_fields_acoustic_adj_dev_(M, r.i(0), r.i(0), r.i(0))
    aniso = "ispec_is_anisotropic" in A
    atten = "att_a1" in A
    c = {k: (A[k + "store"] if aniso else dummy_f) for k in ("c11", "c13", "c15", "c33", "c35", "c55")}
    att = {k: (A["att_" + k] if atten else dummy_f) for k in ("a1", "b1", "a2", "b2")}
    prepare_el = lib.prepare_fields_elastic_device_ if elastic else (lambda *a: None)
    prepare_el(
        M, r.a(A["rmassx"]), r.a(A["rmassz"]), r.i(A["nspec"]), r.a(np.arange(1, A["nspec"] + 1, dtype=np.int32)),
        r.a(A["ispec_is_anisotropic"] if aniso else dummy_i), r.i(1 if aniso else 0),
        r.a(c["c11"]), r.a(dummy_f), r.a(c["c13"]), r.a(c["c15"]), r.a(dummy_f), r.a(dummy_f),
        r.a(c["c33"]), r.a(c["c35"]), r.a(c["c55"]),
        r.i(0), r.a(dummy_i), r.i(1 if atten else 0),
        r.a(att["a2"]), r.a(att["b2"]), r.a(att["a1"]), r.a(att["b1"]))
    if "pml" in A:
        # prepare_PML_device (prepare_gpu.f90:213-227)
        P = A["pml"]
        lib.prepare_pml_device_(
            M, r.i(P["nspec_pml"]), r.i(P["nspec_pml_x"]), r.i(P["nspec_pml_z"]), r.i(P["nspec_pml_xz"]),
            r.a(P["spec_to_pml"]), r.a(P["abs_normalized"]), r.f(P["alpha_max"]), r.f(P["d0_max"]),
            r.f(A["deltat"]), r.a(P["alphax"]), r.a(P["alphaz"]), r.a(P["betax"]), r.a(P["betaz"]),
            r.i(len(P["abs_points_acoustic"])), r.a(P["abs_points_acoustic"]))
    ng2 = 2 * A["nglob"]
    if kernel and elastic:
        lib.prepare_fields_elastic_adj_dev_(M, r.i(ng2), r.i(0), r.i(int(atten)), r.i(0))
    if A["stacey"]:
        ab = A["abs"]
        lib.prepare_stacey_device_(
            M, r.i(int(fluid)), r.i(int(elastic)), r.a(A["rho_vpstore"]), r.a(A["rho_vsstore"]),
            r.i(ab["counts"]["bottom"]), r.i(ab["counts"]["left"]), r.i(ab["counts"]["right"]),
            r.i(ab["counts"]["top"]), r.a(ab["abs_boundary_ispec"]), r.a(ab["abs_boundary_ij"]),
            r.a(ab["abs_boundary_normal"]), r.a(ab["abs_boundary_jacobian1Dw"]), r.i(ab["nface"]),
            r.a(ab["edge_abs"]), r.a(dummy_i), r.a(dummy_i), r.a(dummy_i), r.a(dummy_i))
    if kernel:
        # source_adjoint(nadj_rec_local, NSTEP, NDIM) in Fortran order
        src_adj = np.asfortranarray(adj_src.reshape(A["nrec"], A["nstep"], 2))
        lib.prepare_sim2_or_3_const_device_(M, r.i(A["nrec"]), r.a(src_adj), r.i(A["nstep"]))
    zeros = np.zeros(ng2, np.float32)
    if elastic:
        lib.transfer_fields_el_to_device_(r.i(ng2), r.a(zeros), r.a(zeros.copy()), r.a(zeros.copy()), M)
    if kernel:
        lib.transfer_b_fields_to_device_(r.i(ng2), r.a(zeros), r.a(zeros), r.a(zeros), M)
    if fluid:
        z1 = np.zeros(A["nglob"], np.float32)
        lib.transfer_fields_ac_to_device_(r.i(A["nglob"]), r.a(z1), r.a(z1.copy()), r.a(z1.copy()), M)
    sisux = np.zeros((A["nrec"], nlen), np.float64)
    sisuz = np.zeros_like(sisux)
    seis = np.zeros((A["nrec"], nstep, 2))
    dt, dt2, dtsq2 = ctypes.c_float(A["deltat"]), ctypes.c_float(A["deltatover2"]), ctypes.c_float(A["deltatsquareover2"])
    one, two, zero = ctypes.c_int(1), ctypes.c_int(2), ctypes.c_int(0)
    nspec_c, aniso_c, atten_c = ctypes.c_int(A["nspec"]), ctypes.c_int(int(aniso)), ctypes.c_int(int(atten))
    it_c, cur_c, nlen_c, end_c = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(nlen), ctypes.c_int(nstep)
    stype = ctypes.c_int(A["seismotype"])
    norm = ctypes.c_float(0.0)
    norms = []
    dummy_b = dummy_f.ctypes.data_as(ctypes.c_void_p)
    seismo_current = 0
    ncpl_c = ctypes.c_int(A.get("ncoupling", 0))
    # b_absorb_elastic_* slices (NDIM, NGLLX, nspec_side) and b_absorb_acoustic_* (NGLLX, nspec_side)
    sides = ("left", "right", "top", "bottom")
    nside = {k: (A["abs"]["counts"][k] if A["stacey"] else 0) for k in sides}
    b_el = [np.full(2 * 5 * max(nside[k], 1), np.nan, np.float32) for k in sides]
    b_ac = [np.full(5 * max(nside[k], 1), np.nan, np.float32) for k in sides]
    p_el = [b.ctypes.data_as(ctypes.c_void_p) for b in b_el]
    p_ac = [b.ctypes.data_as(ctypes.c_void_p) for b in b_ac]
    nrec_c, nstep_c, itmp_c = ctypes.c_int(A["nrec"]), ctypes.c_int(A["nstep"]), ctypes.c_int(0)
    three = ctypes.c_int(3)
    trick_c = ctypes.c_int(A.get("use_trick", 0))

    def saved_slices_are_zero(slices):
        # SAVE_FORWARD: the host stores the slices it got back as b_absorb_*(..., it)
        assert all(np.all(b == 0) for b, k in zip(slices, sides) if nside[k] > 0)

    def acoustic_phase(w1, w2):
        """compute_forces_viscoacoustic_GPU (compute_gpu_acoustic.f90:36-220)."""
        c1, c2 = (one if w1 else zero), (one if w2 else zero)
        if A["nfree"] > 0:
            lib.acoustic_enforce_free_surf_cuda_(M, ctypes.byref(c1), ctypes.byref(c2))
        for iphase in (one, two):
            lib.compute_forces_acoustic_cuda_(M, ctypes.byref(iphase), ctypes.byref(zero), ctypes.byref(zero),
                                              ctypes.byref(zero), ctypes.byref(c1), ctypes.byref(c2))
            if "pml" in A:
                lib.pml_boundary_acoustic_cuda_(M, ctypes.byref(c1), ctypes.byref(c2))
            if iphase is not one:
                continue
            if A["stacey"]:
                lib.compute_stacey_acoustic_cuda_(M, ctypes.byref(one), *p_ac, ctypes.byref(c1), ctypes.byref(c2),
                                                  ctypes.byref(zero))
                if save_forward:
                    saved_slices_are_zero(b_ac)
            if elastic:
                for w, kind in ((w1, one), (w2, three)):
                    if w:
                        lib.compute_coupling_ac_el_cuda_(M, ctypes.byref(one), ctypes.byref(ncpl_c), ctypes.byref(kind))
            if not kernel:
                lib.compute_add_sources_ac_cuda_(M, ctypes.byref(one), ctypes.byref(it_c))
            else:
                if A["nrec"] > 0 and w1:
                    lib.add_sources_ac_sim_2_or_3_cuda_(M, ctypes.byref(one), ctypes.byref(itmp_c),
                                                        ctypes.byref(nrec_c), ctypes.byref(nstep_c))
                if w2:
                    lib.compute_add_sources_ac_s3_cuda_(M, ctypes.byref(one), ctypes.byref(itmp_c))
        lib.kernel_3_acoustic_cuda_(M, ctypes.byref(dt2), ctypes.byref(dt2), ctypes.byref(c1), ctypes.byref(c2))
        lib.acoustic_enforce_free_surf_cuda_(M, ctypes.byref(c1), ctypes.byref(c2))

    def elastic_phase(w1, w2):
        """compute_forces_viscoelastic_GPU (compute_gpu_elastic.f90:36-215)."""
        c1, c2 = (one if w1 else zero), (one if w2 else zero)
        for iphase in (one, two):
            lib.compute_forces_viscoelastic_cuda_(M, ctypes.byref(iphase), ctypes.byref(dt), ctypes.byref(zero),
                                                  ctypes.byref(nspec_c), ctypes.byref(aniso_c), ctypes.byref(atten_c),
                                                  ctypes.byref(c1), ctypes.byref(c2))
            if iphase is not one:
                continue
            if A["stacey"]:
                lib.compute_stacey_viscoelastic_cuda_(M, ctypes.byref(one), *p_el, ctypes.byref(c1),
                                                      ctypes.byref(c2), ctypes.byref(zero))
                if save_forward:
                    saved_slices_are_zero(b_el)
            if fluid:
                for w, kind in ((w1, one), (w2, three)):
                    if w:
                        lib.compute_coupling_el_ac_cuda_(M, ctypes.byref(one), ctypes.byref(ncpl_c), ctypes.byref(kind))
            if not kernel:
                lib.compute_add_sources_el_cuda_(M, ctypes.byref(one), ctypes.byref(it_c))
            else:
                if A["nrec"] > 0 and w1:
                    lib.add_sources_el_sim_type_2_or_3_(M, ctypes.byref(one), ctypes.byref(itmp_c),
                                                        ctypes.byref(nrec_c), ctypes.byref(nstep_c))
                if w2:
                    lib.compute_add_sources_el_s3_cuda_(M, ctypes.byref(one), ctypes.byref(itmp_c))
        lib.kernel_3_a_cuda_(M, ctypes.byref(dt2), ctypes.byref(dt2), ctypes.byref(c1), ctypes.byref(c2))

    for it in range(1, nstep + 1):
        it_c.value = it
        itmp_c.value = A["nstep"] - it + 1
        if fluid:
            lib.update_displacement_ac_cuda_(M, ctypes.byref(dt), ctypes.byref(dtsq2), ctypes.byref(dt2),
                                             ctypes.byref(dt), ctypes.byref(dtsq2), ctypes.byref(dt2),
                                             ctypes.byref(one), ctypes.byref(zero))
        if elastic:
            lib.update_displacement_cuda_(M, ctypes.byref(dt), ctypes.byref(dtsq2), ctypes.byref(dt2),
                                          ctypes.byref(dt), ctypes.byref(dtsq2), ctypes.byref(dt2))
        if not kernel:
            # forward: fluid then solid (iterate_time.F90:262-285)
            if fluid:
                acoustic_phase(True, False)
            if elastic:
                elastic_phase(True, False)
        elif fluid and elastic:
            # kernel run of a coupled mesh: solid then fluid for the adjoint field,
            # fluid then solid for the replayed one (iterate_time.F90:298-360)
            elastic_phase(True, False)
            acoustic_phase(True, False)
            acoustic_phase(False, True)
            elastic_phase(False, True)
        elif fluid:
            acoustic_phase(True, True)
        else:
            elastic_phase(True, True)
        if kernel and it == 1:
            # read_forward_arrays: the last frame of the saved forward run
            if fluid:
                z1 = np.zeros(A["nglob"], np.float32)
                lib.transfer_b_fields_ac_to_device_(r.i(A["nglob"]), r.a(z1), r.a(z1), r.a(z1), M)
            if elastic:
                lib.transfer_b_fields_to_device_(r.i(ng2), r.a(zeros), r.a(zeros), r.a(zeros), M)
        seismo_current += 1
        cur_c.value = seismo_current
        lib.compute_seismograms_cuda_(M, ctypes.byref(one), sisux.ctypes.data_as(ctypes.c_void_p),
                                      sisuz.ctypes.data_as(ctypes.c_void_p), ctypes.byref(cur_c),
                                      ctypes.byref(nlen_c), ctypes.byref(one), ctypes.byref(zero),
                                      ctypes.byref(trick_c), ctypes.byref(atten_c), ctypes.byref(it_c),
                                      ctypes.byref(end_c))
        if seismo_current == nlen or it == nstep:
            # write_seismograms saves the buffer and starts it again
            n = seismo_current
            seis[:, it - n:it, 0] = sisux[:, :n]
            seis[:, it - n:it, 1] = sisuz[:, :n]
            seismo_current = 0
        if kernel:
            # compute_kernels (compute_kernels.f90:35-70): fluid, then solid
            if fluid:
                lib.compute_kernels_acoustic_cuda_(M, ctypes.byref(dt))
            if elastic:
                lib.compute_kernels_elastic_cuda_(M, ctypes.byref(dt))
        if kernel and (it % check_every == 0 or it == nstep):
            # (forward/adjoint, backward) norm pairs: solid, then fluid
            entry = []
            for fn, present in ((lib.get_norm_elastic_from_device_, elastic), (lib.get_norm_acoustic_from_device_, fluid)):
                if present:
                    fn(ctypes.byref(norm), M, ctypes.byref(one))
                    f_norm = float(norm.value)
                    fn(ctypes.byref(norm), M, ctypes.byref(three))
                    entry.append((f_norm, float(norm.value)))
            norms.append(entry[0] if len(entry) == 1 else tuple(entry))
        elif it % check_every == 0 or it == nstep:
            lib.get_norm_elastic_from_device_(ctypes.byref(norm), M, ctypes.byref(one))
            if fluid:
                n_el = float(norm.value)
                lib.get_norm_acoustic_from_device_(ctypes.byref(norm), M, ctypes.byref(one))
                norms.append((n_el, float(norm.value)))
            else:
                norms.append(float(norm.value))
    displ = np.zeros(ng2, np.float32)
    if elastic:
        lib.transfer_displ_from_device_(r.i(ng2), r.a(displ), M)
    pot = None
    if fluid:
        pot = np.zeros(A["nglob"], np.float32)
        lib.transfer_fields_ac_from_device_(r.i(A["nglob"]), r.a(pot), r.a(np.zeros_like(pot)), r.a(np.zeros_like(pot)), M)
    kl = None
    if kernel:
        # it_transfer_from_GPU (iterate_time.F90:462-504)
        kl = {k: np.zeros((A["nspec"], 5, 5), np.float32) for k in ("rho", "mu", "kappa", "rho_ac", "kappa_ac")}
        if fluid:
            lib.transfer_kernels_ac_to_host_(M, r.a(kl["rho_ac"]), r.a(kl["kappa_ac"]), r.i(A["nspec"]))
        if elastic:
            lib.transfer_kernels_el_to_host_(M, r.a(kl["rho"]), r.a(kl["mu"]), r.a(kl["kappa"]), r.i(A["nspec"]))
        if fluid:
            kl["pot"] = pot
    lib.prepare_cleanup_device_(M, r.i(0), r.i(1), r.i(int(aniso)), r.i(0), r.i(0), r.i(int(atten)), r.i(0),
                                r.a(dummy_f))
    if kernel:
        return seis, displ.reshape(-1, 2), norms, kl
    if fluid:
        return seis, displ.reshape(-1, 2), norms, pot
    return seis, displ.reshape(-1, 2), norms
