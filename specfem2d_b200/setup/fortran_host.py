"""The arrays the reference's Fortran host hands its GPU library, in Fortran
memory order, for driving include/sf2d_fortran.h the way SPECFEM2D does.

Restates what src/specfem2D/prepare_gpu.f90 passes to prepare_constants_device,
prepare_fields_acoustic_device, prepare_fields_elastic_device and
prepare_Stacey_device (init_host_to_dev_variable, :346-640: local sources and
their time functions, receiver rotations as CUSTOM_REAL, the free-surface faces
and the fluid-solid faces with the fluid element's normals and jacobian1D * w)
and the absorbing-face arrays of prepare_timerun.F90:1270-1440
(abs_boundary_ij with NGLLX + 1 marking a corner point that the neighbouring
face covers, outward normals, jacobian1D * w, edge_abs = 1 bottom, 2 right,
3 top, 4 left).  Every array is a C-contiguous numpy array whose memory
matches the Fortran array (the first index varies fastest); indices are
1-based.
"""
from __future__ import annotations

import numpy as np

from . import acoustic as ac_setup
from .gll import NGLL
from .mesh import IBOTTOM, ILEFT, IRIGHT, ITOP
from .solver_setup import edge_normal

f32 = np.float32


def _fortran(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def abs_boundary_arrays(db):
    """abs_boundary_ispec, abs_boundary_ij (2, NGLLX, nface), abs_boundary_normal
    (2, NGLLX, nface), abs_boundary_jacobian1Dw (NGLLX, nface), edge_abs and the
    per-side face counts, for the absorbing faces of db.mesh.  On a fluid face
    every point the fluid Stacey loop skips (ibegin/iend_edge: corners and
    points shared with a fluid-solid edge) is marked NGLLX + 1
    (prepare_timerun.F90:1330-1420)."""
    mesh = db.mesh
    geo = dict(xix=db.xix, xiz=db.xiz, gammax=db.gammax, gammaz=db.gammaz, jacobian=db.jacobian)
    nf = 0 if mesh.abs_ispec is None else len(mesh.abs_ispec)
    ispec = np.zeros(nf, np.int32)
    ij = np.zeros((nf, NGLL, 2), np.int32)
    normal = np.zeros((nf, NGLL, 2), f32)
    jw = np.zeros((nf, NGLL), f32)
    edge = np.zeros(nf, np.int32)
    for k in range(nf):
        e, t = int(mesh.abs_ispec[k]), int(mesh.abs_type[k])
        ispec[k] = e + 1
        edge[k] = t
        for p in range(NGLL):
            i, j = {ILEFT: (0, p), IRIGHT: (NGLL - 1, p), IBOTTOM: (p, 0), ITOP: (p, NGLL - 1)}[t]
            ij[k, p] = (i + 1, j + 1)
            normal[k, p, 0], normal[k, p, 1], jw[k, p] = edge_normal(geo, db.gll, e, i, j, t)
        c = mesh.abs_corner[k]
        if t == IBOTTOM:
            if c[0]:
                ij[k, 0, 0] = NGLL + 1
            if c[1]:
                ij[k, NGLL - 1, 0] = NGLL + 1
        elif t == ITOP:
            if c[2]:
                ij[k, 0, 0] = NGLL + 1
            if c[3]:
                ij[k, NGLL - 1, 0] = NGLL + 1
    if db.acoustic is not None and nf:
        is_ac = np.asarray(db.acoustic["ispec"], dtype=bool)
        cpl = ac_setup.coupling_edges(db.ibool, is_ac) if (~is_ac).any() else []
        for (k, e, t, pts) in ac_setup.absorbing_ranges(mesh, cpl):
            if not is_ac[e]:
                continue
            keep = set(pts)
            for p in range(NGLL):
                i, j = ij[k, p] - 1
                if (int(i), int(j)) not in keep and i < NGLL and j < NGLL:
                    ij[k, p, 1 if t in (ILEFT, IRIGHT) else 0] = NGLL + 1
    counts = {name: int(np.sum(edge == code)) for name, code in
              (("bottom", IBOTTOM), ("left", ILEFT), ("right", IRIGHT), ("top", ITOP))}
    return dict(abs_boundary_ispec=ispec, abs_boundary_ij=ij, abs_boundary_normal=normal,
                abs_boundary_jacobian1Dw=jw, edge_abs=edge, nface=nf, counts=counts)


def gpu_arrays(db, nlength_seismogram: int | None = None):
    """Arrays of prepare_constants_device / prepare_fields_elastic_device /
    prepare_Stacey_device for an elastic Newmark Database (one process, all
    sources and receivers local)."""
    nstep = int(db.nstep)
    nsrc, nrec = int(db.source_ispec.size), int(db.rec_ispec.size)
    out = dict(
        nspec=int(db.nspec), nglob=int(db.nglob), nstep=nstep, nsrc=nsrc, nrec=nrec,
        ibool=_fortran(db.ibool + 1, np.int32),
        xix=_fortran(db.xix, f32), xiz=_fortran(db.xiz, f32), gammax=_fortran(db.gammax, f32),
        gammaz=_fortran(db.gammaz, f32), kappastore=_fortran(db.kappastore, f32),
        mustore=_fortran(db.mustore, f32), rho_vpstore=_fortran(db.rho_vpstore, f32),
        rho_vsstore=_fortran(db.rho_vsstore, f32),
        # hprime_xx(i2, i1): the transpose of the C-order [i2][i1] table
        hprime_xx=_fortran(db.gll.hprime.T, f32), hprimewgll_xx=_fortran(db.gll.hprimewgll.T, f32),
        wxgll=_fortran(db.gll.wxgll, f32),
        # sourcearray_loc(NDIM, NGLLX, NGLLZ, nsrc) and source_time_function_loc(nsrc, NSTEP)
        sourcearrays=_fortran(db.sourcearrays, f32),
        source_time_function=_fortran(db.stf[:, :, 0].T, f32),
        ispec_selected_source=_fortran(db.source_ispec + 1, np.int32),
        ispec_selected_rec_loc=_fortran(db.rec_ispec + 1, np.int32),
        cosrot=np.full(nrec, f32(db.cosrot), f32), sinrot=np.full(nrec, f32(db.sinrot), f32),
        # xir_store_loc(nrec, NGLLX), gammar_store_loc(nrec, NGLLX)
        xir_store=_fortran(np.asarray(db.hxir).T, f32), gammar_store=_fortran(np.asarray(db.hgammar).T, f32),
        seismotype=int(db.seismotype),
        nlength_seismogram=int(nlength_seismogram or nstep),
        rmassx=_fortran(db.rmass_inverse_elastic[:, 0], f32),
        rmassz=_fortran(db.rmass_inverse_elastic[:, 1], f32),
        deltat=f32(db.deltat), deltatover2=f32(db.deltatover2), deltatsquareover2=f32(db.deltatsquareover2),
        stacey=bool(db.stacey_iglob.size > 0
                    or (db.acoustic is not None and len(db.acoustic["st_iglob"]) > 0)),
    )
    out["abs"] = abs_boundary_arrays(db)
    if db.acoustic is not None:
        out.update(fluid_arrays(db))
        # write_seismograms.F90 passes it to compute_seismograms_cuda
        out["use_trick"] = int(bool(db.acoustic.get("use_trick", False)))
    if db.aniso is not None:
        out["ispec_is_anisotropic"] = _fortran(db.aniso["ispec"], np.int32)
        for k in ("c11", "c13", "c15", "c33", "c35", "c55"):
            out[k + "store"] = _fortran(db.aniso[k], f32)
    if db.atten is not None:
        # A/B_newmark_nu1 (bulk) and _nu2 (shear), (N_SLS, NGLLX, NGLLZ, nspec)
        for k in ("a1", "b1", "a2", "b2"):
            out["att_" + k] = _fortran(db.atten[k], f32)
    if getattr(db, "pml", None) is not None:
        out["pml"] = pml_arrays(db)
    return out


def pml_arrays(db):
    """prepare_PML_device's arrays (prepare_gpu.f90:213-227, 389-470):
    spec_to_PML_GPU numbering the CPML_X_ONLY elements first, then CPML_Z_ONLY,
    then CPML_XZ (each in ascending element order, 0 outside the layer),
    abs_normalized (NGLLX, NGLLZ, NSPEC_PML) of the X and Z elements,
    ALPHA_MAX_PML and d0_max (the largest acoustic d0, pml_init.F90:884-887),
    alpha and beta = alpha + d of the XZ elements (NGLLX, NGLLZ, NSPEC_PML_XZ)
    and PML_abs_points_acoustic (the fluid points of the layer's outer edge)."""
    from . import pml as pml_setup

    pm = db.pml
    region = np.asarray(pm["region"])
    spec = np.zeros(db.nspec, np.int32)
    n = 0
    counts = []
    for code in (pml_setup.CPML_X_ONLY, pml_setup.CPML_Z_ONLY, pml_setup.CPML_XZ):
        els = np.flatnonzero(region == code)
        spec[els] = n + 1 + np.arange(els.size)
        n += els.size
        counts.append(int(els.size))
    nx, nz, nxz = counts
    absn = np.zeros((max(n, 1), NGLL, NGLL), f32)
    for e in np.flatnonzero(spec > 0):
        p = spec[e] - 1
        if region[e] == pml_setup.CPML_X_ONLY:
            absn[p] = pm["abs_x"][e]
        elif region[e] == pml_setup.CPML_Z_ONLY:
            absn[p] = pm["abs_z"][e]
    xz = np.flatnonzero(region == pml_setup.CPML_XZ)
    st = {k: np.zeros((max(nxz, 1), NGLL, NGLL), f32) for k in ("alphax", "alphaz", "betax", "betaz")}
    for k, e in enumerate(xz):
        st["alphax"][k] = pm["alpha_x"][e]
        st["alphaz"][k] = pm["alpha_z"][e]
        st["betax"][k] = pm["alpha_x"][e] + pm["d_x"][e]
        st["betaz"][k] = pm["alpha_z"][e] + pm["d_z"][e]
    return dict(nspec_pml=n, nspec_pml_x=nx, nspec_pml_z=nz, nspec_pml_xz=nxz, spec_to_pml=spec,
                abs_normalized=_fortran(absn, f32), alpha_max=f32(pm["alpha_max"]), d0_max=f32(pm["d0_max_acoustic"]),
                alphax=_fortran(st["alphax"], f32), alphaz=_fortran(st["alphaz"], f32),
                betax=_fortran(st["betax"], f32), betaz=_fortran(st["betaz"], f32),
                abs_points_acoustic=_fortran(np.asarray(pm["bnd_ac"]) + 1, np.int32))


def fluid_arrays(db):
    """prepare_fields_acoustic_device's arrays: ispec_is_acoustic, the fluid
    mass matrix, rhostore, the free-surface faces (free_ac_ispec and
    free_surface_ij (2, NGLLX, nface) as prepare_gpu.f90:549-580 spans each
    listed edge) and the fluid-solid faces (coupling_ac_el_ispec, _ij, _normal
    and _jacobian1Dw from the fluid element's edge, prepare_gpu.f90:586-640)."""
    is_ac = np.asarray(db.acoustic["ispec"], dtype=bool)
    mesh = db.mesh
    rows = mesh.free_edges if mesh.free_edges is not None else ac_setup.structured_free_edges(mesh, is_ac)
    rows = [r for r in rows if is_ac[r[0]]]
    free_ispec = np.array([r[0] + 1 for r in rows], np.int32)
    free_ij = np.zeros((len(rows), NGLL, 2), np.int32)
    for k, (e, i0, i1, j0, j1) in enumerate(rows):
        ii = [i0] * NGLL if i0 == i1 else list(range(i0, i1 + 1))
        jj = [j0] * NGLL if j0 == j1 else list(range(j0, j1 + 1))
        free_ij[k, :, 0] = np.array(ii) + 1
        free_ij[k, :, 1] = np.array(jj) + 1
    geo = dict(xix=db.xix, xiz=db.xiz, gammax=db.gammax, gammaz=db.gammaz, jacobian=db.jacobian)
    edges = ac_setup.coupling_edges(db.ibool, is_ac) if (~is_ac).any() else []
    n = len(edges)
    c_ispec = np.zeros(n, np.int32)
    c_ij = np.zeros((n, NGLL, 2), np.int32)
    c_normal = np.zeros((n, NGLL, 2), f32)
    c_jw = np.zeros((n, NGLL), f32)
    for k, (ea, edge_a, _, _) in enumerate(edges):
        c_ispec[k] = ea + 1
        for p in range(NGLL):
            i, j = ac_setup._ivalue(p, edge_a)
            c_ij[k, p] = (i + 1, j + 1)
            c_normal[k, p, 0], c_normal[k, p, 1], c_jw[k, p] = ac_setup._edge_normal(geo, ea, i, j, edge_a, db.gll)
    return dict(ispec_is_acoustic=_fortran(is_ac, np.int32), nspec_acoustic=int(is_ac.sum()),
                rmass_acoustic=_fortran(db.acoustic["rmass"], f32), rhostore=_fortran(db.rhostore, f32),
                free_ac_ispec=free_ispec, free_surface_ij=free_ij, nfree=len(rows),
                coupling_ac_el_ispec=c_ispec, coupling_ac_el_ij=c_ij, coupling_ac_el_normal=c_normal,
                coupling_ac_el_jacobian1Dw=c_jw, ncoupling=n)
