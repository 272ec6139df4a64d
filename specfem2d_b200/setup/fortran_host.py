"""The arrays the reference's Fortran host hands its GPU library, in Fortran
memory order, for driving include/sf2d_fortran.h the way SPECFEM2D does.

Restates what src/specfem2D/prepare_gpu.f90 passes to prepare_constants_device,
prepare_fields_elastic_device and prepare_Stacey_device (init_host_to_dev_variable,
:346-470: local sources and their time functions, receiver rotations as
CUSTOM_REAL) and the absorbing-face arrays of prepare_timerun.F90:1270-1440
(abs_boundary_ij with NGLLX + 1 marking a corner point that the neighbouring
face covers, outward normals, jacobian1D * w, edge_abs = 1 bottom, 2 right,
3 top, 4 left).  Every array is a C-contiguous numpy array whose memory
matches the Fortran array (the first index varies fastest); indices are
1-based.
"""
from __future__ import annotations

import numpy as np

from .gll import NGLL
from .mesh import IBOTTOM, ILEFT, IRIGHT, ITOP
from .solver_setup import edge_normal

f32 = np.float32


def _fortran(a, dtype):
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def abs_boundary_arrays(db):
    """abs_boundary_ispec, abs_boundary_ij (2, NGLLX, nface), abs_boundary_normal
    (2, NGLLX, nface), abs_boundary_jacobian1Dw (NGLLX, nface), edge_abs and the
    per-side face counts, for the absorbing faces of db.mesh."""
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
        stacey=bool(db.stacey_iglob.size > 0),
    )
    out["abs"] = abs_boundary_arrays(db)
    if db.aniso is not None:
        out["ispec_is_anisotropic"] = _fortran(db.aniso["ispec"], np.int32)
        for k in ("c11", "c13", "c15", "c33", "c35", "c55"):
            out[k + "store"] = _fortran(db.aniso[k], f32)
    if db.atten is not None:
        # A/B_newmark_nu1 (bulk) and _nu2 (shear), (N_SLS, NGLLX, NGLLZ, nspec)
        for k in ("a1", "b1", "a2", "b2"):
            out["att_" + k] = _fortran(db.atten[k], f32)
    return out
