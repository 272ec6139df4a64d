"""Build a setup Database from a reference-style DATA/ directory.

Supports the internal-mesher subset used by the hot path: interfaces file,
isotropic material table with regions, Stacey, CPML or free edges, force or
moment-tensor sources or an analytical initial field, a receiver line
(src/meshfem2D/save_stations_file.f90: receivers evenly spaced between
(xdeb,zdeb) and (xfin,zfin), written with 7 decimals), Newmark or LDDRK.
"""
from __future__ import annotations

import os

import numpy as np

from .gll import NGLL
from .mesh import internal_mesh, read_interfaces_file, spline_construction, value_spline
from .parfile import material_from_row, read_par_file, read_source_file
from .solver_setup import Source, build_database


def _receivers_from_par(par, top_interface):
    """Receiver lines of all receiver sets, in set order."""
    sets = par.get("receiver_sets") or [par]
    if top_interface is None:
        if any(rs.get("record_at_surface_same_vertical", False) for rs in sets):
            raise NotImplementedError("receivers moved to the surface of an external mesh")
        top_interface = ([0.0, 1.0], [0.0, 0.0])
    xs_t, zs_t = top_interface
    t1 = (zs_t[1] - zs_t[0]) / (xs_t[1] - xs_t[0])
    tn = (zs_t[-1] - zs_t[-2]) / (xs_t[-1] - xs_t[-2])
    coefs = spline_construction(xs_t, zs_t, t1, tn)
    out = []
    for rs in sets:
        nrec = int(rs["nrec"])
        xdeb, zdeb = float(rs["xdeb"]), float(rs["zdeb"])
        xfin, zfin = float(rs["xfin"]), float(rs["zfin"])
        for irec in range(1, nrec + 1):
            if nrec > 1:
                xr = xdeb + float(irec - 1) * (xfin - xdeb) / float(nrec - 1)
                zr = zdeb + float(irec - 1) * (zfin - zdeb) / float(nrec - 1)
            else:
                xr, zr = xdeb, zdeb
            if rs.get("record_at_surface_same_vertical", False):
                zr = value_spline(xr, xs_t, zs_t, coefs)
            out.append((round(xr, 7), round(zr, 7)))
    return out


PAR_KEYS = ("NSTEP", "DT", "time_stepping_scheme", "NGNOD", "xmin", "xmax", "nx", "absorbbottom",
            "absorbright", "absorbtop", "absorbleft", "STACEY_ABSORBING_CONDITIONS", "USER_T0",
            "anglerec", "nrec", "xdeb", "zdeb", "xfin", "zfin", "record_at_surface_same_vertical",
            "seismotype", "materials", "regions", "ATTENUATION_VISCOELASTIC", "PML_BOUNDARY_CONDITIONS",
            "ATTENUATION_f0_REFERENCE", "NELEM_PML_THICKNESS", "receiver_sets", "USE_TRICK_FOR_BETTER_PRESSURE",
            "TOMOGRAPHY_FILE", "MODEL", "K_MIN_PML", "K_MAX_PML", "damping_change_factor_acoustic",
            "damping_change_factor_elastic", "ROTATE_PML_ACTIVATE", "PML_PARAMETER_ADJUSTMENT",
            "initialfield", "read_external_mesh")

# Par_file keys of the external-mesh text files and the tables they fill
EXTERNAL_MESH_FILES = (("mesh_file", "elements"), ("nodes_coords_file", "nodes"), ("materials_file", "materials"),
                       ("free_surface_file", "free_surface"), ("absorbing_surface_file", "absorbing"))


def config_from_data_dir(data_dir: str, par_file: str = "Par_file", source_file: str = "SOURCE") -> dict:
    """Parse Par_file, SOURCE and the interfaces file of a DATA/ directory into a plain dict."""
    par = read_par_file(os.path.join(data_dir, par_file))
    srcs = read_source_file(os.path.join(data_dir, source_file))
    cfg = {k: par[k] for k in PAR_KEYS if k in par}
    cfg["sources"] = srcs
    if par.get("read_external_mesh", False):
        from .external_mesh import read_external_mesh_files

        # the file names are relative to the directory the programs run in, DATA/'s parent
        run_dir = os.path.dirname(os.path.abspath(data_dir))

        def path(key):
            v = str(par.get(key, "dummy")).strip()
            if not v or v == "dummy":
                return None
            return os.path.join(run_dir, v)

        stacey = bool(par["STACEY_ABSORBING_CONDITIONS"])
        pml = bool(par.get("PML_BOUNDARY_CONDITIONS", False))
        cfg["external_mesh"] = read_external_mesh_files(
            path("mesh_file"), path("nodes_coords_file"), path("materials_file"), int(par["NGNOD"]),
            free_surface_file=path("free_surface_file"),
            absorbing_file=path("absorbing_surface_file") if (stacey or pml) else None)
        return cfg
    ifile = str(par["interfacesfile"]).strip()
    cand = [os.path.join(data_dir, ifile), os.path.join(data_dir, os.path.basename(ifile))]
    ipath = next(p for p in cand if os.path.exists(p))
    interfaces, nz_layer = read_interfaces_file(ipath)
    cfg["interfaces"] = [[list(x), list(z)] for (x, z) in interfaces]
    cfg["nz_layer"] = list(nz_layer)
    return cfg


def config_from_mesh_database(data_dir: str, database: str, par_file: str = "Par_file",
                              source_file: str = "SOURCE") -> dict:
    """The run's parameters from DATA/ (Par_file, SOURCE: the solver reads them
    itself) and its mesh and materials from the mesher's database file
    (OUTPUT_FILES/Database00000.bin), as xspecfem2D takes them."""
    from .database_file import read_database

    par = read_par_file(os.path.join(data_dir, par_file))
    cfg = {k: par[k] for k in PAR_KEYS if k in par}
    cfg["sources"] = read_source_file(os.path.join(data_dir, source_file))
    cfg["mesh_database"] = read_database(database)
    return cfg


def database_from_data_dir(data_dir: str, nstep: int | None = None):
    """Return (Database, config dict) for the example whose DATA/ is ``data_dir``."""
    cfg = config_from_data_dir(data_dir)
    return database_from_config(cfg, nstep), cfg


def database_from_config(cfg: dict, nstep: int | None = None, absorbing_as_stacey: bool = False,
                         time_scheme: int | None = None, tomo=None):
    """Build the Database from a parsed example configuration.

    ``absorbing_as_stacey`` puts Stacey conditions on the absorbing edges of
    an example that uses CPML (for comparisons on a time window that ends
    before boundary reflections reach the receivers).  ``tomo`` = (x, z, vp,
    vs, rho) of the TOMOGRAPHY_FILE grid when the material table holds a
    tomographic material (type -1); the whole model then takes the external
    route (define_external_model_from_tomo_file.f90:386-470)."""
    par = cfg
    srcs = cfg["sources"]
    interfaces = [(list(x), list(z)) for (x, z) in cfg.get("interfaces", [])]
    nz_layer = list(cfg.get("nz_layer", []))
    absorb = (bool(par["absorbbottom"]), bool(par["absorbright"]), bool(par["absorbtop"]),
              bool(par["absorbleft"]))
    if not (bool(par["STACEY_ABSORBING_CONDITIONS"]) or bool(par.get("PML_BOUNDARY_CONDITIONS", False))):
        # without Stacey or CPML no edge absorbs: every edge is a free surface
        # (read_parameter_file.F90:1678-1687, read_parameter_file_derive_flags)
        absorb = (False, False, False, False)
    mats = {m["index"]: m for m in (material_from_row(r) for r in par["materials"])}
    if cfg.get("mesh_database") is not None:
        from .database_file import material_rows, mesh_from_database

        # the mesher's database holds the mesh and the material table (read_mesh_databases.F90)
        dbf = cfg["mesh_database"]
        if np.any(dbf["pml"]):
            raise NotImplementedError("CPML flags of a mesh database")
        mats = {m["index"]: m for m in (material_from_row(r) for r in material_rows(dbf))}
        fluid = [k for k, m in mats.items() if m["kind"] == 1 and abs(float(m["vs"])) <= 1e-9]
        mesh = mesh_from_database(dbf, fluid)
        mat_of = np.asarray(dbf["kmato"], dtype=np.int64).copy()
    elif par.get("read_external_mesh", False):
        from .external_mesh import external_mesh

        if bool(par.get("PML_BOUNDARY_CONDITIONS", False)) and not absorbing_as_stacey:
            raise NotImplementedError("CPML layers of an external mesh (absorbing_cpml_file)")

        # free-surface lines are kept on isotropic fluid materials, |vs| <= TINYVAL
        # (read_material_table.f90:179-183, read_external_mesh_files.F90:398-420)
        fluid = [k for k, m in mats.items() if m["kind"] == 1 and abs(float(m["vs"])) <= 1e-9]
        mesh = external_mesh(cfg["external_mesh"], int(par["NGNOD"]), fluid)
        mat_of = np.asarray(cfg["external_mesh"]["materials"], dtype=np.int64).copy()
    else:
        mesh = internal_mesh(float(par["xmin"]), float(par["xmax"]), int(par["nx"]), interfaces, nz_layer,
                             absorb=absorb, ngnod=int(par["NGNOD"]))
        # later regions overwrite earlier ones, in the order of the table
        mat_of = np.zeros(mesh.nspec, dtype=np.int64)
        for (ix0, ix1, iz0, iz1, imat) in par["regions"]:
            for iz in range(iz0, iz1 + 1):
                mat_of[(iz - 1) * mesh.nx + ix0 - 1:(iz - 1) * mesh.nx + ix1] = imat
    missing = sorted(set(int(k) for k in np.unique(mat_of)) - set(mats))
    if missing:
        raise ValueError(f"elements use materials {missing} that the material table does not define")
    rho = np.zeros((mesh.nspec, NGLL, NGLL))
    vp = np.zeros_like(rho)
    vs = np.zeros_like(rho)
    qk = np.full_like(rho, 9999.0)
    qm = np.full_like(rho, 9999.0)
    ckeys = ("c11", "c13", "c15", "c33", "c35", "c55")
    cstore = {k: np.zeros_like(rho) for k in ckeys}
    is_aniso = np.zeros(mesh.nspec, dtype=bool)
    for imat, m in mats.items():
        sel = mat_of == imat
        if not sel.any():
            continue
        rho[sel], vp[sel], vs[sel] = m["rho"], m["vp"], m["vs"]
        qk[sel], qm[sel] = m["qkappa"], m["qmu"]
        if m["kind"] == 2:
            is_aniso[sel] = True
            for k in ckeys:
                cstore[k][sel] = m[k]
    tomo_mats = [k for k, m in mats.items() if m["kind"] == -1]
    external = False
    if tomo_mats:
        if tomo is None:
            raise ValueError("the material table has a tomographic material: pass tomo=(x, z, vp, vs, rho)")
        from .tomography import tomo_values

        # table materials enter the external arrays as rho, sqrt((lambda+2mu)/rho), sqrt(mu/rho)
        for m in mats.values():
            if m["kind"] == -1:
                continue
            lp2m = m["rho"] * m["vp"] * m["vp"]
            mu = m["rho"] * m["vs"] * m["vs"]
            m["vp"], m["vs"] = float(np.sqrt(lp2m / m["rho"])), float(np.sqrt(mu / m["rho"]))
        for imat, m in mats.items():
            sel = mat_of == imat
            vp[sel], vs[sel] = m["vp"], m["vs"]
        external = True
    atten = bool(par.get("ATTENUATION_VISCOELASTIC", False))
    sources = []
    for s in srcs:
        sources.append(Source(x=float(s["xs"]), z=float(s["zs"]), source_type=int(s["source_type"]),
                              time_function_type=int(s["time_function_type"]), f0=float(s["f0"]),
                              tshift=float(s["tshift"]), anglesource_deg=float(s["anglesource"]),
                              Mxx=float(s["Mxx"]), Mzz=float(s["Mzz"]), Mxz=float(s["Mxz"]),
                              factor=float(s["factor"])))
    recs = _receivers_from_par(par, interfaces[-1] if interfaces else None)
    n = int(par["NSTEP"]) if nstep is None else nstep
    stacey = bool(par["STACEY_ABSORBING_CONDITIONS"]) or (
        absorbing_as_stacey and bool(par.get("PML_BOUNDARY_CONDITIONS", False)))
    if tomo_mats:
        from .gll import GLL
        from .mesh import createnum_fast, get_global, setup_mesh_coordinates

        # tomographic values are taken at the global coordinates of the GLL points
        gll = GLL()
        ib0, nglob = createnum_fast(mesh, gll)
        ibool = get_global(ib0)
        coord = setup_mesh_coordinates(mesh, gll, ibool, nglob)["coord"]
        els = np.flatnonzero(np.isin(mat_of, tomo_mats))
        r_t, vp_t, vs_t = tomo_values(tuple(np.asarray(a, dtype=np.float64) for a in tomo), coord, ibool, els)
        rho[els], vp[els], vs[els] = r_t, vp_t, vs_t
        rho, vp, vs = (a.astype(np.float32).astype(np.float64) for a in (rho, vp, vs))
    pml = None
    if bool(par.get("PML_BOUNDARY_CONDITIONS", False)) and not absorbing_as_stacey:
        if par.get("ROTATE_PML_ACTIVATE", False) or par.get("PML_PARAMETER_ADJUSTMENT", False):
            raise NotImplementedError("rotated PML and PML parameter adjustment")
        pml = dict(nelem_thickness=int(par["NELEM_PML_THICKNESS"]), k_min=float(par.get("K_MIN_PML", 1.0)),
                   k_max=float(par.get("K_MAX_PML", 1.0)),
                   damping_acoustic=float(par.get("damping_change_factor_acoustic", 0.5)),
                   damping_elastic=float(par.get("damping_change_factor_elastic", 1.0)))
    db = build_database(mesh, rho, vp, vs, sources, recs, n, float(par["DT"]), pml=pml,
                        stacey=stacey, external_model=external,
                        use_trick=bool(par.get("USE_TRICK_FOR_BETTER_PRESSURE", False)),
                        seismotype=int(par.get("seismotype", 1)),
                        time_scheme=int(time_scheme or par["time_stepping_scheme"]), user_t0=float(par["USER_T0"]),
                        anglerec_deg=float(par["anglerec"]),
                        qkappa=qk if atten else None, qmu=qm if atten else None,
                        attenuation_f0=float(par.get("ATTENUATION_f0_REFERENCE", 1.0)),
                        initialfield=bool(par.get("initialfield", False)))
    if is_aniso.any():
        db.aniso = {"ispec": is_aniso, **{k: v.astype(np.float32) for k, v in cstore.items()}}
    return db
