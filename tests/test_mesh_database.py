"""The mesher's binary database (Database<iproc>.bin, Fortran sequential
unformatted) as an input to the setup.

No Database file ships with the reference (its mesher is a Fortran program
that cannot be built here), so the reader is checked by round trips: an
example's mesh is written in save_databases.f90's record layout, read back,
and the Database the setup builds from it must equal the one built from the
example's own inputs array for array, and the external (Gmsh) example's
traces from the database path equal the direct path's, which are pinned to
its REF_SEIS."""
import os
import struct

import numpy as np
import pytest

from helpers import load_golden, load_kernel_golden, rel_l2
from specfem2d_b200.setup import acoustic as ac_setup
from specfem2d_b200.setup.database_file import read_database, write_database
from specfem2d_b200.setup.from_par_file import database_from_config
from specfem2d_b200.setup.parfile import material_from_row

ARRAYS = ("ibool", "xix", "xiz", "gammax", "gammaz", "jacobian", "rhostore", "kappastore", "mustore",
          "rmass_inverse_elastic", "stacey_iglob", "stacey_weight", "rec_ispec", "rec_xi", "rec_gamma",
          "source_ispec", "src_xi", "src_gamma")


def _materials(cfg):
    """The Par_file material table as the database's (index, kind, 13 values)."""
    out = []
    for row in cfg["materials"]:
        m = material_from_row(row)
        if m["kind"] == 2:
            vals = (m["rho"], m["c11"], m["c13"], m["c15"], m["c33"], m["c35"], m["c55"], 0, 0, 0, 0,
                    m["qkappa"], m["qmu"])
        else:
            vals = (m["rho"], m["vp"], m["vs"], 0, 0, m["qkappa"], m["qmu"], 0, 0, 0, 0, 0, 0)
        out.append((m["index"], m["kind"], vals))
    return out


def _round_trip(cfg, tmp_path, name):
    db = database_from_config(cfg)
    mesh = db.mesh
    is_ac = np.zeros(db.nspec, bool) if db.acoustic is None else np.asarray(db.acoustic["ispec"], bool)
    kmato = _kmato(cfg, db)
    free = mesh.free_edges if mesh.free_edges is not None else ac_setup.structured_free_edges(mesh, is_ac)
    coupled = [(ea + 1, ee + 1) for (ea, _, ee, _) in ac_setup.coupling_edges(db.ibool, is_ac)] if is_ac.any() else None
    path = os.path.join(tmp_path, name + ".bin")
    write_database(path, mesh, kmato, _materials(cfg),
                   params=dict(NSTEP=int(cfg["NSTEP"]), DT=float(cfg["DT"]), NGNOD=mesh.ngnod),
                   coupled=coupled, free_edges=free)
    cfg2 = {k: v for k, v in cfg.items() if k not in ("external_mesh", "interfaces", "nz_layer")}
    cfg2["mesh_database"] = read_database(path)
    return db, database_from_config(cfg2), path


def _kmato(cfg, db):
    if cfg.get("read_external_mesh"):
        return np.asarray(cfg["external_mesh"]["materials"], dtype=np.int64)
    nx = db.mesh.nx
    k = np.zeros(db.nspec, dtype=np.int64)
    for (ix0, ix1, iz0, iz1, imat) in cfg["regions"]:
        for iz in range(iz0, iz1 + 1):
            k[(iz - 1) * nx + ix0 - 1:(iz - 1) * nx + ix1] = imat
    return k


def _same(a, b):
    for k in ARRAYS:
        assert np.array_equal(getattr(a, k), getattr(b, k)), k
    if a.acoustic is not None:
        for k in ("ispec", "rmass", "st_iglob", "st_w", "free_iglob", "cpl_ac_iglob", "cpl_ac_w", "cpl_el_iglob",
                  "cpl_el_w"):
            assert np.array_equal(a.acoustic[k], b.acoustic[k]), k
    assert np.array_equal(a.mesh.abs_ispec, b.mesh.abs_ispec) and np.array_equal(a.mesh.abs_type, b.mesh.abs_type)
    assert np.array_equal(a.mesh.abs_corner, b.mesh.abs_corner)


def test_gmsh_example_round_trip_and_ref_seis(tmp_path):
    """External mesh: 2942 9-node fluid elements, 144 absorbing and 48 free-surface edges."""
    import oracle

    cfg, seis = load_golden("gmsh_stacey_external")
    db, db2, path = _round_trip(cfg, tmp_path, "gmsh")
    d = read_database(path)
    assert d["params"]["nspec"] == 2942 and d["params"]["NGNOD"] == 9 and d["params"]["NSTEP"] == 2400
    assert len(d["absorbing"]) == 144 and len(d["free_surface"]) == 48
    _same(db, db2)
    # the same arrays give the same traces (the direct path's are pinned to REF_SEIS)
    a, b = oracle.Oracle(db, 4).run(800), oracle.Oracle(db2, 4).run(800)
    assert np.array_equal(a, b)
    assert rel_l2(b[5, :, 0], seis["S0006_PRE"][:800]) < 1e-4


def test_fluid_solid_internal_mesh_round_trip(tmp_path):
    """Internal mesher, 9-node elements, fluid-solid coupling, Stacey on all sides."""
    cfg, _, _ = load_kernel_golden("luoyang_fluid_solid_kernel")
    db, db2, path = _round_trip(cfg, tmp_path, "luoyang")
    d = read_database(path)
    assert len(d["coupled"]) > 0 and len(d["free_surface"]) == 0
    _same(db, db2)


def test_elastic_round_trip(tmp_path):
    cfg, _ = load_golden("tromp2005_kernel")
    db, db2, _ = _round_trip(cfg, tmp_path, "tromp")
    _same(db, db2)


def test_reader_rejects_damaged_files(tmp_path):
    cfg, _ = load_golden("tromp2005_kernel")
    _, _, path = _round_trip(cfg, tmp_path, "ok")
    raw = open(path, "rb").read()
    # the first record is the 512-byte title, framed by its length
    assert struct.unpack_from("<i", raw, 0)[0] == 512 and struct.unpack_from("<i", raw, 516)[0] == 512
    bad = os.path.join(tmp_path, "bad.bin")
    for data in (raw[:-9], raw[:516] + struct.pack("<i", 511) + raw[520:], raw + raw[:8]):
        with open(bad, "wb") as f:
            f.write(data)
        with pytest.raises(ValueError):
            read_database(bad)
