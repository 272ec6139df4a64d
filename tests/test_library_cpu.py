"""CPU-side checks of the C-ABI library: it loads without a GPU, exports every
function include/sf2d_b200.h declares, and its tiler keeps its invariants."""
import os
import re

import pytest

from specfem2d_b200 import runtime
from specfem2d_b200.setup.from_par_file import database_from_config
from helpers import load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(sf2d_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = runtime.load_library()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.parametrize("tile_elems", [1, 7, 16, 64, 200])
def test_tiling_invariants(tile_elems):
    cfg, _ = load_golden("tromp2005_kernel")
    db = database_from_config(cfg, nstep=4)
    st = runtime.tiling_stats(db, tile_elems)
    assert st["ntiles"] == -(-db.nspec // tile_elems)
    assert st["n_interior"] + st["nshared"] == db.nglob
    assert st["max_colours"] <= 8


def test_coupled_split_keeps_every_interface_point():
    """The fluid/solid split used by the coupled GPU path: both sub-meshes hold
    every coupling point, solid absorbing points stay in the solid mesh, and
    receivers are partitioned between the domains."""
    from specfem2d_b200 import configs
    from specfem2d_b200.coupled import split

    db = configs.c2_coupled(nstep=10, nrec=8, scale=16)
    sub, fl, cp, maps = split(db)
    assert sub.nspec + fl["nspec"] == db.nspec
    assert (cp["ac_point"] >= 0).all() and (cp["ac_el_point"] >= 0).all()
    assert (cp["el_point"] >= 0).all() and (cp["el_ac_point"] >= 0).all()
    g = db.acoustic["cpl_ac_iglob"]
    assert (maps["fluid_points"][cp["ac_point"]] == g).all() and (maps["solid_points"][cp["ac_el_point"]] == g).all()
    assert len(fl["rec_global"]) + len(cp["el_rec_global"]) == len(db.rec_ispec)
    assert sub.ibool.max() == sub.nglob - 1 and fl["ibool"].max() == fl["nglob"] - 1
