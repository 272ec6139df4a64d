"""CPU-side checks of the C-ABI library: it loads without a GPU, exports every
function include/sf2d_b200.h declares, and its tiler keeps its invariants."""
import os
import re

import numpy as np
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


def fortran_symbols():
    txt = open(os.path.join(ROOT, "include", "sf2d_fortran.h")).read()
    return sorted(set(re.findall(r"^void (\w+_)\(", txt, re.M)))


def test_library_exports_the_reference_fortran_interface():
    """All 91 entry points of the reference's src/gpu Fortran interface
    (specfem2D_gpu_cuda_method_stubs.c) with gfortran's trailing underscore."""
    lib = runtime.load_library()
    names = fortran_symbols()
    assert len(names) == 91
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_exports_only_its_interfaces():
    """The shared object exports the C ABI (sf2d_*) and the Fortran entry points
    and nothing else (a linker version script): no C++ internal of the library
    can bind to a host program's symbols."""
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", runtime.LIB], capture_output=True, text=True,
                         check=True).stdout.split("\n")
    names = {ln.split()[-1] for ln in out if ln.strip()}
    allowed = set(fortran_symbols())
    extra = sorted(n for n in names if not n.startswith("sf2d_") and n not in allowed)
    assert not extra, extra[:10]
    assert allowed <= names


@pytest.mark.parametrize("call,needle", [
    ("pml_boundary_acoustic_cuda_", "Mesh_pointer was not prepared"),
    ("compute_kernels_hess_cuda_", "not provided by libsf2d_b200"),
    ("compute_forces_acoustic_cuda_", "Mesh_pointer was not prepared"),
    ("kernel_3_b_cuda_", "sf2d_fwi_create"),
    ("transfer_boun_accel_from_device_", "MPI"),
    ("update_displacement_cuda_", "Mesh_pointer was not prepared"),
    ("transfer_kernels_el_to_host_", "Mesh_pointer was not prepared"),
    ("transfer_b_fields_from_device_", "sf2d_fwi_create"),
])
def test_fortran_interface_errors_exit_like_the_reference(call, needle):
    """A call the library does not provide, or one on an unprepared handle, prints
    the reason and exits with EXIT_FAILURE, as the reference's exit_on_error does
    (no GPU is touched)."""
    import subprocess
    import sys

    code = ("import ctypes, sys; sys.path.insert(0, %r); from specfem2d_b200.runtime import load_library; "
            "lib = load_library(); h = ctypes.c_long(0); z = ctypes.c_int(0); "
            "getattr(lib, %r)(ctypes.byref(h), ctypes.byref(z), ctypes.byref(z), ctypes.byref(z), "
            "ctypes.byref(z), ctypes.byref(z), ctypes.byref(z)); print('returned')") % (ROOT, call)
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=120)
    assert p.returncode == 1, (p.returncode, p.stdout, p.stderr)
    assert needle in p.stderr and "returned" not in p.stdout


def test_fortran_host_absorbing_faces_give_the_solver_stacey_points():
    """The face arrays of prepare_timerun.F90 (fortran_host), unrolled the way
    prepare_stacey_device unrolls them (points marked NGLLX + 1 left out), are
    the per-point Stacey entries of the solver setup, value for value."""
    import numpy as np

    from specfem2d_b200.setup.fortran_host import gpu_arrays

    cfg, _ = load_golden("tromp2005_kernel")
    db = database_from_config(cfg, nstep=4)
    A = gpu_arrays(db)
    ab = A["abs"]
    ig, nx, nz, w, rvp = [], [], [], [], []
    for f in range(ab["nface"]):
        e = ab["abs_boundary_ispec"][f] - 1
        for k in range(5):
            i, j = ab["abs_boundary_ij"][f, k] - 1
            if i == 5 or j == 5:
                continue
            ig.append(db.ibool[e, j, i])
            nx.append(ab["abs_boundary_normal"][f, k, 0])
            nz.append(ab["abs_boundary_normal"][f, k, 1])
            w.append(ab["abs_boundary_jacobian1Dw"][f, k])
            rvp.append(A["rho_vpstore"][e, j, i])
    assert np.array_equal(np.array(ig), db.stacey_iglob)
    for got, want in ((nx, db.stacey_nx), (nz, db.stacey_nz), (w, db.stacey_weight), (rvp, db.stacey_rho_vp)):
        assert np.array_equal(np.array(got, np.float32), want)
    # hprime_xx(i2, i1) = l'_i1(xi_i2) in Fortran order
    assert A["hprime_xx"].ravel()[1 * 5 + 3] == db.gll.hprime[3, 1]


def test_fortran_host_pml_arrays_restate_the_layer_profiles():
    """prepare_PML_device's arrays for the fluid CPML example: elements numbered
    X, then Z, then XZ; the profiles the GPU path forms from them (alpha =
    ALPHA_MAX_PML (1 - abs), d = 2 d0_max abs^2 in X and Z elements, the stores
    in XZ ones, all in FP32) equal the set-up's K = 1 profiles to FP32 rounding."""
    from specfem2d_b200.setup.fortran_host import pml_arrays

    cfg, _ = load_golden("pressure_source_acoustic")
    db = database_from_config(cfg)
    P = pml_arrays(db)
    pm = db.pml
    region = np.asarray(pm["region"])
    assert (P["nspec_pml_x"], P["nspec_pml_z"], P["nspec_pml_xz"]) == (228, 228, 36)
    spec = P["spec_to_pml"]
    assert np.array_equal(np.flatnonzero(spec), np.flatnonzero(region))
    for code, lo, hi in ((1, 1, 228), (2, 229, 456), (3, 457, 492)):
        els = np.flatnonzero(region == code)
        assert np.array_equal(spec[els], np.arange(lo, hi + 1))
    assert np.all(pm["K_x"] == 1.0) and np.all(pm["K_z"] == 1.0)
    f = np.float32
    for e in np.flatnonzero(region):
        p = spec[e] - 1
        if region[e] < 3:
            a = P["abs_normalized"][p]
            alpha = P["alpha_max"] * (f(1) - a)
            d = (alpha + f(2) * P["d0_max"] * a * a).astype(np.float64) - alpha.astype(np.float64)
            kd, ka = ("d_x", "alpha_x") if region[e] == 1 else ("d_z", "alpha_z")
            assert np.allclose(d, pm[kd][e], rtol=1e-6, atol=1e-6 * pm[kd].max()), e
            assert np.allclose(alpha, pm[ka][e], rtol=1e-6, atol=1e-6 * pm[ka].max()), e
        else:
            k = p - 456
            d = P["betax"][k].astype(np.float64) - P["alphax"][k].astype(np.float64)
            assert np.allclose(d, pm["d_x"][e], rtol=1e-6, atol=1e-6 * pm["d_x"].max()), e
    assert np.array_equal(P["abs_points_acoustic"], np.asarray(pm["bnd_ac"]) + 1)
