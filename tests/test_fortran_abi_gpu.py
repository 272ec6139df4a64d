"""The reference's own Fortran-to-GPU interface (include/sf2d_fortran.h), driven
the way the SPECFEM2D Fortran host drives it (tests/fortran_driver.py: the
call order of prepare_gpu.f90, iterate_time.F90, compute_gpu_elastic.f90 and
write_seismograms.F90, arguments by reference, 1-based indices, Fortran array
order).  No Fortran compiler is needed: the calls are the C symbols gfortran
would make.

Tolerances (relative L2): the reference's REF_SEIS traces within 1e-5; the
same run through this library's own C ABI within 1e-5 (the interface forms
lambda = kappa - mu in FP32 as the reference's GPU kernel does, the C ABI
takes lambda as the CPU solver forms it).
"""
import numpy as np
import pytest

from fortran_driver import run_forward
from helpers import load_golden, rel_l2
from specfem2d_b200.setup.from_par_file import database_from_config

pytestmark = pytest.mark.gpu


def test_tromp2005_through_the_fortran_interface_matches_ref_seis():
    from specfem2d_b200.runtime import ElasticSolver

    cfg, golden = load_golden("tromp2005_kernel")
    db = database_from_config(cfg)
    seis, displ, norms = run_forward(db)
    assert rel_l2(seis[0, :, 0], golden["S0001_BXX"]) < 1e-5
    assert rel_l2(seis[0, :, 1], golden["S0001_BXZ"]) < 1e-5
    sol = ElasticSolver(db)
    s = sol.run(db.nstep)
    d, _, _ = sol.get_fields()
    assert rel_l2(seis, s) < 1e-5
    assert rel_l2(displ, d) < 1e-5
    assert len(norms) == 3 and norms[-1] > 0


def test_seismogram_buffer_flushes_match_one_buffer():
    """NTSTEP_BETWEEN_OUTPUT_SEISMOS shorter than the run: the host's trace
    buffer is handed over five times; the traces are those of one buffer."""
    cfg, _ = load_golden("tromp2005_kernel")
    db = database_from_config(cfg, nstep=1400)
    a, _, _ = run_forward(db)
    b, _, _ = run_forward(db, nlength_seismogram=300)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name", ["anisotropic_isotropic_model", "attenuation_viscoelastic"])
def test_anisotropic_and_attenuating_examples_through_the_fortran_interface(name):
    """Anisotropic elements (c_ij arrays of prepare_fields_elastic_device) and
    3-SLS attenuation (its A/B Newmark arrays), against the FP32 oracle."""
    import oracle

    cfg, _ = load_golden(name)
    db = database_from_config(cfg, absorbing_as_stacey=True)
    seis, displ, _ = run_forward(db)
    o = oracle.Oracle(db, 4)
    ref = o.run(db.nstep)
    assert rel_l2(seis, ref) < 1e-5
    assert rel_l2(displ, o.displ) < 1e-5
