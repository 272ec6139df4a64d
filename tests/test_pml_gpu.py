"""Parity of the CPML absorbing layers on the GPU (solid layer, fluid layer and
the coupling entries next to them) against the CPU oracle and the reference's
own traces.

Tolerance policy (relative L2), as for the other GPU paths: FP32 runs that
differ only in rounding drift apart by about as much as FP32 drifts from FP64,
so each GPU result must be at most 1.5-2x as far from the FP64 oracle as the
FP32 oracle is, or within 1e-5 of the FP32 oracle.
"""
import numpy as np
import pytest

from helpers import load_golden, rel_l2
from specfem2d_b200 import configs
from specfem2d_b200.setup.from_par_file import database_from_config

pytestmark = pytest.mark.gpu


def _close(gpu, ref, ref64, factor=1.5):
    return rel_l2(gpu, ref) < 1e-5 or rel_l2(gpu, ref64) < factor * rel_l2(ref, ref64)


def test_semi_infinite_cpml_matches_oracle_and_ref_seis():
    """EXAMPLES/semi_infinite_homogeneous: 3-element CPML on all four sides
    of an elastic square (564 layer elements), displacement receiver."""
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    cfg, seis = load_golden("semi_infinite_homogeneous")
    db = database_from_config(cfg)
    assert int((db.pml["region"] > 0).sum()) == 564
    gpu = ElasticSolver(db, tile_elems=32).run(db.nstep)
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    assert _close(gpu, o32, o64, 2.0)
    assert rel_l2(gpu[0, :, 0], seis["S0001_BXX"]) < 1e-5
    assert rel_l2(gpu[0, :, 1], seis["S0001_BXZ"]) < 1e-5


@pytest.mark.parametrize("name", ["force_source_elastic", "moment_tensor_dip_slip"])
def test_force_and_moment_tensor_cpml_examples(name):
    """EXAMPLES/check_absolute_amplitude_of_force_source_seismograms_elastic and
    EXAMPLES/infinite_homogeneous_moment_tensor_vertical_dip_slip (3-element
    CPML): traces against the oracle and the reference's REF_SEIS."""
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    cfg, seis = load_golden(name)
    db = database_from_config(cfg)
    gpu = ElasticSolver(db).run(db.nstep)
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    assert _close(gpu, o32, o64, 2.0)
    assert rel_l2(gpu[0, :, 0], seis["S0001_BXX"]) < 1e-5
    assert rel_l2(gpu[0, :, 1], seis["S0001_BXZ"]) < 1e-5


def test_nine_node_topography_fluid_example():
    """EXAMPLES/simple_topography_and_also_a_simple_fluid_layer (9-node elements,
    fluid layer, CPML): the coupled solver against the oracle and REF_SEIS."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    cfg, seis = load_golden("topography_fluid_layer")
    db = database_from_config(cfg)
    gpu = CoupledSolver(db).run(db.nstep)
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    assert _close(gpu, o32, o64, 2.0)
    for k in range(11):
        assert rel_l2(gpu[k, :, 0], seis[f"S{k + 1:04d}_BXX"]) < 1e-5
        assert rel_l2(gpu[k, :, 1], seis[f"S{k + 1:04d}_BXZ"]) < 1e-5


def test_semi_infinite_cpml_fields_and_layer_absorbs():
    """Displacement field after the run (16-element tiles) against the oracle."""
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    cfg, _ = load_golden("semi_infinite_homogeneous")
    db = database_from_config(cfg)
    s = ElasticSolver(db, tile_elems=16)
    s.run(db.nstep, seismograms=False)
    u_gpu = s.get_fields()[0]
    o32, o64 = oracle.Oracle(db, 4), oracle.Oracle(db, 8)
    o32.run(db.nstep)
    o64.run(db.nstep)
    assert _close(u_gpu, o32.displ, o64.displ, 2.0)


@pytest.mark.parametrize("tile_elems,threads", [(32, 256), (16, 250)])
def test_attenuating_cpml_matches_oracle_and_ref_seis(tile_elems, threads):
    """EXAMPLES/attenuation/viscoelastic with its own 3-element CPML layers in an
    attenuating solid (Qkappa 22.3, Qmu 20, 3 SLS; 492 layer elements take the
    viscoelastic layer update), the whole 1400-step trace against REF_SEIS, and
    the final displacement field against the oracle."""
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    cfg, seis = load_golden("attenuation_viscoelastic")
    db = database_from_config(cfg)
    assert int(np.sum(db.pml["visco"])) == 492
    s = ElasticSolver(db, tile_elems=tile_elems, threads_per_block=threads)
    gpu = s.run(db.nstep)
    u_gpu = s.get_fields()[0]
    o32, o64 = oracle.Oracle(db, 4), oracle.Oracle(db, 8)
    r32, r64 = o32.run(db.nstep), o64.run(db.nstep)
    assert _close(gpu, r32, r64, 2.0)
    assert _close(u_gpu, o32.displ, o64.displ, 2.0)
    assert rel_l2(gpu[0, :, 0], seis["S0001_BXX"]) < 1e-5
    assert rel_l2(gpu[0, :, 1], seis["S0001_BXZ"]) < 1e-5


def test_attenuating_cpml_with_lddrk_is_rejected():
    """The reference stops for LDDRK in an attenuating CPML layer
    (pml_compute_memory_variables.f90:736-741); so does the solver."""
    from specfem2d_b200.runtime import ElasticSolver, SF2DError

    cfg, _ = load_golden("attenuation_viscoelastic")
    db = database_from_config(cfg, time_scheme=2)
    with pytest.raises(SF2DError, match="Newmark"):
        ElasticSolver(db)


def test_fluid_only_cpml_pressure_matches_oracle_and_ref_seis():
    """EXAMPLES/check_absolute_amplitude_of_pressure_source_seismograms_acoustic:
    a fluid-only mesh (no solid sub-solver) with CPML on all sides (492 layer
    elements), a Gaussian pressure source with USE_TRICK_FOR_BETTER_PRESSURE
    and one pressure receiver."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    cfg, seis = load_golden("pressure_source_acoustic")
    db = database_from_config(cfg)
    assert int((db.pml["region"] > 0).sum()) == 492 and db.seismotype == 4
    s = CoupledSolver(db)
    gpu = s.run(db.nstep)
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    assert _close(gpu, o32, o64, 2.0)
    assert rel_l2(gpu[0, :, 0], seis["S0001_PRE"]) < 1e-5
    assert s.launch_count(64) > 0


@pytest.fixture(scope="module")
def c2_pml():
    db = configs.c2_coupled(nstep=1200, nrec=24, scale=8, pml_thickness=3)
    assert (db.pml["region"][db.acoustic["ispec"]] > 0).any()
    return db


def test_coupled_cpml_pressure_and_fields(c2_pml):
    """Coupled model with CPML on the sides and bottom: the sea floor crosses
    the side layers, so both coupling directions carry the layer's memory
    terms.  Pressure traces and both domains' fields against the oracle."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db = c2_pml
    s = CoupledSolver(db)
    gpu = s.run(db.nstep)
    f = s.get_fields()
    o32, o64 = oracle.Oracle(db, 4), oracle.Oracle(db, 8)
    r32, r64 = o32.run(db.nstep), o64.run(db.nstep)
    assert _close(gpu, r32, r64)
    assert _close(f["displ"], o32.displ, o64.displ, 2.0)
    assert _close(f["pot"], o32.get(oracle.POT), o64.get(oracle.POT), 2.0)


def test_coupled_cpml_250_threads(c2_pml):
    """250-thread CTAs (one GLL position per thread, hprime rows in
    registers) in both domains' tile kernels, with and without the layer."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db = c2_pml
    gpu = CoupledSolver(db, threads_per_block=250).run(600)
    r32 = oracle.Oracle(db, 4).run(600)
    r64 = oracle.Oracle(db, 8).run(600)
    assert _close(gpu, r32, r64)


def test_coupled_cpml_small_layer_tiles(c2_pml):
    """The benchmark's tile options: 64-element fluid tiles, and the solid
    layer in 16-element tiles of its own 128-thread kernel (its shared-memory
    layout sized by the layer's tiles)."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db = c2_pml
    s = CoupledSolver(db, fluid_tile_elems=64, pml_tile_elems=16, pml_threads_per_block=128)
    gpu = s.run(600)
    f = s.get_fields()
    o32, o64 = oracle.Oracle(db, 4), oracle.Oracle(db, 8)
    r32, r64 = o32.run(600), o64.run(600)
    assert _close(gpu, r32, r64)
    assert _close(f["displ"], o32.displ, o64.displ, 2.0)


def test_semi_infinite_cpml_small_layer_tiles():
    """Elastic layer in 8-element tiles with 128 threads beside 32-element tiles."""
    import oracle
    from specfem2d_b200.runtime import ElasticSolver

    cfg, seis = load_golden("semi_infinite_homogeneous")
    db = database_from_config(cfg)
    gpu = ElasticSolver(db, tile_elems=32, pml_tile_elems=8, pml_threads_per_block=128).run(db.nstep)
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    assert _close(gpu, o32, o64, 2.0)
    assert rel_l2(gpu[0, :, 0], seis["S0001_BXX"]) < 1e-5


def test_coupled_cpml_lddrk(c2_pml):
    """The same model with LDDRK: six stages of every memory variable."""
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db = configs.c2_coupled(nstep=400, nrec=24, scale=8, pml_thickness=3, time_scheme=2)
    gpu = CoupledSolver(db).run(db.nstep)
    r32 = oracle.Oracle(db, 4).run(db.nstep)
    r64 = oracle.Oracle(db, 8).run(db.nstep)
    assert _close(gpu, r32, r64)


def test_coupled_cpml_chunking_is_bitwise(c2_pml):
    """CUDA-graph chunks and plain launches give identical bits with the
    layer's memory variables carried across runs."""
    from specfem2d_b200.coupled import CoupledSolver

    db = c2_pml
    a = CoupledSolver(db)
    ta = np.concatenate([a.run(100), a.run(37), a.run(63)], axis=1)
    b = CoupledSolver(db)
    tb = b.run(200)
    assert np.array_equal(ta, tb)
    fa, fb = a.get_fields(), b.get_fields()
    for k in ("displ", "veloc", "pot", "pot_dot"):
        assert np.array_equal(fa[k], fb[k])
