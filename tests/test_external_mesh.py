"""External (Gmsh) meshes: the reader's edge rules on small cases, and
EXAMPLES/Gmsh_example_Stacey_MPI rebuilt from its MESH/ tables and pinned to
the reference's located source and receivers and its 11 REF_SEIS pressure
traces (oracle on the CPU, the fluid solver on the GPU).

That run was made on 4 MPI slices in FP32: its traces differ from a serial
FP32 run only by rounding, which in this case grows to 1e-4 over the 2400
steps (the FP32 oracle itself is that far from the FP64 oracle).  So the FP64
oracle must be within the FP32 band of REF_SEIS, and each FP32 result within
1.5x that band."""
import numpy as np
import pytest

from helpers import load_golden, rel_l2
from specfem2d_b200.setup.external_mesh import external_mesh
from specfem2d_b200.setup.from_par_file import database_from_config
from specfem2d_b200.setup.mesh import IBOTTOM, ILEFT, IRIGHT, ITOP

NAME = "gmsh_stacey_external"


def _two_quads():
    """Two unit squares side by side, 4-node elements, 1-based node ids."""
    nodes = np.array([[0, 0], [1, 0], [2, 0], [0, 1], [1, 1], [2, 1]], dtype=np.float64)
    elements = np.array([[1, 2, 5, 4], [2, 3, 6, 5]])
    return {"elements": elements, "nodes": nodes, "materials": np.array([1, 2]),
            "absorbing": np.zeros((0, 5), np.int64), "free_surface": np.zeros((0, 4), np.int64)}


def test_absorbing_lines_give_the_element_edge_whatever_the_node_order():
    t = _two_quads()
    # element 1: bottom (2-1, reversed), left; element 2: right, top (5-6 reversed)
    t["absorbing"] = np.array([[1, 2, 2, 1, 1], [1, 2, 4, 1, 4], [2, 2, 3, 6, 2], [2, 2, 6, 5, 3]])
    m = external_mesh(t, 4, fluid_materials=[1, 2])
    assert list(m.abs_ispec) == [0, 0, 1, 1]
    assert list(m.abs_type) == [IBOTTOM, ILEFT, IRIGHT, ITOP]
    # the bottom edge of element 1 skips its corner with the left edge; element 2's top its right corner
    assert m.abs_corner.tolist() == [[True, False, False, False], [False] * 4, [False] * 4,
                                     [False, False, False, True]]


def test_free_surface_lines_give_gll_ranges_and_skip_solid_elements():
    t = _two_quads()
    t["free_surface"] = np.array([[1, 2, 5, 4], [2, 2, 6, 5], [1, 1, 1, 0]])
    m = external_mesh(t, 4, fluid_materials=[1])
    # element 2 is not fluid; element 1: top edge (i 0..4, j 4) and the bottom-left corner point
    assert m.free_edges.tolist() == [[0, 0, 4, 4, 4], [0, 0, 0, 0, 0]]


def test_lines_that_name_no_element_edge_are_rejected():
    t = _two_quads()
    t["absorbing"] = np.array([[1, 2, 1, 5, 1]])      # a diagonal
    with pytest.raises(ValueError):
        external_mesh(t, 4, fluid_materials=[1])
    t["absorbing"] = np.array([[1, 3, 1, 2, 1]])      # three nodes
    with pytest.raises(ValueError):
        external_mesh(t, 4, fluid_materials=[1])
    t = _two_quads()
    t["free_surface"] = np.array([[1, 2, 1, 3]])      # node 3 is not a corner of element 1
    with pytest.raises(ValueError):
        external_mesh(t, 4, fluid_materials=[1])


@pytest.fixture(scope="module")
def gmsh():
    cfg, seis = load_golden(NAME)
    return database_from_config(cfg), cfg, seis


def test_gmsh_setup_matches_reference_log(gmsh):
    """The source and the 11 receivers land at the reference's (xi, gamma) to
    1e-12 (its element numbers are those of its MPI slices); 2942 fluid
    elements, 144 absorbing edges, 48 free-surface edges (193 points)."""
    db, cfg, _ = gmsh
    assert db.nspec == 2942 and db.mesh.ngnod == 9
    assert len(db.acoustic["ispec"]) == 2942
    assert len(db.mesh.abs_ispec) == 144 and len(db.mesh.free_edges) == 48
    assert len(db.acoustic["free_iglob"]) == 193
    log = np.array([[xi, ga] for (_, xi, ga) in cfg["log_locations"]])
    got = np.array([[db.src_xi[0], db.src_gamma[0]]] + [[x, g] for x, g in zip(db.rec_xi, db.rec_gamma)])
    assert np.abs(got - log).max() < 1e-12


def test_gmsh_oracle_reproduces_ref_seis(gmsh):
    import oracle

    db, _, seis = gmsh
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    assert float(seis["t_first"]) == pytest.approx(-db.t0)
    for k in range(11):
        ref = seis[f"S{k + 1:04d}_PRE"]
        band = rel_l2(o32[k, :, 0], o64[k, :, 0])
        assert band < 5e-4
        assert rel_l2(o64[k, :, 0], ref) < band
        assert rel_l2(o32[k, :, 0], ref) < 1.5 * band


def test_gmsh_pin_detects_a_missing_free_surface():
    """A mistake planted in the oracle's input: without the listed free
    surface the traces are O(1) away from REF_SEIS."""
    import oracle

    cfg, seis = load_golden(NAME)
    cfg["external_mesh"]["free_surface"] = cfg["external_mesh"]["free_surface"][:0]
    db = database_from_config(cfg, nstep=1200)
    out = oracle.Oracle(db, 8).run(db.nstep)
    assert rel_l2(out[5, :, 0], seis["S0006_PRE"][:1200]) > 0.1


@pytest.mark.gpu
def test_gmsh_gpu_matches_oracle_and_ref_seis(gmsh):
    import oracle
    from specfem2d_b200.coupled import CoupledSolver

    db, _, seis = gmsh
    s = CoupledSolver(db)
    gpu = s.run(db.nstep)
    assert s.launch_count(64) > 0
    s.close()
    o32 = oracle.Oracle(db, 4).run(db.nstep)
    o64 = oracle.Oracle(db, 8).run(db.nstep)
    for k in range(11):
        band = rel_l2(o32[k, :, 0], o64[k, :, 0])
        assert rel_l2(gpu[k, :, 0], o32[k, :, 0]) < 1e-5 or rel_l2(gpu[k, :, 0], o64[k, :, 0]) < 1.5 * band
        assert rel_l2(gpu[k, :, 0], seis[f"S{k + 1:04d}_PRE"]) < 2.0 * band
