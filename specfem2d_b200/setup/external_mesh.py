"""External (Gmsh / CUBIT) meshes: the text files the mesher reads when
``read_external_mesh`` is set, turned into a setup Mesh.

* element connectivity, node coordinates, material per element, free-surface
  and absorbing edge lists -- src/meshfem2D/read_external_mesh_files.F90:43-516
  (text form; every node id is shifted by the smallest id of the connectivity,
  element ids of the edge lists too)
* absorbing edge code from the two listed nodes (the element edge whose
  corners they are, in either order) -- src/meshfem2D/part_unstruct.F90:765-818,
  one entry per listed line (an element with two absorbing edges is listed
  twice), then the corner flags of src/specfem2D/read_mesh_databases.F90:985-1030
* free-surface GLL range of an edge from its nodes -- get_acoustic_edge in
  src/specfem2D/construct_acoustic_surface.f90:72-200; only edges of acoustic
  (fluid, non-anisotropic) elements are kept
  (read_external_mesh_files.F90:398-420)

The listed edges keep the file's order, as the mesher writes them.
"""
from __future__ import annotations

import numpy as np

from .gll import NGLL
from .mesh import IBOTTOM, ILEFT, IRIGHT, ITOP, Mesh, absorbing_corners

L = NGLL - 1

# element corners of each edge code: bottom 0-1, right 1-2, top 2-3, left 3-0
_EDGE_CORNERS = {IBOTTOM: (0, 1), IRIGHT: (1, 2), ITOP: (2, 3), ILEFT: (3, 0)}
# GLL (i, j) of the four corners
_CORNER_IJ = ((0, 0), (L, 0), (L, L), (0, L))


def _read_table(path: str, ncols: int, dtype):
    """A count on the first line, then that many rows of `ncols` numbers."""
    with open(path) as f:
        n = int(f.readline().split()[0])
        rows = np.loadtxt(f, dtype=dtype, ndmin=2, max_rows=n) if n else np.zeros((0, ncols), dtype)
    if rows.shape != (n, ncols):
        raise ValueError(f"{path}: expected {n} rows of {ncols} values, read {rows.shape}")
    return rows


def read_external_mesh_files(mesh_file: str, nodes_file: str, materials_file: str, ngnod: int,
                             free_surface_file: str | None = None, absorbing_file: str | None = None) -> dict:
    """The raw tables of the external-mesh text files, ids as in the files:
    ``elements`` (nspec, ngnod), ``nodes`` (nnodes, 2), ``materials``
    (nspec,), ``absorbing`` (nabs, 5) and ``free_surface`` (nfree, 4)."""
    if ngnod not in (4, 9):
        raise ValueError("NGNOD should be either 4 or 9 for external meshes")
    out = {"elements": _read_table(mesh_file, ngnod, np.int64), "nodes": _read_table(nodes_file, 2, np.float64)}
    with open(materials_file) as f:
        mat = np.array([int(ln.split()[0]) for ln in f if ln.strip()], dtype=np.int64)
    if mat.size < len(out["elements"]):
        raise ValueError(f"{materials_file}: {mat.size} materials for {len(out['elements'])} elements")
    out["materials"] = mat[:len(out["elements"])]
    if np.any(out["materials"] == 0):
        raise ValueError("some elements have material index zero")
    out["absorbing"] = _read_table(absorbing_file, 5, np.int64) if absorbing_file else np.zeros((0, 5), np.int64)
    out["free_surface"] = (_read_table(free_surface_file, 4, np.int64) if free_surface_file
                           else np.zeros((0, 4), np.int64))
    return out


def _edge_code(corners, n1: int, n2: int) -> int:
    """The edge of an element (corner node ids `corners`) whose two corners are n1 and n2."""
    hit = [t for t, (a, b) in _EDGE_CORNERS.items() if {n1, n2} == {int(corners[a]), int(corners[b])}]
    if len(hit) != 1:
        raise ValueError("an absorbing line must name the two corner nodes of one element edge")
    return hit[0]


def _free_range(corners, nn: int, n1: int, n2: int):
    """(imin, imax, jmin, jmax) of a listed free-surface point (nn = 1) or edge."""
    where = {int(c): k for k, c in enumerate(corners[:4])}
    if n1 not in where or (nn != 1 and n2 not in where):
        raise ValueError("a free-surface line must name corner nodes of its element")
    i1, j1 = _CORNER_IJ[where[n1]]
    if nn == 1:
        return i1, i1, j1, j1
    i2, j2 = _CORNER_IJ[where[n2]]
    if i1 != i2 and j1 != j2:
        raise ValueError("a free-surface line must name the two corners of one element edge")
    return min(i1, i2), max(i1, i2), min(j1, j2), max(j1, j2)


def external_mesh(tables: dict, ngnod: int, fluid_materials) -> Mesh:
    """Mesh of the raw tables.  ``fluid_materials`` holds the 1-based material
    numbers of acoustic, non-anisotropic materials: free-surface lines of other
    elements are dropped."""
    elm = np.asarray(tables["elements"], dtype=np.int64)
    shift = int(elm.min())
    knods = elm - shift
    nodes = np.asarray(tables["nodes"], dtype=np.float64)
    if int(knods.max()) >= len(nodes):
        raise ValueError("the connectivity names more nodes than the coordinates file holds")
    mesh = Mesh(nspec=len(knods), ngnod=ngnod, knods=knods, coorg=nodes.copy())
    ab = np.asarray(tables["absorbing"], dtype=np.int64)
    isp, typ = [], []
    for row in ab:
        e, nn, n1, n2 = int(row[0]) - shift, int(row[1]), int(row[2]) - shift, int(row[3]) - shift
        if nn != 2:
            raise ValueError("only two nodes per absorbing element can be listed")
        if not 1 <= int(row[4]) <= 4:
            raise ValueError("absorbing element type must be between 1 (IBOTTOM) and 4 (ILEFT)")
        isp.append(e)
        typ.append(_edge_code(knods[e], n1, n2))
    mesh.abs_ispec = np.array(isp, dtype=np.int64)
    mesh.abs_type = np.array(typ, dtype=np.int64)
    mesh.abs_corner = absorbing_corners(mesh.abs_ispec, mesh.abs_type)
    mat = np.asarray(tables["materials"], dtype=np.int64)
    fluid = set(int(m) for m in fluid_materials)
    free = []
    for row in np.asarray(tables["free_surface"], dtype=np.int64):
        e = int(row[0]) - shift
        if int(mat[e]) not in fluid:
            continue
        free.append((e,) + _free_range(knods[e], int(row[1]), int(row[2]) - shift, int(row[3]) - shift))
    mesh.free_edges = np.array(free, dtype=np.int64).reshape(-1, 5)
    mesh.free_top = False
    mesh.absorb = (False, False, False, False)
    return mesh
