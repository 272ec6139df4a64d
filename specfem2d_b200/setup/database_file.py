"""The mesher's binary mesh database, OUTPUT_FILES/Database<iproc>.bin.

A Fortran sequential unformatted file (gfortran: every record framed by its
byte length as a 4-byte integer before and after it; integers and logicals
4 bytes, doubles 8, strings at their declared length).  Written by
src/meshfem2D/save_databases.f90:34-702 with the writers of
src/meshfem2D/part_unstruct.F90 (write_glob2loc_nodes_database :416-448,
write_partition_database :457-499, write_surface_database :624-698,
write_abs_merge_database :956-1000, write_fluidsolid_edges_database
:1195-1231, write_axial_elements_database :1241-1285), and read back by the
solver in the same order (read_mesh_for_init, read_mesh_databases:
src/specfem2D/read_mesh_databases.F90:34-402, 409-1400).

`read_database` parses one file into plain arrays; `mesh_from_database` turns
them into a setup Mesh (absorbing edge codes from the codeabs flags, corner
flags as the solver sets them, free-surface GLL ranges from the listed
nodes); `write_database` writes the same layout (for round trips, and to
hand one of this package's meshes to the reference's solver).  The record
order and field types are the format's definition and are kept as the
reference has them.
"""
from __future__ import annotations

import struct

import numpy as np

from .mesh import IBOTTOM, ILEFT, IRIGHT, ITOP, Mesh, absorbing_corners

STRING_LEN = 512  # MAX_STRING_LEN (constants.h)

# save_databases_init, one entry per record: (names, field codes); i int32,
# l logical (int32), d float64, s string (the whole record)
INIT_RECORDS = (
    (("title",), "s"),
    (("NOISE_TOMOGRAPHY", "UNDO_ATTENUATION_AND_OR_PML"), "il"),
    (("nspec",), "i"),
    (("npgeo", "NPROC"), "ii"),
    (("output_grid_Gnuplot", "interpol"), "ll"),
    (("NTSTEP_BETWEEN_OUTPUT_INFO",), "i"),
    (("NTSTEP_BETWEEN_OUTPUT_SEISMOS",), "i"),
    (("NTSTEP_BETWEEN_OUTPUT_IMAGES",), "i"),
    (("PML_BOUNDARY_CONDITIONS",), "l"),
    (("ROTATE_PML_ACTIVATE",), "l"),
    (("ROTATE_PML_ANGLE",), "d"),
    (("K_MIN_PML",), "d"),
    (("K_MAX_PML",), "d"),
    (("damping_change_factor_acoustic",), "d"),
    (("damping_change_factor_elastic",), "d"),
    (("PML_PARAMETER_ADJUSTMENT",), "l"),
    (("read_external_mesh",), "l"),
    (("NELEM_PML_THICKNESS",), "i"),
    (("NTSTEP_BETWEEN_OUTPUT_SAMPLE", "imagetype_JPEG", "imagetype_wavefield_dumps"), "iii"),
    (("output_postscript_snapshot", "output_color_image"), "ll"),
    (("meshvect", "modelvect", "boundvect", "cutsnaps", "subsamp_postscript", "sizemax_arrows"), "llldid"),
    (("anglerec",), "d"),
    (("initialfield",), "l"),
    (("add_Bielak_conditions_bottom", "add_Bielak_conditions_right", "add_Bielak_conditions_top",
      "add_Bielak_conditions_left"), "llll"),
    (("seismotype", "imagetype_postscript"), "si"),
    (("MODEL",), "s"),
    (("SAVE_MODEL",), "s"),
    (("TOMOGRAPHY_FILE",), "s"),
    (("output_grid_ASCII", "OUTPUT_ENERGY", "NTSTEP_BETWEEN_OUTPUT_ENERGY", "output_wavefield_dumps"), "llil"),
    (("use_binary_for_wavefield_dumps",), "l"),
    (("ATTENUATION_VISCOELASTIC", "ATTENUATION_PORO_FLUID_PART", "ATTENUATION_VISCOACOUSTIC"), "lll"),
    (("USE_SOLVOPT",), "l"),
    (("save_ASCII_seismograms",), "l"),
    (("save_binary_seismograms_single", "save_binary_seismograms_double"), "ll"),
    (("USE_TRICK_FOR_BETTER_PRESSURE",), "l"),
    (("COMPUTE_INTEGRATED_ENERGY_FIELD",), "l"),
    (("save_ASCII_kernels",), "l"),
    (("NTSTEP_BETWEEN_COMPUTE_KERNELS",), "i"),
    (("APPROXIMATE_HESS_KL",), "l"),
    (("NO_BACKWARD_RECONSTRUCTION",), "l"),
    (("DRAW_SOURCES_AND_RECEIVERS",), "l"),
    (("Q0_poroelastic", "freq0_poroelastic"), "dd"),
    (("AXISYM",), "l"),
    (("P_SV",), "l"),
    (("factor_subsample_image",), "d"),
    (("USE_CONSTANT_MAX_AMPLITUDE",), "l"),
    (("CONSTANT_MAX_AMPLITUDE_TO_USE",), "d"),
    (("USE_SNAPSHOT_NUMBER_IN_FILENAME",), "l"),
    (("DRAW_WATER_IN_BLUE",), "l"),
    (("US_LETTER",), "l"),
    (("POWER_DISPLAY_COLOR",), "d"),
    (("SU_FORMAT",), "l"),
    (("USER_T0",), "d"),
    (("time_stepping_scheme",), "i"),
    (("ADD_PERIODIC_CONDITIONS",), "l"),
    (("PERIODIC_HORIZ_DIST",), "d"),
    (("GPU_MODE",), "l"),
    (("setup_with_binary_database",), "i"),
    (("NSTEP", "DT"), "id"),
    (("NT_DUMP_ATTENUATION",), "i"),
    (("ACOUSTIC_FORCING",), "l"),
    (("NUMBER_OF_SIMULTANEOUS_RUNS",), "i"),
    (("BROADCAST_SAME_MESH_AND_MODEL",), "l"),
    (("ADD_RANDOM_PERTURBATION_TO_THE_MESH", "ADD_PERTURBATION_AROUND_SOURCE_ONLY"), "ll"),
)

_WIDTH = {"i": 4, "l": 4, "d": 8}
_FMT = {"i": "i", "l": "i", "d": "d"}
ISOTROPIC, ANISOTROPIC, POROELASTIC = 1, 2, 3

# defaults of the init block for write_database (a Par_file's usual values)
INIT_DEFAULTS = dict(title="sf2d-b200 mesh", NOISE_TOMOGRAPHY=0, UNDO_ATTENUATION_AND_OR_PML=False,
                     output_grid_Gnuplot=False, interpol=True, NTSTEP_BETWEEN_OUTPUT_INFO=100,
                     NTSTEP_BETWEEN_OUTPUT_SEISMOS=1000, NTSTEP_BETWEEN_OUTPUT_IMAGES=100,
                     PML_BOUNDARY_CONDITIONS=False, ROTATE_PML_ACTIVATE=False, ROTATE_PML_ANGLE=30.0,
                     K_MIN_PML=1.0, K_MAX_PML=1.0, damping_change_factor_acoustic=0.5,
                     damping_change_factor_elastic=1.0, PML_PARAMETER_ADJUSTMENT=False, read_external_mesh=False,
                     NELEM_PML_THICKNESS=3, NTSTEP_BETWEEN_OUTPUT_SAMPLE=1, imagetype_JPEG=3,
                     imagetype_wavefield_dumps=1, output_postscript_snapshot=False, output_color_image=False,
                     meshvect=True, modelvect=False, boundvect=True, cutsnaps=1.0, subsamp_postscript=1,
                     sizemax_arrows=1.0, anglerec=0.0, initialfield=False, add_Bielak_conditions_bottom=False,
                     add_Bielak_conditions_right=False, add_Bielak_conditions_top=False,
                     add_Bielak_conditions_left=False, seismotype="1", imagetype_postscript=1, MODEL="default",
                     SAVE_MODEL="default", TOMOGRAPHY_FILE="dummy", output_grid_ASCII=False, OUTPUT_ENERGY=False,
                     NTSTEP_BETWEEN_OUTPUT_ENERGY=10, output_wavefield_dumps=False,
                     use_binary_for_wavefield_dumps=False, ATTENUATION_VISCOELASTIC=False,
                     ATTENUATION_PORO_FLUID_PART=False, ATTENUATION_VISCOACOUSTIC=False, USE_SOLVOPT=False,
                     save_ASCII_seismograms=True, save_binary_seismograms_single=True,
                     save_binary_seismograms_double=False, USE_TRICK_FOR_BETTER_PRESSURE=False,
                     COMPUTE_INTEGRATED_ENERGY_FIELD=False, save_ASCII_kernels=True,
                     NTSTEP_BETWEEN_COMPUTE_KERNELS=1, APPROXIMATE_HESS_KL=False, NO_BACKWARD_RECONSTRUCTION=False,
                     DRAW_SOURCES_AND_RECEIVERS=True, Q0_poroelastic=1.0, freq0_poroelastic=10.0, AXISYM=False,
                     P_SV=True, factor_subsample_image=1.0, USE_CONSTANT_MAX_AMPLITUDE=False,
                     CONSTANT_MAX_AMPLITUDE_TO_USE=1.17e4, USE_SNAPSHOT_NUMBER_IN_FILENAME=False,
                     DRAW_WATER_IN_BLUE=True, US_LETTER=False, POWER_DISPLAY_COLOR=0.3, SU_FORMAT=False,
                     USER_T0=0.0, time_stepping_scheme=1, ADD_PERIODIC_CONDITIONS=False, PERIODIC_HORIZ_DIST=0.0,
                     GPU_MODE=True, setup_with_binary_database=0, NSTEP=1000, DT=1e-3, NT_DUMP_ATTENUATION=500,
                     ACOUSTIC_FORCING=False, NUMBER_OF_SIMULTANEOUS_RUNS=1, BROADCAST_SAME_MESH_AND_MODEL=True,
                     ADD_RANDOM_PERTURBATION_TO_THE_MESH=False, ADD_PERTURBATION_AROUND_SOURCE_ONLY=False)


class _Records:
    """Sequential reader of length-framed records."""

    def __init__(self, data: bytes, path: str):
        self.data, self.pos, self.path, self.count = data, 0, path, 0

    def next(self) -> bytes:
        if self.pos + 4 > len(self.data):
            raise ValueError(f"{self.path}: file ends before record {self.count + 1}")
        (n,) = struct.unpack_from("<i", self.data, self.pos)
        end = self.pos + 4 + n
        if n < 0 or end + 4 > len(self.data):
            raise ValueError(f"{self.path}: record {self.count + 1} has a bad length marker {n}")
        (n2,) = struct.unpack_from("<i", self.data, end)
        if n2 != n:
            raise ValueError(f"{self.path}: record {self.count + 1} markers disagree ({n} vs {n2})")
        rec = self.data[self.pos + 4:end]
        self.pos = end + 4
        self.count += 1
        return rec

    def fields(self, codes: str):
        """Decodes the next record; an 's' field takes the bytes the others leave."""
        rec = self.next()
        fixed = sum(_WIDTH[c] for c in codes if c != "s")
        if ("s" not in codes and len(rec) != fixed) or ("s" in codes and len(rec) < fixed):
            raise ValueError(f"{self.path}: record {self.count} holds {len(rec)} bytes, expected fields {codes!r}")
        out, o = [], 0
        for c in codes:
            if c == "s":
                w = len(rec) - fixed
                out.append(rec[o:o + w].decode("latin-1").rstrip(" \x00"))
                o += w
            else:
                (v,) = struct.unpack_from("<" + _FMT[c], rec, o)
                out.append(bool(v) if c == "l" else v)
                o += _WIDTH[c]
        return out

    def array(self, dtype, count: int):
        rec = self.next()
        a = np.frombuffer(rec, dtype=dtype)
        if a.size != count:
            raise ValueError(f"{self.path}: record {self.count} holds {a.size} values, expected {count}")
        return a


def read_database(path: str) -> dict:
    """Parses one Database<iproc>.bin into a dict of parameters and arrays (ids 1-based as in the file)."""
    with open(path, "rb") as f:
        R = _Records(f.read(), path)
    params = {}
    for names, codes in INIT_RECORDS:
        params.update(zip(names, R.fields(codes)))
    npgeo = params["npgeo"]
    coorg = np.zeros((npgeo, 2))
    seen = np.zeros(npgeo, dtype=bool)
    for _ in range(npgeo):
        ip, x, z = R.fields("idd")
        if not 1 <= ip <= npgeo:
            raise ValueError(f"{path}: control node {ip} outside 1..{npgeo}")
        coorg[ip - 1] = (x, z)
        seen[ip - 1] = True
    if not seen.all():
        raise ValueError(f"{path}: some control nodes have no coordinates")
    nbmodels, ngnod, nspec, pointsdisp, lowerleft = R.fields("iiiil")
    if nspec != params["nspec"]:
        raise ValueError(f"{path}: element counts disagree ({nspec} vs {params['nspec']})")
    counts = dict(zip(("nelemabs", "nelemacforcing", "nelem_acoustic_surface", "nedges_coupled",
                       "nedges_acporo_coupled", "nedges_elporo_coupled", "nnodes_tangential_curve",
                       "nelem_on_the_axis"), R.fields("iiiiiiii")))
    n_sls, f0_ref, read_at_f0 = R.fields("idl")
    params.update(NGNOD=ngnod, nbmodels=nbmodels, pointsdisp=pointsdisp, plot_lowerleft_corner_only=lowerleft,
                  N_SLS=n_sls, ATTENUATION_f0_REFERENCE=f0_ref, READ_VELOCITIES_AT_f0=read_at_f0, **counts)
    materials = []
    for _ in range(nbmodels):
        v = R.fields("ii" + "d" * 13)
        materials.append((v[0], v[1], tuple(v[2:])))
    knods = np.zeros((nspec, ngnod), dtype=np.int64)
    kmato = np.zeros(nspec, dtype=np.int64)
    pml = np.zeros(nspec, dtype=np.int64)
    for _ in range(nspec):
        v = R.fields("i" * (ngnod + 3))
        e = v[0]
        if not 1 <= e <= nspec:
            raise ValueError(f"{path}: element {e} outside 1..{nspec}")
        kmato[e - 1], knods[e - 1], pml[e - 1] = v[1], v[2:2 + ngnod], v[2 + ngnod]
    ninterface, _max_interfaces = R.fields("ii")
    if ninterface:
        raise NotImplementedError(f"{path}: a slice with MPI interfaces (one slice per run is supported)")
    # absorbing edges: anyabs = nelemabs > 0 (read_mesh_databases.F90:813-818)
    absorbing = [R.fields("illlli" + "i" * 8) for _ in range(counts["nelemabs"])]
    if params["ACOUSTIC_FORCING"]:
        raise NotImplementedError(f"{path}: acoustic forcing edges")
    free = np.array([R.fields("iiii") for _ in range(counts["nelem_acoustic_surface"])],
                    dtype=np.int64).reshape(-1, 4)
    coupled = np.array([R.fields("ii") for _ in range(counts["nedges_coupled"])], dtype=np.int64).reshape(-1, 2)
    for key in ("nedges_acporo_coupled", "nedges_elporo_coupled"):
        if counts[key]:
            raise NotImplementedError(f"{path}: poroelastic coupling edges")
    force_normal, rec_normal = R.fields("ll")
    if force_normal or rec_normal:
        for _ in range(counts["nnodes_tangential_curve"]):
            R.fields("dd")
    if counts["nelem_on_the_axis"]:
        raise NotImplementedError(f"{path}: axisymmetric elements")
    if R.pos != len(R.data):
        raise ValueError(f"{path}: {len(R.data) - R.pos} bytes after the last record")
    return dict(params=params, coorg=coorg, knods=knods, kmato=kmato, pml=pml, materials=materials,
                absorbing=absorbing, free_surface=free, coupled=coupled)


def material_rows(d: dict):
    """The material table as Par_file rows (index, kind, rho, vp, vs, 0, 0, Qkappa, Qmu) for isotropic
    and tomographic materials, (index, 2, rho, c11, c13, c15, c33, c35, c55, c12, c23, c25, c22, Qkappa,
    Qmu) for anisotropic ones (save_databases.f90:150-205)."""
    rows = []
    for (i, kind, v) in d["materials"]:
        if kind == ANISOTROPIC:
            row = [i, 2, *v[:11], v[11], v[12]]
        elif kind == POROELASTIC:
            raise NotImplementedError("poroelastic materials")
        else:
            row = [i, kind, v[0], v[1], v[2], 0, 0, v[5], v[6]]
        rows.append([repr(x) for x in row])  # Par_file tokens, exact
    return rows


def mesh_from_database(d: dict, fluid_materials=()) -> Mesh:
    """Mesh of a parsed database: control nodes, connectivity, absorbing edges
    (one per record, code from the codeabs flags: edge 1 bottom, 2 right, 3
    top, 4 left; corner flags as read_mesh_databases.F90:985-1030 sets them)
    and the listed free-surface edges of fluid elements (get_acoustic_edge,
    construct_acoustic_surface.f90:72-200)."""
    from .external_mesh import _free_range

    knods = d["knods"] - 1
    mesh = Mesh(nspec=len(knods), ngnod=int(d["params"]["NGNOD"]), knods=knods, coorg=d["coorg"].copy())
    isp, typ = [], []
    for rec in d["absorbing"]:
        e, flags = rec[0] - 1, rec[1:5]
        if sum(bool(f) for f in flags) != 1:
            raise ValueError("must have one and only one absorbing edge per absorbing line cited")
        isp.append(e)
        typ.append((IBOTTOM, IRIGHT, ITOP, ILEFT)[[bool(f) for f in flags].index(True)])
    mesh.abs_ispec = np.array(isp, dtype=np.int64)
    mesh.abs_type = np.array(typ, dtype=np.int64)
    mesh.abs_corner = absorbing_corners(mesh.abs_ispec, mesh.abs_type)
    fluid = set(int(m) for m in fluid_materials)
    free = []
    for (e1, nn, n1, n2) in d["free_surface"]:
        e = int(e1) - 1
        if int(d["kmato"][e]) not in fluid:
            continue
        free.append((e,) + _free_range(knods[e], int(nn), int(n1) - 1, int(n2) - 1))
    mesh.free_edges = np.array(free, dtype=np.int64).reshape(-1, 5)
    mesh.free_top = False
    mesh.absorb = (False, False, False, False)
    return mesh


def _pack(codes: str, values) -> bytes:
    out = b""
    for c, v in zip(codes, values):
        if c == "s":
            b = str(v).encode("latin-1")[:STRING_LEN]
            out += b + b" " * (STRING_LEN - len(b))
        else:
            out += struct.pack("<" + _FMT[c], int(v) if c in "il" else float(v))
    return out


def write_database(path: str, mesh: Mesh, kmato, materials, params: dict | None = None, pml=None,
                   coupled=None, free_edges=None) -> None:
    """Writes a one-slice Database in save_databases.f90's record order.

    `materials`: (index, kind, 13 values) as read_database returns them;
    `kmato`: 1-based material per element; absorbing edges from mesh.abs_ispec /
    abs_type (codeabs flags, type = edge code, full GLL ranges 1..5); free
    surface edges (element, imin, imax, jmin, jmax), default mesh.free_edges,
    written as their corner nodes; `coupled`: (fluid element, solid element)
    1-based pairs."""
    p = dict(INIT_DEFAULTS)
    p.update(params or {})
    p["nspec"], p["npgeo"], p["NPROC"] = mesh.nspec, len(mesh.coorg), 1
    recs = []
    for names, codes in INIT_RECORDS:
        recs.append(_pack(codes, [p[n] for n in names]))
    for ip, (x, z) in enumerate(mesh.coorg):
        recs.append(_pack("idd", (ip + 1, x, z)))
    nabs = 0 if mesh.abs_ispec is None else len(mesh.abs_ispec)
    free_edges = mesh.free_edges if free_edges is None else free_edges
    free = [] if free_edges is None else list(free_edges)
    coupled = np.zeros((0, 2), np.int64) if coupled is None else np.asarray(coupled)
    recs.append(_pack("iiiil", (len(materials), mesh.ngnod, mesh.nspec, p.get("pointsdisp", 6), False)))
    recs.append(_pack("iiiiiiii", (nabs, 0, len(free), len(coupled), 0, 0, 0, 0)))
    recs.append(_pack("idl", (p.get("N_SLS", 3), p.get("ATTENUATION_f0_REFERENCE", 5.196152422706633),
                              p.get("READ_VELOCITIES_AT_f0", False))))
    for (i, kind, vals) in materials:
        recs.append(_pack("ii" + "d" * 13, (i, kind, *vals)))
    pml = np.zeros(mesh.nspec, np.int64) if pml is None else pml
    for e in range(mesh.nspec):
        recs.append(_pack("i" * (mesh.ngnod + 3), (e + 1, kmato[e], *(mesh.knods[e] + 1), pml[e])))
    recs.append(_pack("ii", (0, 0)))
    if nabs:
        for e, t in zip(mesh.abs_ispec, mesh.abs_type):
            flags = [t == IBOTTOM, t == IRIGHT, t == ITOP, t == ILEFT]
            recs.append(_pack("illlli" + "i" * 8, (e + 1, *flags, t, 1, 5, 1, 5, 1, 5, 1, 5)))
    corner_of = {(0, 0): 0, (4, 0): 1, (4, 4): 2, (0, 4): 3}
    for (e, i0, i1, j0, j1) in free:
        a = mesh.knods[e][corner_of[(i0, j0)]] + 1
        if (i0, j0) == (i1, j1):
            recs.append(_pack("iiii", (e + 1, 1, a, -1)))
        else:
            recs.append(_pack("iiii", (e + 1, 2, a, mesh.knods[e][corner_of[(i1, j1)]] + 1)))
    for (ea, es) in coupled:
        recs.append(_pack("ii", (ea, es)))
    recs.append(_pack("ll", (False, False)))
    with open(path, "wb") as f:
        for r in recs:
            n = struct.pack("<i", len(r))
            f.write(n + r + n)
