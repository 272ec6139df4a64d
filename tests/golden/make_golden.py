"""Generate the golden fixtures in this directory from the reference tree.

Run from the repository root, in a container where the reference is mounted:

    python tests/golden/make_golden.py /root/reference [example name ...]

For each pinned example it writes ``<name>.json`` (the parsed Par_file
subset, SOURCE and interfaces needed to rebuild the run, plus the source and
receiver locations the reference printed in REF_SEIS/output.log),
``<name>_seis.npz`` (the REF_SEIS seismogram values as float64, with the
first time sample and the time step of the trace) and, for a tomographic
model, ``<name>_tomo.npz`` (the gridded model the example's script writes) and,
for an external mesh, ``<name>_mesh.npz`` (the tables of its MESH/ text files).
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from specfem2d_b200.setup.from_par_file import config_from_data_dir  # noqa: E402

EXAMPLES = {
    # name: (example dir, list of (station, component) traces, Par_file name, SOURCE name)
    "tromp2005_kernel": ("EXAMPLES/Tromp2005_kernel", [("S0001", "BXX"), ("S0001", "BXZ")], "Par_file", "SOURCE"),
    "anisotropic_isotropic_model": ("EXAMPLES/anisotropic_isotropic_model", [("S0001", "BXX"), ("S0001", "BXZ")],
                                    "Par_file", "SOURCE"),
    # REF_SEIS of this example was made with the "shared_by_four_elements" variant
    # (its output.log locates the source at x = z = 1000 m)
    "attenuation_viscoelastic": ("EXAMPLES/attenuation/viscoelastic", [("S0001", "BXX"), ("S0001", "BXZ")],
                                 "Par_file_attenuation_2D_source_in_point_shared_by_four_elements",
                                 "SOURCE_attenuation_2D_source_in_point_shared_by_four_elements"),
    # fluid layer (tomographic acoustic model) over an elastic layer: coupling, acoustic Stacey,
    # acoustic free surface, displacement receivers in both domains
    "tomographic_ocean_model": ("EXAMPLES/tomographic_ocean_model",
                                [(f"S{k:04d}", c) for k in (1, 3, 6, 9, 12, 14, 16, 18, 20, 22) for c in ("BXX", "BXZ")],
                                "Par_file", "SOURCE"),
}

EXAMPLES["semi_infinite_homogeneous"] = (
    # elastic half space with CPML layers (3 elements) on all four sides
    "EXAMPLES/semi_infinite_homogeneous", [("S0001", "BXX"), ("S0001", "BXZ")], "Par_file", "SOURCE")

EXAMPLES["pressure_source_acoustic"] = (
    # fluid only, CPML on all sides, Gaussian pressure source with USE_TRICK_FOR_BETTER_PRESSURE
    "EXAMPLES/check_absolute_amplitude_of_pressure_source_seismograms_acoustic", [("S0001", "PRE")],
    "../REF_SEIS/Par_file", "../REF_SEIS/SOURCE")

EXAMPLES["force_source_elastic"] = (
    # elastic medium with 3-element CPML, vertical force at a corner shared by four elements
    "EXAMPLES/check_absolute_amplitude_of_force_source_seismograms_elastic", [("S0001", "BXX"), ("S0001", "BXZ")],
    "../REF_SEIS/Par_file", "../REF_SEIS/SOURCE")

EXAMPLES["moment_tensor_dip_slip"] = (
    # moment-tensor source (vertical dip slip) in an elastic medium with 3-element CPML
    "EXAMPLES/infinite_homogeneous_moment_tensor_vertical_dip_slip", [("S0001", "BXX"), ("S0001", "BXZ")],
    "Par_file", "SOURCE")

EXAMPLES["topography_fluid_layer"] = (
    # 9-node elements (curved topography), fluid layer, 3-element CPML; the reference
    # stored the traces of the first of its two receiver lines (11 stations)
    "EXAMPLES/simple_topography_and_also_a_simple_fluid_layer",
    [(f"S{k:04d}", c) for k in range(1, 12) for c in ("BXX", "BXZ")], "Par_file", "SOURCE")

EXAMPLES["initial_mode_lddrk"] = (
    # fluid-only 2 km x 2 km square (50 x 50 elements, no absorbing terms), LDDRK, initial
    # potential = the (2, 3) membrane mode of prepare_initial_field.F90, one receiver
    "EXAMPLES/initial_mode_LDDRK", [("S0001", "BXX"), ("S0001", "BXZ")], "Par_file", "SOURCE")

EXAMPLES["gmsh_stacey_external"] = (
    # external (Gmsh) mesh of 2942 9-node fluid elements with a circular inclusion, Stacey on
    # three sides, a listed free surface; 11 pressure stations.  The reference ran it on 4 MPI
    # slices (its output.log numbers elements per slice); Par_file.serial is the same run on one
    "EXAMPLES/Gmsh_example_Stacey_MPI", [(f"S{k:04d}", "PRE") for k in range(1, 12)], "Par_file.serial", "SOURCE")

# examples whose TOMOGRAPHY_FILE is written by a script of the reference
TOMO_SCRIPTS = {"tomographic_ocean_model": "utils/createTomographyFile.py"}


def tomography_grid(ref_root, script):
    """Run the reference's tomography-file script (its plotting calls go to a
    stub) in a scratch directory and parse the file it writes."""
    import tempfile
    import types

    from specfem2d_b200.setup.tomography import read_tomo_file

    stub = types.ModuleType("matplotlib")
    stub.pyplot = types.SimpleNamespace(**{k: (lambda *a, **kw: None) for k in
                                           ("clf", "title", "plot", "savefig", "show", "xlabel", "ylabel")})
    saved = {k: sys.modules.get(k) for k in ("matplotlib", "matplotlib.pyplot")}
    sys.modules["matplotlib"], sys.modules["matplotlib.pyplot"] = stub, stub.pyplot
    cwd, argv = os.getcwd(), sys.argv
    try:
        with tempfile.TemporaryDirectory(dir=HERE) as tmp:
            os.chdir(tmp)
            path = os.path.join(ref_root, script)
            sys.argv = [path]
            code = compile(open(path).read(), path, "exec")
            exec(code, {"__name__": "__main__"})
            return read_tomo_file(os.path.join(tmp, "profile.xyz"))
    finally:
        os.chdir(cwd)
        sys.argv = argv
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v


def log_locations(path):
    """(element, xi, gamma) triples printed by locate_source / locate_receivers."""
    out = []
    elem = None
    with open(path) as f:
        for ln in f:
            m = re.search(r"in element\s+(\d+)", ln)
            if m:
                elem = int(m.group(1))
            m = re.search(r"at xi,gamma coordinates =\s+(\S+)\s+(\S+)", ln)
            if m and elem is not None:
                out.append([elem, float(m.group(1)), float(m.group(2))])
                elem = None
    return out


def kernel_log_values(path):
    """Numbers printed by the adjoint-source tool and the kernel run in
    REF_KERNEL/output.log: the cross-correlation norm per component, the
    adjoint sources' min/max as read by the solver, the elastic kernels'
    maxima (save_adjoint_kernels.f90:202-216) and, after "Acoustic kernels:",
    the fluid kernels' maxima (save_adjoint_kernels.f90:453-460)."""
    out = {"norm": [], "kernel_max": {}}
    keys = {"rho  kernel": "rho", "kappa kernel": "kappa", "mu kernel": "mu", "rho prime kernel": "rhop",
            "alpha kernel": "alpha", "beta kernel": "beta"}
    ac_keys = {"rho kernel": "rho", "kappa kernel": "kappa", "rho prime kernel": "rhop", "alpha kernel": "alpha"}
    with open(path) as f:
        section = "elastic"
        for ln in f:
            if "Acoustic kernels:" in ln:
                section = "acoustic"
            elif "Elastic kernels:" in ln:
                section = "elastic"
            if section == "acoustic":
                for k, v in ac_keys.items():
                    m = re.search(r"maximum value of " + k + r"\s*=\s*(\S+)", ln)
                    if m:
                        out.setdefault("acoustic_kernel_max", {})[v] = float(m.group(1))
                continue
            m = re.match(r"\s*Norm =\s+(\S+)", ln)
            if m:
                out["norm"].append(float(m.group(1)))
            m = re.search(r"adjoint sources min/max\s*=\s*(\S+)\s+(\S+)", ln)
            if m:
                out["adj_min_max"] = [float(m.group(1)), float(m.group(2))]
            for k, v in keys.items():
                m = re.search(r"maximum value of " + k + r"\s*=\s*(\S+)", ln)
                if m:
                    out["kernel_max"][v] = float(m.group(1))
    return out


# adjoint (SIMULATION_TYPE = 3) run of an example: its REF_KERNEL traces (the
# adjoint wavefield at the adjoint station) and the numbers of its log
KERNEL_RUNS = {"tromp2005_kernel": ("EXAMPLES/Tromp2005_kernel", [("S0001", "BXX"), ("S0001", "BXZ")])}


# kernel examples without REF_SEIS: (example dir, Par_file, station, component).  Their
# REF_KERNEL holds the adjoint source the example's tool made from the forward trace
# (the forward trace, zeroed after its window), the adjoint run's trace at the
# station and the log of both runs
KERNEL_ONLY = {"luoyang_fluid_solid_kernel": ("EXAMPLES/LuoYang_fluid_solid_kernel", "Par_file", "S0001", "POT")}


def kernel_only(ref_root, name):
    rel, par_file, st, comp = KERNEL_ONLY[name]
    ex = os.path.join(ref_root, rel)
    kdir = os.path.join(ex, "REF_KERNEL")
    cfg = config_from_data_dir(os.path.join(ex, "DATA"), par_file, "SOURCE")
    cfg["log_locations"] = log_locations(os.path.join(kdir, "output.log"))
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(cfg, f, indent=1, default=str)
    ext = "semx" if comp == "POT" else ("semp" if comp == "PRE" else "semd")
    adj = np.loadtxt(os.path.join(kdir, f"AA.{st}.{comp}.adj"))
    trace = np.loadtxt(os.path.join(kdir, f"AA.{st}.{comp}.{ext}"))
    np.savez_compressed(os.path.join(HERE, name + "_adjoint.npz"), t=adj[:, 0], adj_source=adj[:, 1],
                        t_adjoint=trace[:, 0], adjoint_trace=trace[:, 1])
    with open(os.path.join(HERE, name + "_adjoint.json"), "w") as f:
        json.dump(kernel_log_values(os.path.join(kdir, "output.log")), f, indent=1)


def main(ref_root, names=None):
    """Write the fixtures of `names` (all examples when None)."""
    for name in KERNEL_ONLY:
        if not names or name in names:
            kernel_only(ref_root, name)
            print("wrote", name)
    for name, (rel, traces, par_file, source_file) in EXAMPLES.items():
        if names and name not in names:
            continue
        ex = os.path.join(ref_root, rel)
        cfg = config_from_data_dir(os.path.join(ex, "DATA"), par_file, source_file)
        cfg["log_locations"] = log_locations(os.path.join(ex, "REF_SEIS", "output.log"))
        ext = cfg.pop("external_mesh", None)
        if ext is not None:
            # the mesh files' tables, ids as in the files
            np.savez_compressed(os.path.join(HERE, name + "_mesh.npz"), **ext)
        with open(os.path.join(HERE, name + ".json"), "w") as f:
            json.dump(cfg, f, indent=1, default=str)
        arrs = {}
        for st, comp in traces:
            ext = "semp" if comp == "PRE" else "semd"
            d = np.loadtxt(os.path.join(ex, "REF_SEIS", f"AA.{st}.{comp}.{ext}"))
            arrs[f"{st}_{comp}"] = d[:, 1]
            arrs["t_first"] = np.array(d[0, 0])
            arrs["t_step"] = np.array(d[1, 0] - d[0, 0])
        np.savez_compressed(os.path.join(HERE, name + "_seis.npz"), **arrs)
        if name in KERNEL_RUNS:
            rel_k, ktraces = KERNEL_RUNS[name]
            kdir = os.path.join(ref_root, rel_k, "REF_KERNEL")
            # sample times of the forward traces as the adjoint-source tool reads them
            karr = {"t_forward": np.loadtxt(os.path.join(ex, "REF_SEIS", f"AA.{ktraces[0][0]}.{ktraces[0][1]}.semd"))[:, 0]}
            for st, comp in ktraces:
                d = np.loadtxt(os.path.join(kdir, f"AA.{st}.{comp}.semd"))
                karr[f"{st}_{comp}"] = d[:, 1]
            np.savez_compressed(os.path.join(HERE, name + "_adjoint.npz"), **karr)
            with open(os.path.join(HERE, name + "_adjoint.json"), "w") as f:
                json.dump(kernel_log_values(os.path.join(kdir, "output.log")), f, indent=1)
        if name in TOMO_SCRIPTS:
            x, z, vp, vs, rho = tomography_grid(ref_root, TOMO_SCRIPTS[name])
            np.savez_compressed(os.path.join(HERE, name + "_tomo.npz"), x=x, z=z, vp=vp, vs=vs, rho=rho)
        print("wrote", name)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference root> [example name ...]")
    main(sys.argv[1], sys.argv[2:] or None)
