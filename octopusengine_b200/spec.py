"""Declarative scene specs: a small JSON-able dict that maps one to one onto the reference's
constructor enums (Element, Material, Mass_Distribution, VBD_Version, XPBD_FEM_VERSION) and
the scene description, standing in for the reference's hard-coded SimulationArgs
(octopus/include/Scene/BaseScene.h:34-51).

    {"element": "Tetra10", "beam": {"cells": [64, 16, 16], "size": [4, 1, 1]},
     "material": "Stable_NeoHooke", "young": 1e6, "poisson": 0.49, "density": 1100,
     "mass_distribution": "FemShape", "solver": "VBD", "iterations": 10,
     "fixed": {"plane": {"origin": [0.01, 0, 0], "normal": [-1, 0, 0]}},
     "gravity": [0, 0, -9.81], "frame": {"dt": 0.0166667, "substeps": 5}}
"""
import json

import numpy as np

from . import capi

ELEMENTS = {"Tetra": capi.TETRA, "Hexa": capi.HEXA, "Tetra10": capi.TETRA10, "Tetra20": capi.TETRA20,
            "Hexa27": capi.HEXA27}
MATERIALS = {"Hooke": capi.HOOKE, "StVK": capi.STVK, "NeoHooke": capi.NEOHOOKE, "Stable_NeoHooke": capi.STABLE_NEOHOOKE,
             "Corotated": capi.COROTATED, "FixedCorotated": capi.FIXED_COROTATED}
MASS = {"Uniform": capi.MASS_UNIFORM, "FemShape": capi.MASS_FEMSHAPE}
SOLVERS = {"VBD": capi.SOLVER_VBD, "XPBD": capi.SOLVER_XPBD, "Explicit": capi.SOLVER_EXPLICIT}
VBD_VERSIONS = {"Base": capi.VBD_BASE, "Threaded_Quadrature": capi.VBD_THREADED_QUADRATURE,
                "Reduction_Symmetry": capi.VBD_REDUCTION_SYMMETRY, "Better_Coloration": capi.VBD_BETTER_COLORATION}
XPBD_VERSIONS = {"XPBD": capi.XPBD_XPBD, "Quadrature": capi.XPBD_QUADRATURE, "OptiShared": capi.XPBD_OPTISHARED,
                 "OptiGroup": capi.XPBD_OPTIGROUP}
PRECISIONS = {"plain": capi.PREC_PLAIN, "mixed": capi.PREC_MIXED}

# The benchmark configurations as specs (seeded parts — per-element Young moduli, initial
# velocities — are drawn by the caller from the spec's "seed").
CONFIGS = {
    "config1": {"element": "Tetra", "beam": {"cells": [8, 2, 2], "size": [1.0, 0.25, 0.25]},
                "material": "Stable_NeoHooke", "young": 1e5, "poisson": 0.45, "density": 1000.0,
                "mass_distribution": "FemShape", "solver": "VBD", "iterations": 20,
                "fixed": {"plane": {"origin": [0.01, 0, 0], "normal": [-1, 0, 0]}}, "gravity": [0, 0, -9.81],
                "frame": {"dt": 0.01, "substeps": 1}},
    "config2": {"element": "Tetra10", "beam": {"cells": [64, 16, 16], "size": [4.0, 1.0, 1.0]},
                "material": "Stable_NeoHooke", "young": 1e6, "poisson": 0.49, "density": 1100.0,
                "mass_distribution": "FemShape", "solver": "VBD", "iterations": 10,
                "fixed": {"plane": {"origin": [0.01, 0, 0], "normal": [-1, 0, 0]}}, "gravity": [0, 0, -9.81],
                "frame": {"dt": 1.0 / 60.0, "substeps": 5}, "initial_velocity_sigma": 0.05, "seed": 2024},
}


def _enum(table, value, what):
    if isinstance(value, int):
        return value
    if value not in table:
        raise ValueError("unknown %s %r (one of %s)" % (what, value, ", ".join(table)))
    return table[value]


def mesh_and_kwargs(spec):
    """(element, X, T, Scene keyword arguments) of a spec; no GPU needed."""
    spec = dict(spec)
    element = _enum(ELEMENTS, spec["element"], "element")
    if "beam" in spec:
        b = spec["beam"]
        X, T = capi.beam_mesh(element, b["cells"], b["size"], b.get("offset", (0.0, 0.0, 0.0)))
    else:
        X = np.asarray(spec["positions"], np.float32).reshape(-1, 3)
        T = np.asarray(spec["topology"], np.int32).reshape(-1, capi.ELEMENT_NODES[element])
    kw = dict(solver=_enum(SOLVERS, spec.get("solver", "VBD"), "solver"),
              material=_enum(MATERIALS, spec.get("material", "Stable_NeoHooke"), "material"),
              young=float(spec.get("young", 1e6)), poisson=float(spec.get("poisson", 0.45)),
              density=float(spec.get("density", 1000.0)),
              mass_distribution=_enum(MASS, spec.get("mass_distribution", "FemShape"), "mass distribution"),
              damping=float(spec.get("damping", 0.0)), iterations=int(spec.get("iterations", 1)),
              rho=float(spec.get("rho", 0.0)), gravity=tuple(spec.get("gravity", (0.0, -9.81, 0.0))),
              vbd_version=_enum(VBD_VERSIONS, spec.get("vbd_version", "Reduction_Symmetry"), "VBD version"),
              target_color=int(spec.get("target_color", -1)),
              xpbd_version=_enum(XPBD_VERSIONS, spec.get("xpbd_version", "OptiShared"), "XPBD version"),
              global_damping=float(spec.get("global_damping", 0.0)),
              precision=_enum(PRECISIONS, spec.get("precision", "plain"), "precision"),
              mg_linear=float(spec.get("mg_linear", 0.0)))
    fixed = spec.get("fixed")
    if fixed and "plane" in fixed:
        kw["fixed_ids"] = capi.fixed_by_plane(X, fixed["plane"]["origin"], fixed["plane"]["normal"])
    elif fixed and "ids" in fixed:
        kw["fixed_ids"] = np.asarray(fixed["ids"], np.int32)
    if spec.get("young_per_element") is not None:
        kw["young_per_element"] = np.asarray(spec["young_per_element"], np.float32)
    if spec.get("initial_velocity_sigma"):
        rng = np.random.default_rng(int(spec.get("seed", 0)))
        kw["initial_velocity"] = rng.normal(0.0, float(spec["initial_velocity_sigma"]), X.shape).astype(np.float32)
    if "box" in spec:
        kw.update(box_limit=1, box_min=tuple(spec["box"][0]), box_max=tuple(spec["box"][1]))
    return element, X, T, kw


def load(path_or_name):
    """A spec from a JSON file, or one of CONFIGS by name."""
    if path_or_name in CONFIGS:
        return dict(CONFIGS[path_or_name])
    with open(path_or_name) as f:
        return json.load(f)


def scene(ctx, spec):
    """Builds the Scene a spec describes; returns (scene, frame dt, sub-steps)."""
    from . import Scene
    element, X, T, kw = mesh_and_kwargs(spec)
    frame = spec.get("frame", {})
    return Scene(ctx, element, X, T, **kw), float(frame.get("dt", 1.0 / 60.0)), int(frame.get("substeps", 1))
