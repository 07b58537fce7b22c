"""Shared scene builders for the parity tests: the same mesh, masses, fixed nodes and
colouring go to the CUDA product (through the C ABI) and to the CPU oracle."""
import numpy as np

import oracle_lib as O

# Beam fixed at x = 0 as the reference scenes do: Plane(0.01 x^, -x^) (BaseScene.h:164-170).
PLANE = ((0.01, 0.0, 0.0), (-1.0, 0.0, 0.0))


def make_mesh(element, cells, size, offset=(0.0, 0.0, 0.0)):
    X, T = O.beam_mesh(element, cells, size, offset)
    return X, T


def pair(ctx, element, cells=(4, 2, 2), size=(1.0, 0.25, 0.25), material=O.STABLE_NEOHOOKE, young=1e5,
         poisson=0.45, density=1000.0, gravity=(0.0, 0.0, -9.81), iterations=10, damping=0.0, v0=None,
         solver="vbd", precision=0, tpv=0, version=2, target=-1, rho=0.0, young_per_element=None, box=None,
         global_damping=0.0, color_algo=0, fixed=None, xpbd_version=2):
    """Returns (product Scene, oracle fp32 solver, oracle fp64 solver, mesh dict)."""
    import octopusengine_b200 as ob
    X, T = make_mesh(element, cells, size)
    m = O.masses(element, X, T, density, 1)
    if fixed is None:
        fixed = O.fixed_by_plane(X, *PLANE)
    kind = {"vbd": ob.SOLVER_VBD, "xpbd": ob.SOLVER_XPBD, "explicit": ob.SOLVER_EXPLICIT}[solver]
    kw = dict(solver=kind, masses=m, material=material, young=young, poisson=poisson, damping=damping,
              gravity=gravity, fixed_ids=fixed, iterations=iterations, precision=precision,
              threads_per_vertex=tpv, vbd_version=version, target_color=target, rho=rho, color_algo=color_algo,
              global_damping=global_damping, xpbd_version=xpbd_version)
    if v0 is not None:
        kw["initial_velocity"] = v0
    if young_per_element is not None:
        kw["young_per_element"] = young_per_element
    if box is not None:
        kw.update(box_limit=1, box_min=box[0], box_max=box[1])
    scene = ob.Scene(ctx, element, X, T, **kw)
    colors, n_colors = None, 0
    in_place = True
    if solver == "vbd":
        colors, n_colors = O.colour(element, T, len(X), color_algo, target if version == 3 else -1)
        in_place = O.conflicts(element, T, len(X), colors) == 0
    okw = dict(material=material, young=young, poisson=poisson, damping=damping, gravity=gravity, fixed=fixed,
               v0=v0, iterations=iterations, rho=rho, in_place=in_place, colors=colors, n_colors=n_colors,
               young_per_element=young_per_element, box=box, global_damping=global_damping, xpbd_version=xpbd_version)
    s32 = O.Scene(element, X, T, m, **okw)
    s64 = O.Scene(element, X, T, m, **okw)
    o32 = O.Solver(solver, s32, fp64=False)
    o64 = O.Solver(solver, s64, fp64=True)
    return scene, o32, o64, dict(X=X, T=T, m=m, fixed=fixed, colors=colors, n_colors=n_colors, keep=(s32, s64))


def rel_err(a, b):
    """max-norm error relative to the max-norm of the reference positions."""
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(b).max(), 1e-30))


def disp_err(a, b, X):
    """max-norm error relative to the max-norm of the reference displacement."""
    d = np.asarray(b) - X
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(np.abs(d).max(), 1e-30))


def check_parity(p, o32, o64, X, label="", factor=3.0):
    """The parity bar of the GPU tests, on both scales: positions within 1e-5 of the position
    magnitude against the FP64 oracle, and the error relative to the step's displacement at
    most `factor` times the FP32 oracle's own (plus the FP32 rounding of the positions, which
    bounds what any FP32 state can resolve).  Returns (product error, FP32 oracle error) on the
    displacement scale."""
    ref = o64.get(0)
    assert rel_err(p, ref) < 1e-5, (label, rel_err(p, ref))
    d = np.abs(np.asarray(ref) - X).max()
    floor = 2.0 * np.finfo(np.float32).eps * np.abs(ref).max() / max(d, 1e-30)
    e = disp_err(p, ref, X)
    e32 = disp_err(o32.get(0), ref, X)
    assert e <= factor * e32 + floor, (label, e, e32, floor)
    return e, e32
