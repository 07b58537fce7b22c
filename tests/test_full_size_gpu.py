"""Parity at the benchmark sizes and in the benchmarked precision, against the FP64 oracle.

* Config 2 at full size: the P2 beam of 64 x 16 x 16 cells (98,304 tet10, 140,481 nodes),
  E = 1e6, nu = 0.49, rho = 1100, x = 0 face fixed, v0 ~ N(0, 0.05) from the seed; one VBD
  sub-step of 1/300 s with 10 iterations, in the drop-in (plain) and the mixed precision; one
  XPBD frame of 5 sub-steps; 10 explicit steps of 1e-5 s.
* Config 3 at 16^3 cells: the 1 m cube of P3 (117,649 nodes) and of Q2 (35,937 nodes) with a
  per-element Young modulus log-uniform in [1e4, 1e6], bottom fixed, top moved down by the
  first of 50 increments of 20 %; one frame of 2 sub-steps x 10 iterations.
* Config 4 sample: 9 scenes of the benchmark's own 256-scene draw (the first three of each
  element type with at most 40,000 nodes), batched in mixed precision with the autotuned lane
  mapping, one 1/240 s sub-step of 20 iterations.

Every error is the max-norm position error relative to the max-norm displacement of the FP64
oracle over the step (`disp_err`), the scale on which a step's motion is resolved.  The bar is
the FP32 oracle's own error on the same step: the FP32 drop-in may not exceed a small multiple
of it, and the mixed precision (compensated sums, FP64 for ill-conditioned solves) may not
exceed it."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import disp_err

pytestmark = pytest.mark.gpu

ORACLE_FLOOR = 2e-6   # below this both errors are at the FP32 rounding of the positions


@pytest.fixture(scope="module", autouse=True)
def oracle_threads():
    O.set_threads()
    yield
    O.set_threads(1)


def _oracle_pair(element, X, T, m, colors, **kw):
    n_colors = int(colors.max()) + 1
    out = []
    for fp64 in (False, True):
        sc = O.Scene(element, X, T, m, colors=colors, n_colors=n_colors, in_place=True, **kw)
        out.append((O.Solver("vbd", sc, fp64=fp64), sc))
    return out


def _check(name, errs, e32):
    print("%s: fp32 oracle %.3e, %s" % (name, e32, ", ".join("%s %.3e" % kv for kv in errs.items())))
    assert errs["plain"] <= 3.0 * e32 + ORACLE_FLOOR, (name, errs, e32)
    if "mixed" in errs:
        assert errs["mixed"] <= 1.0 * e32 + ORACLE_FLOOR, (name, errs, e32)


def test_config2_full_size_one_substep(ctx):
    import octopusengine_b200 as ob
    X, T = ob.beam_mesh(ob.TETRA10, (64, 16, 16), (4.0, 1.0, 1.0))
    assert len(X) == 140481 and len(T) == 98304
    fixed = ob.fixed_by_plane(X, (0.01, 0.0, 0.0), (-1.0, 0.0, 0.0))
    m = ob.lumped_masses(ob.TETRA10, X, T, 1100.0, ob.MASS_FEMSHAPE)
    v0 = np.random.default_rng(2024).normal(0, 0.05, X.shape).astype(np.float32)
    common = dict(material=ob.STABLE_NEOHOOKE, young=1e6, poisson=0.49, gravity=(0.0, 0.0, -9.81), iterations=10)
    dt = 1.0 / 300.0
    got = {}
    colors = None
    for name, prec in (("plain", ob.PREC_PLAIN), ("mixed", ob.PREC_MIXED)):
        s = ob.Scene(ctx, ob.TETRA10, X, T, masses=m, fixed_ids=fixed, initial_velocity=v0, precision=prec, **common)
        colors = s.coloring()[0]
        s.step(dt, 1)
        got[name] = s.get_position()
        s.close()
    (o32, k32), (o64, k64) = _oracle_pair(O.TETRA10, X, T, m, colors, fixed=fixed, v0=v0, **common)
    o32.step(dt, 1)
    o64.step(dt, 1)
    ref = o64.get(0)
    _check("config 2 (140,481 nodes)", {k: disp_err(p, ref, X) for k, p in got.items()}, disp_err(o32.get(0), ref, X))


def _cube(element, n, seed=5):
    import octopusengine_b200 as ob
    X, T = ob.beam_mesh(element, (n, n, n), (1.0, 1.0, 1.0))
    E = np.exp(np.random.default_rng(seed).uniform(np.log(1e4), np.log(1e6), len(T))).astype(np.float32)
    bottom = np.nonzero(X[:, 2] < 1e-6)[0]
    top = np.nonzero(X[:, 2] > 1.0 - 1e-6)[0]
    fixed = np.concatenate([bottom, top]).astype(np.int32)
    group = np.concatenate([np.zeros(len(bottom)), np.ones(len(top))]).astype(np.int32)
    order = np.argsort(fixed, kind="stable")
    return X, T, E, fixed[order], group[order]


@pytest.mark.parametrize("element,nodes", [(O.TETRA20, 117649), (O.HEXA27, 35937)])
def test_config3_cube_16_one_frame(ctx, element, nodes):
    import octopusengine_b200 as ob
    X, T, E, fixed, group = _cube(element, 16)
    assert len(X) == nodes
    m = ob.lumped_masses(element, X, T, 1000.0, ob.MASS_FEMSHAPE)
    common = dict(young=1e5, young_per_element=E, poisson=0.45, gravity=(0.0, 0.0, -9.81), iterations=10)
    off = (0.0, 0.0, -0.2 / 50)
    got = {}
    colors = None
    for name, prec in (("plain", ob.PREC_PLAIN), ("mixed", ob.PREC_MIXED)):
        s = ob.Scene(ctx, element, X, T, masses=m, fixed_ids=fixed, fixed_group=group, precision=prec, **common)
        colors = s.coloring()[0]
        s.set_fixation(off, group=1)
        s.step(1 / 60, 2)
        got[name] = s.get_position()
        s.close()
    (o32, k32), (o64, k64) = _oracle_pair(element, X, T, m, colors, fixed=fixed, fixed_group=group, **common)
    for o in (o32, o64):
        o.set_fixation(off, group=1)
        o.step(1 / 60, 2)
    ref = o64.get(0)
    _check("config 3 %s 16^3" % {O.TETRA20: "P3", O.HEXA27: "Q2"}[element],
           {k: disp_err(p, ref, X) for k, p in got.items()}, disp_err(o32.get(0), ref, X))


def test_config4_sample_batched_mixed_autotuned(ctx):
    import bench
    import octopusengine_b200 as ob
    specs, iterations, substeps, frame_dt = bench.workload_specs("batched", 2024)
    chosen, per_type = [], {}
    for sp in specs:
        X, T = ob.beam_mesh(sp["element"], sp["cells"], sp["size"])
        if len(X) <= 40000 and per_type.get(sp["element"], 0) < 3:
            per_type[sp["element"]] = per_type.get(sp["element"], 0) + 1
            chosen.append((sp, X, T))
    assert sorted(per_type.values()) == [3, 3, 3]
    dt = frame_dt / substeps
    scenes, meshes = [], []
    for sp, X, T in chosen:
        fixed = ob.fixed_by_plane(X, (0.01, 0.0, 0.0), (-1.0, 0.0, 0.0))
        m = ob.lumped_masses(sp["element"], X, T, sp["density"], ob.MASS_FEMSHAPE)
        kw = dict(material=ob.STABLE_NEOHOOKE, young=sp["young"], poisson=sp["poisson"], gravity=(0.0, 0.0, -9.81),
                  iterations=iterations)
        scenes.append(ob.Scene(ctx, sp["element"], X, T, masses=m, fixed_ids=fixed, precision=ob.PREC_MIXED, **kw))
        meshes.append((sp["element"], X, T, m, fixed, kw))
    mapping = ob.autotune_mapping(ctx, scenes, dt, 2)
    assert set(mapping) == {ob.TETRA, ob.TETRA10, ob.HEXA}
    b = ob.Batch(ctx, scenes)
    b.step(dt, 1)
    assert (b.status() == 0).all()
    for s, (e, X, T, m, fixed, kw) in zip(scenes, meshes):
        (o32, k32), (o64, k64) = _oracle_pair(e, X, T, m, s.coloring()[0], fixed=fixed, **kw)
        o32.step(dt, 1)
        o64.step(dt, 1)
        ref = o64.get(0)
        e32 = disp_err(o32.get(0), ref, X)
        got = disp_err(s.get_position(), ref, X)
        print("config 4 scene e%d n%d mapping %d: mixed %.3e, fp32 oracle %.3e" % (e, len(X), s.mapping(), got, e32))
        assert got <= 1.0 * e32 + ORACLE_FLOOR, (e, len(X), got, e32)
    b.close()


@pytest.mark.parametrize("solver", ["xpbd", "explicit"])
def test_config2_full_size_xpbd_and_explicit(ctx, solver):
    """Config 2's other two solvers at full size (98,304 P2 elements, 140,481 nodes): one XPBD
    frame of 5 sub-steps (1/60 s, the reference default OptiShared form), or 10 explicit
    symplectic-Euler steps of 1e-5 s, against the FP64 oracle with the FP32 oracle's error as
    the bar."""
    import octopusengine_b200 as ob
    X, T = ob.beam_mesh(ob.TETRA10, (64, 16, 16), (4.0, 1.0, 1.0))
    fixed = ob.fixed_by_plane(X, (0.01, 0.0, 0.0), (-1.0, 0.0, 0.0))
    m = ob.lumped_masses(ob.TETRA10, X, T, 1100.0, ob.MASS_FEMSHAPE)
    v0 = np.random.default_rng(2024).normal(0, 0.05, X.shape).astype(np.float32)
    kind = {"xpbd": ob.SOLVER_XPBD, "explicit": ob.SOLVER_EXPLICIT}[solver]
    frame, n = (1.0 / 60.0, 5) if solver == "xpbd" else (1e-4, 10)
    s = ob.Scene(ctx, ob.TETRA10, X, T, solver=kind, masses=m, fixed_ids=fixed, initial_velocity=v0,
                 material=ob.STABLE_NEOHOOKE, young=1e6, poisson=0.49, gravity=(0.0, 0.0, -9.81))
    s.step(frame, n)
    got = s.get_position()
    s.close()
    out = []
    for fp64 in (False, True):
        sc = O.Scene(O.TETRA10, X, T, m, material=O.STABLE_NEOHOOKE, young=1e6, poisson=0.49,
                     gravity=(0.0, 0.0, -9.81), fixed=fixed, v0=v0)
        o = O.Solver(solver, sc, fp64=fp64)
        o.step(frame, n)
        out.append(o.get(0))
    e = disp_err(got, out[1], X)
    e32 = disp_err(out[0], out[1], X)
    print("config 2 %s: product %.3e, fp32 oracle %.3e" % (solver, e, e32))
    assert e <= 3.0 * e32 + ORACLE_FLOOR, (solver, e, e32)
