"""GPU parity of the XPBD coloured element projection and of the explicit integrator
against the CPU oracle (GPU_PBD + kernel_XPBD_V0/V1/V2 and GPU_SemiExplicit +
kernel_fem_eval_force semantics)."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import check_parity, pair, rel_err

pytestmark = pytest.mark.gpu


XPBD_MATERIALS = [O.STABLE_NEOHOOKE, O.NEOHOOKE, O.STVK, O.HOOKE, O.COROTATED, O.FIXED_COROTATED]


def s_rest(s):
    import ctypes as C
    from octopusengine_b200 import capi
    X = np.zeros((s.n_nodes, 3), np.float32)
    capi.check(capi.lib().oct_scene_get_rest_positions(s.handle, capi.ptr(X, C.c_float)), "rest positions")
    return X


def _run_xpbd(s, o32, o64, frames):
    """Steps product and oracles together.  After the first frame the product matches the FP32
    oracle within 1e-5; against FP64 it is never worse than twice the FP32 oracle's own error
    (XPBD in FP32 drifts from FP64 over frames whatever the summation order)."""
    for k in range(frames):
        s.step(1 / 60, 5)
        o32.step(1 / 60, 5)
        o64.step(1 / 60, 5)
        p = s.get_position()
        if k == 0:
            assert rel_err(p, o32.get(0)) < 1e-5
            check_parity(p, o32, o64, s_rest(s), "xpbd first frame")
        ref32 = rel_err(o32.get(0), o64.get(0))
        e64 = rel_err(p, o64.get(0))
        assert e64 < max(1e-5, 2.0 * ref32), (k, e64, ref32)
    return p


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10, O.TETRA20, O.HEXA27])
@pytest.mark.parametrize("material", XPBD_MATERIALS)
def test_xpbd_parity(ctx, element, material):
    """Reference default version (OptiShared: V0 for Tetra4, the raw V2 update otherwise)."""
    cells = (4, 2, 2) if element in (O.TETRA, O.HEXA, O.TETRA10) else (2, 1, 1)
    s, o32, o64, mesh = pair(ctx, element, cells=cells, material=material, solver="xpbd", young=1e5,
                             global_damping=0.5)
    _run_xpbd(s, o32, o64, 3)
    assert np.isfinite(s.get_velocity()).all()


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10])
@pytest.mark.parametrize("version", [O.XPBD_V0, O.XPBD_QUADRATURE, O.XPBD_OPTISHARED, O.XPBD_OPTIGROUP])
def test_xpbd_versions(ctx, element, version):
    s, o32, o64, mesh = pair(ctx, element, cells=(4, 2, 2), solver="xpbd", young=1e5, xpbd_version=version)
    p = _run_xpbd(s, o32, o64, 3)
    free = np.setdiff1d(np.arange(len(p)), mesh["fixed"])
    sag = np.abs(p[free, 2] - mesh["X"][free, 2]).max()
    if version == O.XPBD_OPTIGROUP and element != O.TETRA:
        # no projection: every free node falls freely
        assert np.allclose(p[free, 2] - mesh["X"][free, 2], p[free[0], 2] - mesh["X"][free[0], 2], atol=1e-6)
    else:
        assert sag > 0   # constrained motion


@pytest.mark.parametrize("solver", ["vbd", "explicit"])
def test_corotated_materials_are_xpbd_only(ctx, solver):
    import octopusengine_b200 as ob
    X, T = O.beam_mesh(O.TETRA, (2, 1, 1), (1, 0.5, 0.5))
    kind = {"vbd": ob.SOLVER_VBD, "explicit": ob.SOLVER_EXPLICIT}[solver]
    with pytest.raises(ob.OctError) as e:
        ob.Scene(ctx, O.TETRA, X, T, solver=kind, material=ob.COROTATED)
    assert e.value.status == 6   # OCT_ENOTSUP


def test_xpbd_element_colouring_matches_reference_order(ctx):
    import octopusengine_b200 as ob
    X, T = O.beam_mesh(O.TETRA10, (4, 2, 2), (1, 0.25, 0.25))
    c1, n1 = O.colour(O.TETRA10, T, len(X), 2)
    c2, n2, _ = ob.color(O.TETRA10, T, len(X), 2)
    assert n1 == n2 and np.array_equal(c1, c2)


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10, O.TETRA20, O.HEXA27])
def test_explicit_parity(ctx, element):
    cells = (3, 2, 2) if element in (O.TETRA20, O.HEXA27) else (4, 2, 2)
    s, o32, o64, mesh = pair(ctx, element, cells=cells, solver="explicit", young=1e5, damping=1e-4)
    for _ in range(5):
        s.step(1e-3, 20)
        o32.step(1e-3, 20)
        o64.step(1e-3, 20)
    assert rel_err(s.get_position(), o32.get(0)) < 1e-5
    check_parity(s.get_position(), o32, o64, mesh["X"], ("explicit", element))
    v = s.get_velocity()
    assert np.abs(v - o32.get(1)).max() < 1e-3 * max(1.0, np.abs(o32.get(1)).max())


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10, O.TETRA20, O.HEXA27])
@pytest.mark.parametrize("material", [O.HOOKE, O.STVK, O.NEOHOOKE, O.STABLE_NEOHOOKE])
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("damping", [0.0, 1e-3])
def test_explicit_force_pass_materials(ctx, element, material, precision, damping):
    """The element-centric explicit force pass (each element's stress once per point, its
    per-node contributions summed per node in owner order) for every material, without damping
    (P~ = V P JX_inv^T once per point) and with damping acting on an initial velocity (the
    k_d H v term), on distorted, non-affine elements."""
    import octopusengine_b200 as ob
    cells = (2, 1, 1) if element in (O.TETRA20, O.HEXA27) else (3, 2, 1)
    X, T = O.beam_mesh(element, cells, (0.6, 0.3, 0.2))
    X = (X + np.random.default_rng(4).uniform(-0.005, 0.005, X.shape)).astype(np.float32)
    m = O.masses(element, X, T, 1000.0, 1)
    fixed = O.fixed_by_plane(X, (0.02, 0, 0), (-1, 0, 0))
    v0 = np.random.default_rng(9).normal(0, 0.05, X.shape).astype(np.float32)
    kw = dict(material=material, young=1e5, poisson=0.4, damping=damping, gravity=(0.0, 0.0, -9.81))
    s = ob.Scene(ctx, element, X, T, solver=ob.SOLVER_EXPLICIT, masses=m, fixed_ids=fixed, initial_velocity=v0,
                 precision=precision, **kw)
    okw = dict(fixed=fixed, v0=v0, colors=None, n_colors=0, in_place=True, **kw)
    o32 = O.Solver("explicit", O.Scene(element, X, T, m, **okw), fp64=False)
    o64 = O.Solver("explicit", O.Scene(element, X, T, m, **okw), fp64=True)
    for _ in range(4):
        s.step(2e-4, 10)
        o32.step(2e-4, 10)
        o64.step(2e-4, 10)
    check_parity(s.get_position(), o32, o64, X, ("explicit", element, material, precision))
    ref_v = o64.get(1)
    assert np.abs(s.get_velocity() - ref_v).max() < 1e-3 * max(1.0, np.abs(ref_v).max())
    s.close()


@pytest.mark.parametrize("solver", ["vbd", "xpbd", "explicit"])
def test_frame_graph_replays_the_same_launches(ctx, solver):
    """oct_scene_set_capture: replayed frames equal frames launched one kernel at a time."""
    rng = np.random.default_rng(4)
    X, T = O.beam_mesh(O.TETRA10, (3, 2, 2), (1.0, 0.25, 0.25))
    v0 = rng.normal(0, 0.05, size=X.shape).astype(np.float32)
    a, _, _, mesh = pair(ctx, O.TETRA10, cells=(3, 2, 2), solver=solver, young=1e5, v0=v0, damping=1e-4)
    b, _, _, _ = pair(ctx, O.TETRA10, cells=(3, 2, 2), solver=solver, young=1e5, v0=v0, damping=1e-4)
    b.set_capture(True)
    dt, n = (1e-3, 10) if solver == "explicit" else (1 / 60, 4)
    for k in range(4):
        if k == 2:
            n += 1   # a new (dt, substeps) recaptures
        a.step(dt, n)
        b.step(dt, n)
        np.testing.assert_array_equal(a.get_position(), b.get_position())
    np.testing.assert_array_equal(a.get_velocity(), b.get_velocity())
    assert np.abs(a.get_position() - mesh["X"]).max() > 0
