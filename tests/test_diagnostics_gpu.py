"""GPU parity of the per-element diagnostics (GPU_FEM::get_stress / get_volume /
get_volume_diff / get_inverted, GPU_FEM.cu:20-107) and of the per-vertex VBD residual
(GPU_VBD_FEM::get_forces, GPU_VBD_FEM.cu:482-559) against the CPU oracle, evaluated at the
same positions."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import pair

pytestmark = pytest.mark.gpu

ELEMENTS = [O.TETRA, O.HEXA, O.TETRA10, O.TETRA20, O.HEXA27]


def _deformed(ctx, element, material=O.STABLE_NEOHOOKE, solver="vbd"):
    cells = (4, 2, 2) if element in (O.TETRA, O.HEXA, O.TETRA10) else (2, 1, 1)
    s, o32, o64, mesh = pair(ctx, element, cells=cells, material=material, solver=solver, young=3e4, iterations=5)
    for _ in range(3):
        s.step(1 / 60, 2)
    return s, o64, mesh


@pytest.mark.parametrize("element", ELEMENTS)
@pytest.mark.parametrize("material", [O.STABLE_NEOHOOKE, O.NEOHOOKE, O.STVK, O.HOOKE])
def test_element_data_matches_oracle(ctx, element, material):
    import octopusengine_b200 as ob
    s, o64, mesh = _deformed(ctx, element, material)
    p = s.get_position()
    assert np.abs(p - mesh["X"]).max() > 1e-3   # really deformed
    o64.set(0, p.astype(np.float64))             # the oracle evaluates at the product's positions
    kinds = (ob.capi.DIAG_STRESS, ob.capi.DIAG_VOLUME, ob.capi.DIAG_VOLUME_DIFF, ob.capi.DIAG_INVERTED,
             ob.capi.DIAG_STRESS_ACCUMULATED, ob.capi.DIAG_VOLUME_ACCUMULATED, ob.capi.DIAG_VOLUME_DIFF_ACCUMULATED)
    vol = o64.element_data(ob.capi.DIAG_VOLUME)
    for kind in kinds:
        got = s.element_data(kind).astype(np.float64)
        ref = o64.element_data(kind)
        if kind == ob.capi.DIAG_INVERTED:
            np.testing.assert_array_equal(got, ref)
            assert got.sum() == 0
        elif kind in (ob.capi.DIAG_VOLUME_DIFF, ob.capi.DIAG_VOLUME_DIFF_ACCUMULATED):
            assert np.abs(got - ref).max() <= 1e-6 * max(vol.max(), np.abs(ref).max())
        else:
            # both in FP64 at the same positions; the output is rounded to FP32
            assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max(), kind
    if element == O.TETRA:   # one quadrature point: nothing to accumulate
        np.testing.assert_array_equal(s.element_data(ob.capi.DIAG_STRESS_ACCUMULATED),
                                      s.element_data(ob.capi.DIAG_STRESS))
        np.testing.assert_array_equal(s.element_data(ob.capi.DIAG_VOLUME_ACCUMULATED),
                                      s.element_data(ob.capi.DIAG_VOLUME))


def test_volumes_sum_to_the_beam_volume_at_rest(ctx):
    import octopusengine_b200 as ob
    s, o32, o64, mesh = pair(ctx, O.HEXA27, cells=(2, 1, 1))
    vol = s.element_data(ob.capi.DIAG_VOLUME)
    assert abs(vol.sum() - 1.0 * 0.25 * 0.25) < 1e-6
    np.testing.assert_allclose(s.element_data(ob.capi.DIAG_VOLUME_DIFF), 0.0, atol=1e-8)
    # the rest state has no stress for the rest-stress-free materials with a single point
    s1, _, _, _ = pair(ctx, O.TETRA, cells=(2, 1, 1))
    np.testing.assert_allclose(s1.element_data(ob.capi.DIAG_STRESS), 0.0, atol=1e-6)


def test_inverted_flags_an_inverted_element(ctx):
    import octopusengine_b200 as ob
    s, o32, o64, mesh = pair(ctx, O.TETRA, cells=(2, 1, 1))
    X, T = mesh["X"].copy(), mesh["T"]
    # push node 3 of element 0 through the opposite face: that element (and maybe neighbours) inverts
    e = T[0]
    c = X[e[:3]].mean(axis=0)
    X[e[3]] = c - (X[e[3]] - c)
    s.set_position(X)
    o64.set(0, X.astype(np.float64))
    got = s.element_data(ob.capi.DIAG_INVERTED)
    ref = o64.element_data(ob.capi.DIAG_INVERTED)
    np.testing.assert_array_equal(got, ref)
    assert got[0] == 1


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10, O.HEXA27])
def test_vertex_residuals(ctx, element):
    cells = (4, 2, 2) if element != O.HEXA27 else (2, 1, 1)
    s, o32, o64, mesh = pair(ctx, element, cells=cells, iterations=4, damping=1e-3)
    # a perturbed state before the first step: last position and inertia target are the rest
    # pose in both, so the residual has identical inputs
    rng = np.random.default_rng(11)
    P = (mesh["X"] + rng.normal(0, 2e-3, mesh["X"].shape)).astype(np.float32)
    s.set_position(P)
    o64.set(0, P.astype(np.float64))
    dt = 1 / 120
    r = s.vertex_residuals(dt)
    ref = o64.forces(dt)
    assert np.abs(r - ref).max() <= 1e-4 * np.abs(ref).max()
    # after a step the fixed vertices are masked, and the vectors agree with the reduced norms
    s.step(1 / 60, 2)
    r = s.vertex_residuals(dt)
    assert np.all(r[mesh["fixed"]] == 0)
    norms = s.residual(dt)
    nr = np.linalg.norm(r.astype(np.float64), axis=1)
    assert abs(nr.sum() - norms[0]) <= 1e-5 * norms[0]
    assert abs(nr.max() - norms[1]) <= 1e-5 * norms[1]


def test_vertex_residuals_are_zero_for_other_solvers(ctx):
    s, o32, o64, mesh = pair(ctx, O.TETRA10, cells=(2, 1, 1), solver="xpbd")
    s.step(1 / 60, 2)
    assert not s.vertex_residuals(1 / 120).any()
