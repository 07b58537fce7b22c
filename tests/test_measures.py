"""Shape-function values (FEM_Shape::build_shape) and the accuracy measures of the reference's
experiments (MeshDiff / Beam_MSE_Sampling, octopus/include/Script/Measure/MeshDiff.h; flexion and
torsion error recorders, octopus/src/Script/Record/Recorder.cpp:190-330), on host arrays."""
import numpy as np
import pytest

import oracle_lib as O

ELEMENTS = [O.TETRA, O.HEXA, O.TETRA10, O.TETRA20, O.HEXA27]


@pytest.mark.parametrize("element", ELEMENTS)
def test_shape_values_interpolate_and_match_the_pinned_derivatives(built, element):
    from octopusengine_b200 import capi
    nodes = capi.reference_nodes(element)
    for j, x in enumerate(nodes):   # Kronecker property at the element's nodes
        N = capi.shape_values(element, x)
        np.testing.assert_allclose(N, np.eye(len(nodes))[j], atol=1e-12)
    coords, w, dN = O.shape(element)   # golden-pinned derivatives at the quadrature points
    h = 1e-6
    for q in range(len(w)):
        x = np.asarray(coords[q], float)
        assert abs(capi.shape_values(element, x).sum() - 1.0) < 1e-12   # partition of unity
        for k in range(3):
            e = np.zeros(3)
            e[k] = h
            fd = (capi.shape_values(element, x + e) - capi.shape_values(element, x - e)) / (2 * h)
            np.testing.assert_allclose(fd, dN[q][:, k], atol=1e-7)


def test_mesh_error_statistics(built):
    from octopusengine_b200 import capi
    rng = np.random.default_rng(1)
    a = rng.normal(size=(50, 3)).astype(np.float32)
    b = rng.normal(size=(50, 3)).astype(np.float32)
    off = np.array([0.1, -0.2, 0.3], np.float32)
    e = np.linalg.norm(a.astype(np.float64) - b - off, axis=1)
    r = capi.mesh_error(a, b, off)
    np.testing.assert_allclose([r["MSE"], r["RMSE"], r["MAE"], r["max"], r["L1"], r["L2"]],
                               [np.mean(e ** 2), np.sqrt(np.mean(e ** 2)), e.mean(), e.max(), e.sum(), (e ** 2).sum()],
                               rtol=1e-12)


def _beams(elements, cells=(4, 2, 2), size=(2.0, 1.0, 1.0)):
    from octopusengine_b200 import capi
    out = []
    for e in elements:
        X, T = capi.beam_mesh(e, cells, size)
        out.append((e, X, T))
    return out


def test_beam_sampling_compares_discretisations(built):
    from octopusengine_b200 import capi
    meshes = _beams([O.HEXA27, O.TETRA, O.HEXA, O.TETRA10])
    S = capi.BeamSampler(meshes, reference=0, nb_sample=4)
    assert S.n_samples == (4 * 2 + 1) * (4 + 1) * (4 + 1)
    # at rest every discretisation reproduces the samples
    for m, (e, X, T) in enumerate(meshes):
        assert S.error(m, X, meshes[0][1])["max"] < 1e-5
    # an affine deformation is reproduced by every element type
    A = np.array([[1.1, 0.2, 0.0], [0.0, 0.9, 0.1], [0.05, 0.0, 1.0]], np.float32)
    for m, (e, X, T) in enumerate(meshes):
        assert S.error(m, X @ A.T, meshes[0][1] @ A.T)["max"] < 1e-5
    # a quadratic bending field: the quadratic elements agree with Q2, the linear ones do not
    def bend(X):
        Y = X.copy()
        Y[:, 2] += 0.1 * X[:, 0] ** 2
        return Y
    err = {e: S.error(m, bend(X), bend(meshes[0][1]))["max"] for m, (e, X, T) in enumerate(meshes)}
    assert err[O.TETRA10] < 1e-5 and err[O.HEXA27] < 1e-5
    assert err[O.TETRA] > 1e-3 and err[O.HEXA] > 1e-3


def test_flexion_error(built):
    from octopusengine_b200 import capi
    X, T = capi.beam_mesh(O.TETRA, (4, 1, 1), (1.0, 0.25, 0.25))
    cur = X.copy()
    cur[:, 2] -= 0.1
    follow = X[-1]
    err, pid = capi.flexion_error(X, cur, follow, follow)
    assert pid == len(X) - 1 and abs(err - 0.01) < 1e-6


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10, O.HEXA27])
def test_torsion_profile_of_a_twisted_beam(built, element):
    from octopusengine_b200 import capi
    L = 2.0
    X, T = capi.beam_mesh(element, (8, 2, 2), (L, 1.0, 1.0))
    # rigid twist about the axis (y, z) = (0.5, 0.5): theta(x) = 30 deg * x / L
    th = np.radians(30.0) * X[:, 0] / L
    c, s = np.cos(th), np.sin(th)
    cur = X.copy()
    cur[:, 1] = 0.5 + c * (X[:, 1] - 0.5) - s * (X[:, 2] - 0.5)
    cur[:, 2] = 0.5 + s * (X[:, 1] - 0.5) + c * (X[:, 2] - 0.5)
    d, a = capi.torsion_profile(element, X, cur, T, 5, L)
    assert len(d) >= 9 and np.all(np.diff(d) > 0)
    # the linear elements interpolate the twist between nodes, the quadratic ones nearly exactly
    tol = 0.2 if element in (O.TETRA, O.HEXA) else 0.05
    np.testing.assert_allclose(a, 30.0 * d, atol=tol)
