"""CPU checks of the oracle's XPBD restatement: the polar decomposition behind the corotated
constraints (mat3x3_polardecomposition, CUMatrix.cu:75-96), the constraint gradients of every
material pair against finite differences of C (eval_material, GPU_PBD_FEM_Materials.cu:97-117),
and the algebraic equivalence of the normalised V0 update (GPU_PBD_FEM.cu:13-93) with the raw
V1/V2 update (:141-263) on a scene without fixed nodes."""
import numpy as np
import pytest

import oracle_lib as O


def _rot(rng, angle=0.6):
    """Rotation by a random axis and the given angle (Rodrigues)."""
    a = rng.normal(size=3)
    a /= np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * K @ K


def _rodrigues(a, angle):
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(angle) * K + (1 - np.cos(angle)) * K @ K


@pytest.mark.parametrize("angle", [0.05, 0.6, 1.5, 2.5])
def test_polar_of_a_rotation_follows_the_iteration(angle):
    """For F a rotation by theta about a, every iterate is a rotation about a; with residual
    angle psi the step is |omega| = 2 sin(psi) (1/|1 + 2 cos(psi)| + 1e-9), ten steps at most,
    stopping below 1e-8: a closed-form known answer for the iteration."""
    rng = np.random.default_rng(int(angle * 100))
    a = rng.normal(size=3)
    a /= np.linalg.norm(a)
    F = _rodrigues(a, angle)
    phi = 0.0
    for _ in range(10):
        psi = angle - phi
        w = 2 * np.sin(psi) * (1 / abs(1 + 2 * np.cos(psi)) + 1e-9)
        if abs(w) < 1e-8:
            break
        phi += w
    R, S = O.polar(F, fp64=True)
    np.testing.assert_allclose(R, _rodrigues(a, phi), atol=1e-12)
    np.testing.assert_allclose(R @ S, F, atol=1e-12)


@pytest.mark.parametrize("seed", range(5))
def test_polar_decomposition(seed):
    rng = np.random.default_rng(seed)
    Q = _rot(rng)
    A = rng.normal(size=(3, 3)) * 0.2
    Ssym = np.eye(3) + 0.5 * (A + A.T)   # symmetric positive definite stretch
    F = Q @ Ssym
    R, S = O.polar(F, fp64=True)
    np.testing.assert_allclose(R.T @ R, np.eye(3), atol=1e-10)
    assert np.linalg.det(R) > 0
    np.testing.assert_allclose(R @ S, F, atol=1e-10)
    # ten iterations bring R most of the way to Q (the reference stops there)
    assert np.abs(R - Q).max() < 0.05 * np.abs(np.eye(3) - Q).max()
    Rf, _ = O.polar(F, fp64=False)
    np.testing.assert_allclose(Rf, R, atol=2e-6)
    # symmetric F: the iteration does not move off the identity
    R2, S2 = O.polar(Ssym)
    np.testing.assert_array_equal(R2, np.eye(3))


def test_polar_of_identity_is_identity():
    R, S = O.polar(np.eye(3))
    np.testing.assert_array_equal(R, np.eye(3))
    np.testing.assert_array_equal(S, np.eye(3))


# P is the gradient of C for every pair except the three where the reference's P is not dC/dF
# (Corotated first: C = tr((S - I)^2) but P = 2 tr(S - I) R; Corotated second: P = R(2S - I);
# FixedCorotated second: P = 4R(S - I)); those are pinned by their formulas only.
@pytest.mark.parametrize("material,m", [(0, 0), (0, 1), (1, 0), (1, 1), (2, 0), (2, 1), (3, 0), (3, 1),
                                        (5, 0)])
def test_xpbd_pair_gradient(material, m):
    rng = np.random.default_rng(material * 2 + m)
    A = 0.1 * rng.normal(size=(3, 3))
    # corotated pairs at a symmetric stretch, where the polar rotation is exactly I
    F = np.eye(3) + (0.5 * (A + A.T) if material >= 4 else A)
    lam, mu = 2.0, 0.7
    P, c = O.xpbd_pair(material, m, lam, mu, F)
    h = 1e-6
    G = np.zeros((3, 3))
    for i in range(3):
        for j in range(3):
            Fp, Fm = F.copy(), F.copy()
            Fp[i, j] += h
            Fm[i, j] -= h
            G[i, j] = (O.xpbd_pair(material, m, lam, mu, Fp)[1] - O.xpbd_pair(material, m, lam, mu, Fm)[1]) / (2 * h)
    np.testing.assert_allclose(P, G, rtol=1e-5, atol=1e-6 * max(1.0, np.abs(G).max()))


def test_corotated_pairs_vanish_at_rest_rotation():
    rng = np.random.default_rng(3)
    R = _rot(rng, 0.05)
    for mat in (4, 5):
        P, c = O.xpbd_pair(mat, 0, 1.0, 1.0, R)
        assert abs(c) < 1e-10 and np.abs(P).max() < 1e-5


@pytest.mark.parametrize("element", [O.TETRA10, O.HEXA])
def test_v0_and_raw_update_agree_without_fixed_nodes(element):
    X, T = O.beam_mesh(element, (3, 2, 2), (1.0, 0.3, 0.3))
    m = O.masses(element, X, T, 1000.0, 1)
    rng = np.random.default_rng(1)
    v0 = rng.normal(0, 0.3, size=X.shape).astype(np.float32)
    res = {}
    for ver in (O.XPBD_V0, O.XPBD_OPTISHARED, O.XPBD_QUADRATURE):
        sc = O.Scene(element, X, T, m, young=1e5, poisson=0.3, v0=v0, xpbd_version=ver, gravity=(0, 0, 0))
        so = O.Solver("xpbd", sc, fp64=True)
        for _ in range(3):
            so.step(1 / 60, 4)
        res[ver] = so.get(0)
    assert np.abs(res[O.XPBD_V0] - X).max() > 1e-3   # the scene really deformed
    np.testing.assert_allclose(res[O.XPBD_OPTISHARED], res[O.XPBD_V0], atol=1e-9)
    np.testing.assert_array_equal(res[O.XPBD_QUADRATURE], res[O.XPBD_OPTISHARED])


def test_optigroup_projects_only_tetra4():
    for element, moves in ((O.TETRA, True), (O.TETRA10, False)):
        X, T = O.beam_mesh(element, (3, 2, 2), (1.0, 0.3, 0.3))
        m = O.masses(element, X, T, 1000.0, 1)
        out = []
        for ver in (O.XPBD_OPTIGROUP,):
            sc = O.Scene(element, X, T, m, young=1e5, xpbd_version=ver, gravity=(0, 0, -9.81))
            so = O.Solver("xpbd", sc)
            so.step(1 / 60, 2)
            out.append(so.get(0))
        # without projection every node falls freely: z = -g t^2 summed over the sub-steps
        free_fall = np.allclose(out[0][:, 2] - X[:, 2], out[0][0, 2] - X[0, 2])
        assert free_fall != moves
