"""The algebraic identities the colour kernels rely on instead of the reference's literal
contraction, checked in FP64 on the host against the shape tables (which are pinned to the
reference's FEM_Shape.h by test_host.py) — no GPU.

* Q1: Jx_q = sum_i u_i (x) dN_qi equals the kernel's form from the seven monomial
  coefficients of the trilinear field (butterflies over nodes i / i + 4 and (0, 3) / (1, 2) of
  each face), evaluated at the Gauss point signs / sqrt(3).
* P1 compact owner entry: with the vertex's own node r first and G_j = JX_inv^T dN_j of the
  other three, F = I + sum_j (u_j - u_r) (x) G_j and g_r = -sum_j G_j, which equal
  F = I + Jx JX_inv and g_r = JX_inv^T dN_r (GPU_VBD_FEM.cu compute_f_H_sym) since
  sum_i dN_i = 0.
"""
import numpy as np

from octopusengine_b200 import capi

HEX_SIGNS = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                      [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)


def hex_coefficients(u):
    """The kernel's butterfly (hex_q1_coefficients): a_x, a_y, a_z, a_xy, a_xz, a_yz, a_xyz."""
    p = u[4:8] + u[0:4]
    m = u[4:8] - u[0:4]
    pe0, po0, pe1, po1 = p[0] + p[3], p[3] - p[0], p[1] + p[2], p[2] - p[1]
    me0, mo0, me1, mo1 = m[0] + m[3], m[3] - m[0], m[1] + m[2], m[2] - m[1]
    s = 0.125
    return dict(x=(pe1 - pe0) * s, y=(po1 + po0) * s, xy=(po1 - po0) * s, z=(me1 + me0) * s,
                xz=(me1 - me0) * s, yz=(mo1 + mo0) * s, xyz=(mo1 - mo0) * s)


def test_hexa8_node_signs_and_gauss_points_match_the_shape_table(built):
    np.testing.assert_array_equal(capi.reference_nodes(capi.HEXA), HEX_SIGNS)
    qp, w, _ = capi.shape_table(capi.HEXA)
    np.testing.assert_allclose(qp, HEX_SIGNS / np.sqrt(3.0), rtol=0, atol=1e-15)


def test_q1_jacobian_from_monomial_coefficients(built):
    _, _, dN = capi.shape_table(capi.HEXA)   # (8 points, 8 nodes, 3)
    rng = np.random.default_rng(7)
    for _ in range(20):
        u = rng.normal(size=(8, 3))
        h = hex_coefficients(u)
        for q in range(8):
            xi, et, ze = HEX_SIGNS[q] / np.sqrt(3.0)
            J0 = h["x"] + h["xy"] * et + h["xz"] * ze + h["xyz"] * (et * ze)
            J1 = h["y"] + h["xy"] * xi + h["yz"] * ze + h["xyz"] * (xi * ze)
            J2 = h["z"] + h["xz"] * xi + h["yz"] * et + h["xyz"] * (xi * et)
            direct = np.einsum("ic,ik->kc", u, dN[q])   # row k: Jx column k = sum_i u_i dN_qi[k]
            np.testing.assert_allclose(np.stack([J0, J1, J2]), direct, rtol=1e-12, atol=1e-12)


def test_p1_compact_entry_gives_the_same_f_and_g(built):
    _, _, dN = capi.shape_table(capi.TETRA)   # (1, 4, 3)
    dN = dN[0]
    rng = np.random.default_rng(11)
    for _ in range(20):
        X = rng.normal(size=(4, 3))
        J = np.einsum("ic,ik->ck", X, dN)        # J[row, col] = sum_i X_i[row] dN_i[col]
        Jinv = np.linalg.inv(J)
        u = 0.05 * rng.normal(size=(4, 3))
        F_ref = np.eye(3) + np.einsum("ic,ik->ck", u, dN) @ Jinv
        for r in range(4):
            others = [i for i in range(4) if i != r]
            G = [Jinv.T @ dN[j] for j in others]
            F = np.eye(3) + sum(np.outer(u[j] - u[r], Gj) for j, Gj in zip(others, G))
            np.testing.assert_allclose(F, F_ref, rtol=1e-12, atol=1e-12)
            np.testing.assert_allclose(-(G[0] + G[1] + G[2]), Jinv.T @ dN[r], rtol=1e-12, atol=1e-12)
