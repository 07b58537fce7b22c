"""Oracle (test infrastructure only): numpy restatement of the reference's accuracy measures, used
by the tests as the checker of the product's host measures (octopusengine_b200/csrc/measure.cpp).
Nothing in the product imports this file.

  error_stats      Error::update over a set of error vectors (MeshDiff.h:9-25)
  mesh_diff_mse    MeshDiff_MSE::get_error with MeshDiff::late_init's initial offset
                   (MeshDiff.h:30-40,64-83)
  torsion_profile  FEM_Torsion_error_recorder::init + compute_errors
                   (octopus/src/Script/Record/Recorder.cpp:222-309) for Tetra4 and Hexa8, with
                   Tetra_4 / Hexa_8 ::build_shape and ::get_vertices (FEM_Shape.h:49-55,182-224)

The reference computes in FP32 (glm); this restatement evaluates the same formulas in FP64.
"""
import numpy as np

TETRA, HEXA = 3, 6


def error_stats(e):
    """MSE, RMSE, MAE, max, L1, L2 of the error vectors e (n x 3), as Error::update accumulates them."""
    e = np.asarray(e, np.float64)
    d = np.linalg.norm(e, axis=1)
    n = len(d)
    L1, L2 = float(d.sum()), float((d * d).sum())
    return {"MSE": L2 / n, "RMSE": np.sqrt(L2 / n), "MAE": L1 / n, "max": float(d.max()), "L1": L1, "L2": L2}


def mesh_diff_mse(ref_positions, ref_rest0, positions, rest0):
    """Error of a mesh against the reference mesh, node by node: e_i = r_i - p_i - offset with
    offset = (reference rest node 0) - (mesh rest node 0), taken once at late_init."""
    off = np.asarray(ref_rest0, np.float64) - np.asarray(rest0, np.float64)
    return error_stats(np.asarray(ref_positions, np.float64) - np.asarray(positions, np.float64) - off)


def _shape(element, r):
    s, t, l = r
    if element == TETRA:
        return np.array([1 - s - t - l, s, t, l])
    a = 1.0 / 8.0
    return a * np.array([(1 - s) * (1 - t) * (1 - l), (1 + s) * (1 - t) * (1 - l), (1 + s) * (1 + t) * (1 - l),
                         (1 - s) * (1 + t) * (1 - l), (1 - s) * (1 - t) * (1 + l), (1 + s) * (1 - t) * (1 + l),
                         (1 + s) * (1 + t) * (1 + l), (1 - s) * (1 + t) * (1 + l)])


def _vertices(element):
    if element == TETRA:
        return np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float64)
    return np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                     [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], np.float64)


def torsion_profile(element, rest, current, T, samples_per_edge, beam_length):
    """(distance, angle) samples along the beam's y = z = 0 edge.

    init: every element with two corners on that edge (rest y, z < 1e-6) gets samples_per_edge
    reference points spread from the first such corner to the second.  compute_errors: each
    sample interpolated in the rest state (p) and the current state (p0); its angle in degrees
    between the two directions from the section centre (0.5, 0.5) in the y-z plane, its
    distance p0.x / beam_length; sorted by distance, samples closer than 1e-4 merged with their
    angles averaged.  (In the reference the variable named init_positions holds the current
    positions and positions the rest ones; the formulas are restated with their roles.)"""
    rest = np.asarray(rest, np.float64)
    cur = np.asarray(current, np.float64)
    T = np.asarray(T)
    verts = _vertices(element)
    n_lin = 4 if element == TETRA else 8
    dist, ang = [], []
    for el in T:
        edge = [j for j in range(n_lin) if rest[el[j], 1] < 1e-6 and rest[el[j], 2] < 1e-6]
        if len(edge) < 2:
            continue
        a, b = verts[edge[0]], verts[edge[1]]
        for j in range(samples_per_edge):
            t = j / (samples_per_edge - 1)
            w = _shape(element, a + t * (b - a))
            p = w @ rest[el[:len(w)]]
            p0 = w @ cur[el[:len(w)]]
            di = p0[1:] - 0.5
            di = di / np.linalg.norm(di)
            dc = p[1:] - 0.5
            dc = dc / np.linalg.norm(dc)
            angle = abs(np.arctan2(dc[0] * di[1] - dc[1] * di[0], dc[0] * di[0] + dc[1] * di[1]))
            dist.append(p0[0] / beam_length)
            ang.append(np.degrees(angle))
    order = np.argsort(dist, kind="stable")
    dist = list(np.asarray(dist)[order])
    ang = list(np.asarray(ang)[order])
    out_d, out_a = [], []
    i = 0
    while i < len(dist):
        j, acc = 1, ang[i]
        while i + j < len(dist) and abs(dist[i] - dist[i + j]) < 1e-4:
            acc += ang[i + j]
            j += 1
        out_a.append(acc / j)
        out_d.append(dist[i])
        i += j
    return np.array(out_d), np.array(out_a)
