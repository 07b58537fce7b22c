"""Pins the CPU oracle to the reference: shape tables against the expressions in the
reference's FEM_Shape.h, and beam meshes + lumped masses against the meshes the reference
itself wrote (assets/result/vtk/References).  Fixtures: tests/golden/make_golden.py."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle_lib as O

HERE = os.path.dirname(os.path.abspath(__file__))
SHAPES = json.load(open(os.path.join(HERE, "golden", "shapes.json")))
MESHES = json.load(open(os.path.join(HERE, "golden", "meshes.json")))
ELEM = {"Tetra": O.TETRA, "Hexa": O.HEXA, "Tetra10": O.TETRA10, "Tetra20": O.TETRA20, "Hexa27": O.HEXA27}


@pytest.mark.parametrize("name", sorted(ELEM))
def test_shape_tables_match_reference(name):
    q, w, d = O.shape(ELEM[name])
    g = SHAPES[name]
    np.testing.assert_allclose(q, np.array(g["quadrature"]), rtol=0, atol=1e-15)
    np.testing.assert_allclose(w, np.array(g["weights"]), rtol=1e-14, atol=0)
    np.testing.assert_allclose(d, np.array(g["dN"]), rtol=0, atol=1e-13)


@pytest.mark.parametrize("name", sorted(ELEM))
def test_shape_kats(name):
    """Partition of unity (sum_i dN_i = 0) and quadrature weights summing to the reference volume."""
    q, w, d = O.shape(ELEM[name])
    assert np.abs(d.sum(axis=1)).max() < 1e-12
    vol = 1.0 / 6.0 if name.startswith("Tetra") else 8.0
    assert abs(w.sum() - vol) < 1e-12


@pytest.mark.parametrize("name", sorted(MESHES))
def test_beam_mesh_and_masses_match_reference_output(name):
    g = MESHES[name]
    X, T = O.beam_mesh(ELEM[name], g["cells"], g["size"], offset=g["origin"])
    assert len(X) == g["n_points"] and len(T) == g["n_elements"]
    assert hashlib.sha256(T.astype("<i4").tobytes()).hexdigest() == g["topology_sha256"]
    assert T.ravel()[: len(g["topology_head"])].tolist() == g["topology_head"]
    np.testing.assert_allclose(X[:: g["point_stride"]], np.array(g["points_sample"]), rtol=0, atol=1e-6)
    m = O.masses(ELEM[name], X, T, g["density"], 1)
    # the VTK file prints 6 significant digits
    np.testing.assert_allclose(m[:: g["point_stride"]], np.array(g["mass_sample"]), rtol=1e-5)
    assert abs(m.sum() - g["mass_sum"]) / g["mass_sum"] < 1e-5


def test_dsat_is_a_proper_colouring_and_reduction_creates_conflicts():
    X, T = O.beam_mesh(O.TETRA10, (4, 2, 2), (1, 0.25, 0.25))
    c, n = O.colour(O.TETRA10, T, len(X), 0)
    assert O.conflicts(O.TETRA10, T, len(X), c) == 0
    for t in T:   # no element holds two nodes of one colour
        assert len(set(c[t])) == len(t)
    r, nr = O.colour(O.TETRA10, T, len(X), 0, target=n - 3)
    assert nr == n - 3 and r.max() < nr
    assert O.conflicts(O.TETRA10, T, len(X), r) > 0


def test_oracle_fp32_close_to_fp64_on_config1():
    X, T = O.beam_mesh(O.TETRA, (8, 2, 2), (1.0, 0.25, 0.25))
    m = O.masses(O.TETRA, X, T, 1000.0, 1)
    fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
    c, n = O.colour(O.TETRA, T, len(X), 0)
    res = []
    for fp64 in (False, True):
        s = O.Scene(O.TETRA, X, T, m, young=1e5, poisson=0.45, fixed=fixed, iterations=20, colors=c, n_colors=n)
        v = O.Solver("vbd", s, fp64=fp64)
        for _ in range(10):
            v.step(0.01, 1)
        res.append(v.get(0))
    assert np.abs(res[0] - res[1]).max() / np.abs(res[1]).max() < 1e-5


def test_cpu_reference_vbd_tracks_gpu_semantics():
    """The CPU Gauss-Seidel path (timed baseline) and the GPU-semantics oracle converge to
    the same motion on config 1 (different sweep orders, so not bit-equal)."""
    X, T = O.beam_mesh(O.TETRA, (8, 2, 2), (1.0, 0.25, 0.25))
    m = O.masses(O.TETRA, X, T, 1000.0, 1)
    fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
    c, n = O.colour(O.TETRA, T, len(X), 0)
    s = O.Scene(O.TETRA, X, T, m, young=1e5, poisson=0.45, fixed=fixed, iterations=20, colors=c, n_colors=n)
    gpu_like = O.Solver("vbd", s, fp64=True)
    cpu = O.CpuVBD(s)
    for _ in range(20):
        gpu_like.step(0.01, 1)
        cpu.step(0.01, 1)
    a, b = gpu_like.get(0), cpu.get(0)
    assert np.abs(a - b).max() < 2e-3
