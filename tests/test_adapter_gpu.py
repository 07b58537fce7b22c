"""The reference-shaped C++ adapters (include/octopus_b200.hpp: GPU_ParticleSystem, GPU_VBD,
GPU_VBD_FEM, GPU_Fix_Constraint, compute_fem_mass) drive the same C ABI and reproduce the
Python-path and oracle results on config 1."""
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as O
from scenes import rel_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _compile(tmp_path, name="adapter_demo"):
    exe = str(tmp_path / name)
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", name + ".cpp"),
                           "-L", os.path.join(ROOT, "octopusengine_b200"), "-loctb",
                           "-Wl,-rpath," + os.path.join(ROOT, "octopusengine_b200"), "-o", exe])
    return exe


def test_adapter_compiles(built, tmp_path):
    assert os.path.exists(_compile(tmp_path))
    assert os.path.exists(_compile(tmp_path, "adapter_controller"))


@pytest.mark.gpu
def test_adapter_matches_oracle(built, tmp_path):
    exe = _compile(tmp_path)
    run = subprocess.run([exe, "5"], text=True, capture_output=True, check=True)
    out = run.stdout
    diag = dict(zip(run.stderr.split()[::2], map(float, run.stderr.split()[1::2])))
    assert abs(diag["volume"] - 1.0 * 0.25 * 0.25) < 1e-3 and diag["inverted"] == 0 and diag["rmax"] > 0
    p = np.array([[float(v) for v in ln.split()] for ln in out.strip().split("\n")])
    X, T = O.beam_mesh(O.TETRA, (8, 2, 2), (1.0, 0.25, 0.25))
    m = O.masses(O.TETRA, X, T, 1000.0, 1)
    fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
    c, n = O.colour(O.TETRA, T, len(X), 0)
    s = O.Scene(O.TETRA, X, T, m, young=1e5, poisson=0.45, fixed=fixed, iterations=20, colors=c, n_colors=n,
                in_place=True)
    ref = O.Solver("vbd", s, fp64=True)
    for _ in range(5):
        ref.step(0.01, 1)
    assert rel_err(p, ref.get(0)) < 1e-5


@pytest.mark.gpu
def test_adapter_controller_matches_oracle(built, tmp_path):
    """Two fixation groups (one moving), a high stretch on for two frames, a box limit."""
    from test_effects_gpu import _farthest
    from octopusengine_b200 import capi
    exe = _compile(tmp_path, "adapter_controller")
    out = subprocess.check_output([exe, "6"], text=True)
    p = np.array([[float(v) for v in ln.split()] for ln in out.strip().split("\n")])
    X, T = O.beam_mesh(O.TETRA, (8, 2, 2), (1.0, 0.25, 0.25))
    m = O.masses(O.TETRA, X, T, 1000.0, 1)
    left = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
    right = O.fixed_by_plane(X, (0.99, 0, 0), (1, 0, 0))
    fixed = np.concatenate([left, right]).astype(np.int32)
    group = np.concatenate([np.zeros(len(left)), np.ones(len(right))]).astype(np.int32)
    c, n = O.colour(O.TETRA, T, len(X), 0)
    s = O.Scene(O.TETRA, X, T, m, young=1e5, poisson=0.45, fixed=fixed, fixed_group=group, iterations=10, colors=c,
                n_colors=n, in_place=True, box=((-10, -5, -10), (10, 5, 10)))
    ref = O.Solver("vbd", s, fp64=True)
    k = ref.add_effect(2, (6, 0.03), _farthest(X, capi.surface_nodes(O.TETRA, T), 6))
    for f in range(6):
        ref.set_fixation((0.0, 0.0, -0.01 * (f + 1)), group=1)
        ref.set_effect_active(k, f in (3, 4))
        ref.step(1 / 60, 1)
    assert rel_err(p, ref.get(0)) < 1e-5
    assert abs(p[right, 2] - (X[right, 2] - 0.06)).max() < 1e-5
