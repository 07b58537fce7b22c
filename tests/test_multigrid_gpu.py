"""Multigrid VBD (MG_VBD_FEM, octopus/src/Dynamic/VBD/MG_VertexBlockDescent.cpp): iterations
alternate between the linear mesh of the corners (its own colouring and masses) and the full
P2 / Q2 mesh, mid nodes following the corners by prolongation; the GPU path against the FP64
oracle restatement."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import PLANE, rel_err

pytestmark = pytest.mark.gpu


def _setup(ctx, element, mg, iterations=10, cells=(4, 2, 2)):
    import octopusengine_b200 as ob
    X, T = O.beam_mesh(element, cells, (1.0, 0.25, 0.25))
    m = O.masses(element, X, T, 1000.0, 1)
    lin_e, nl = (O.TETRA, 4) if element == O.TETRA10 else (O.HEXA, 8)
    ml = O.masses(lin_e, X, np.ascontiguousarray(T[:, :nl]), 1000.0, 1)
    fixed = O.fixed_by_plane(X, *PLANE)
    s = ob.Scene(ctx, element, X, T, masses=m, young=1e5, poisson=0.45, fixed_ids=fixed, iterations=iterations,
                 gravity=(0.0, 0.0, -9.81), mg_linear=mg)
    c, n = O.colour(element, T, len(X), 0)
    sc = O.Scene(element, X, T, m, young=1e5, fixed=fixed, iterations=iterations, colors=c, n_colors=n, in_place=True,
                 mg_linear=mg, mg_masses=ml)
    return s, O.Solver("vbd", sc, fp64=True), (X, T, sc)


@pytest.mark.parametrize("element", [O.TETRA10, O.HEXA27])
@pytest.mark.parametrize("mg,iterations", [(0.5, 10), (0.3, 7), (1.0, 4)])
def test_multigrid_matches_oracle(ctx, element, mg, iterations):
    s, o64, keep = _setup(ctx, element, mg, iterations)
    for _ in range(4):
        s.step(1 / 60, 2)
        o64.step(1 / 60, 2)
    p = s.get_position()
    assert rel_err(p, o64.get(0)) < 1e-5
    assert np.abs(p - keep[0]).max() > 1e-3


def test_multigrid_is_a_different_solver_than_full(ctx):
    s, o64, keep = _setup(ctx, O.TETRA10, 0.5)
    full, _, _ = _setup(ctx, O.TETRA10, 0.0)
    for _ in range(3):
        s.step(1 / 60, 2)
        full.step(1 / 60, 2)
    d = np.abs(s.get_position() - full.get_position()).max()
    assert 1e-6 < d < 0.05


def test_multigrid_restrictions(ctx):
    import octopusengine_b200 as ob
    X, T = O.beam_mesh(O.TETRA, (2, 1, 1), (1.0, 0.25, 0.25))
    with pytest.raises(ob.OctError):
        ob.Scene(ctx, O.TETRA, X, T, mg_linear=0.5)
    s, _, _ = _setup(ctx, O.TETRA10, 0.5, cells=(2, 1, 1))
    with pytest.raises(ob.OctError):
        ob.Batch(ctx, [s])
