"""Edge cases of the scene boundary: empty, out-of-range and degenerate inputs are refused with
OCT_EINVAL before anything runs; the smallest scenes (one element, every node fixed, one
iteration, many sub-steps) step like the oracle."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import rel_err

pytestmark = pytest.mark.gpu


def _refused(ctx, element, X, T, **kw):
    import octopusengine_b200 as ob
    with pytest.raises(ob.OctError) as e:
        ob.Scene(ctx, element, X, T, **kw)
    return e.value.status


def test_invalid_meshes_are_refused(ctx):
    from octopusengine_b200 import capi
    X, T = O.beam_mesh(O.TETRA, (2, 1, 1), (1.0, 0.25, 0.25))
    assert _refused(ctx, O.TETRA, X, T[:0]) == capi.EINVAL                       # no elements
    bad = T.copy()
    bad[0, 0] = len(X)
    assert _refused(ctx, O.TETRA, X, bad) == capi.EINVAL                         # node id out of range
    flat = X.copy()
    flat[:, 2] = 0.0
    assert _refused(ctx, O.TETRA, flat, T) == capi.EINVAL                        # zero-volume elements
    assert _refused(ctx, O.TETRA, X, T, fixed_ids=np.array([len(X)])) == capi.EINVAL
    assert _refused(ctx, O.TETRA, X, T, threads_per_vertex=3) == capi.EINVAL
    assert _refused(ctx, O.TETRA, X, T, fixed_ids=np.array([0]), fixed_group=np.array([4])) == capi.EINVAL


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10, O.TETRA20, O.HEXA27])
def test_one_element_scene(ctx, element):
    import octopusengine_b200 as ob
    X, T = O.beam_mesh(element, (1, 1, 1), (0.5, 0.5, 0.5))
    T = T[:1]
    used = np.unique(T)
    remap = -np.ones(len(X), np.int64)
    remap[used] = np.arange(len(used))
    X, T = X[used], remap[T].astype(np.int32)
    m = O.masses(element, X, T, 1000.0, 1)
    fixed = np.nonzero(X[:, 0] < 1e-6)[0].astype(np.int32)
    s = ob.Scene(ctx, element, X, T, masses=m, fixed_ids=fixed, young=1e5, iterations=6, gravity=(0.0, 0.0, -9.81))
    c, n = O.colour(element, T, len(X), 0)
    ref = O.Solver("vbd", O.Scene(element, X, T, m, young=1e5, fixed=fixed, iterations=6, colors=c, n_colors=n,
                                  in_place=True), fp64=True)
    for _ in range(3):
        s.step(1 / 60, 2)
        ref.step(1 / 60, 2)
    assert rel_err(s.get_position(), ref.get(0)) < 1e-5


def test_every_node_fixed_follows_its_group(ctx):
    import octopusengine_b200 as ob
    X, T = O.beam_mesh(O.HEXA, (2, 1, 1), (1.0, 0.25, 0.25))
    s = ob.Scene(ctx, O.HEXA, X, T, fixed_ids=np.arange(len(X), dtype=np.int32), iterations=3)
    s.set_fixation((0.1, 0.0, 0.0))
    s.step(1 / 60, 2)
    np.testing.assert_allclose(s.get_position(), X + np.array([0.1, 0.0, 0.0], np.float32), atol=1e-6)


@pytest.mark.parametrize("iterations,substeps", [(1, 1), (1, 40)])
def test_minimal_iterations_and_many_substeps(ctx, iterations, substeps):
    import octopusengine_b200 as ob
    from scenes import pair
    s, o32, o64, mesh = pair(ctx, O.TETRA10, cells=(3, 1, 1), iterations=iterations)
    s.step(1 / 60, substeps)
    o64.step(1 / 60, substeps)
    assert rel_err(s.get_position(), o64.get(0)) < 1e-5


def test_invalid_step_arguments(ctx):
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    from scenes import pair
    s, o32, o64, mesh = pair(ctx, O.TETRA, cells=(2, 1, 1))
    for dt, sub in ((0.0, 1), (-1.0, 1), (1 / 60, 0)):
        with pytest.raises(ob.OctError) as e:
            s.step(dt, sub)
        assert e.value.status == capi.EINVAL
    with pytest.raises(ob.OctError):
        s.set_fixation((0, 0, 0), group=4)
