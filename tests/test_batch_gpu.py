"""Batching equivalence: each scene stepped alone (reference launch structure) and inside a
mixed batch (one launch per element type and colour, CUDA graph) gives the same result
within the FP32 tolerance, and the batch's host-state round trip is exact."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import check_parity, pair, rel_err

pytestmark = pytest.mark.gpu


def _mix(ctx, rng, n, precision=0):
    import octopusengine_b200 as ob
    out = []
    for i in range(n):
        e = [O.TETRA, O.TETRA10, O.HEXA][i % 3]
        cells = (int(rng.integers(2, 7)), int(rng.integers(1, 4)), int(rng.integers(1, 4)))
        young = float(np.exp(rng.uniform(np.log(1e4), np.log(1e7))))
        nu = float(rng.uniform(0.3, 0.49))
        X, T = O.beam_mesh(e, cells, (cells[0] * 0.1, cells[1] * 0.1, cells[2] * 0.1))
        fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
        kw = dict(density=1000.0, mass_distribution=ob.MASS_FEMSHAPE, young=young, poisson=nu, fixed_ids=fixed,
                  iterations=8, gravity=(0.0, 0.0, -9.81), precision=precision)
        out.append((e, X, T, kw))
    return out


def test_batch_equals_single_scenes(ctx):
    import octopusengine_b200 as ob
    rng = np.random.default_rng(11)
    specs = _mix(ctx, rng, 12)
    alone = [ob.Scene(ctx, e, X, T, **kw) for e, X, T, kw in specs]
    mixed = [ob.Scene(ctx, e, X, T, **kw) for e, X, T, kw in specs]
    batch = ob.Batch(ctx, mixed)
    for _ in range(3):
        for s in alone:
            s.step(1 / 60, 4)
        batch.step(1 / 60, 4)
    for a, b in zip(alone, mixed):
        # the same kernels over the same work items: a batch gives each scene its own result
        np.testing.assert_array_equal(b.get_position(), a.get_position())
    for s in alone + mixed:
        s.close()
    batch.close()


def test_batch_matches_oracle_and_state_round_trip(ctx):
    import octopusengine_b200 as ob
    s1, o32, o64, mesh = pair(ctx, O.TETRA10, cells=(4, 2, 2), iterations=6)
    s2, p32, p64, mesh2 = pair(ctx, O.HEXA, cells=(3, 2, 2), iterations=6)
    batch = ob.Batch(ctx, [s1, s2])
    batch.step(1 / 60, 3)
    for o in (o32, o64, p32, p64):
        o.step(1 / 60, 3)
    check_parity(s1.get_position(), o32, o64, mesh["X"], "P2 in a batch")
    check_parity(s2.get_position(), p32, p64, mesh2["X"], "Q1 in a batch")
    state = np.zeros(batch.state_size, np.float32)
    batch.get_state(state)
    n1 = s1.n_nodes
    np.testing.assert_allclose(state[: 3 * n1].reshape(-1, 3) + mesh["X"], s1.get_position(), atol=1e-6)
    batch.set_state(state)
    state2 = np.zeros_like(state)
    batch.get_state(state2)
    assert np.array_equal(state, state2)
    batch.close()


def test_batch_rejects_mismatched_iterations(ctx):
    import octopusengine_b200 as ob
    X, T = O.beam_mesh(O.TETRA, (2, 1, 1), (1, 1, 1))
    a = ob.Scene(ctx, O.TETRA, X, T, iterations=3)
    b = ob.Scene(ctx, O.TETRA, X, T, iterations=4)
    with pytest.raises(ob.OctError):
        ob.Batch(ctx, [a, b])


def test_autotune_keeps_state_and_picks_a_valid_mapping(ctx):
    """oct_autotune_mapping times every mapping without touching positions or velocities; the
    scenes then step exactly as scenes created with the chosen mapping."""
    import octopusengine_b200 as ob
    rng = np.random.default_rng(5)
    specs = _mix(ctx, rng, 9)
    tuned = [ob.Scene(ctx, e, X, T, **kw) for e, X, T, kw in specs]
    for s in tuned:
        s.step(1 / 60, 2)
    before = [(s.get_position(), s.get_velocity()) for s in tuned]
    chosen = ob.autotune_mapping(ctx, tuned, 1 / 240, sweeps=2)
    assert set(chosen) == {O.TETRA, O.TETRA10, O.HEXA}
    assert all(v in (-1, 1, 2, 4, 8, 16, 32) for v in chosen.values())
    for s, (p, v) in zip(tuned, before):
        np.testing.assert_array_equal(s.get_position(), p)
        np.testing.assert_array_equal(s.get_velocity(), v)
    ref = []
    for (e, X, T, kw) in specs:   # same history: default mapping for the first frame, then the chosen one
        r = ob.Scene(ctx, e, X, T, **kw)
        r.step(1 / 60, 2)
        r.set_mapping(chosen[e])
        assert r.mapping() == chosen[e]
        ref.append(r)
    batch = ob.Batch(ctx, tuned)
    rbatch = ob.Batch(ctx, ref)
    for _ in range(2):
        batch.step(1 / 60, 2)
        rbatch.step(1 / 60, 2)
    for a, b in zip(tuned, ref):
        np.testing.assert_array_equal(a.get_position(), b.get_position())


@pytest.mark.parametrize("mapping", [-1, 1, 2, 8])
def test_set_mapping_mid_run_matches_oracle(ctx, mapping):
    s, o32, o64, mesh = pair(ctx, O.TETRA10, cells=(4, 2, 2), iterations=6)
    s.step(1 / 60, 2)
    o64.step(1 / 60, 2)
    assert s.mapping() == 1   # the measured default for P2 (corner colours widen to 4 lanes)
    s.set_mapping(mapping)
    assert s.mapping() == mapping
    s.set_capture(True)
    for _ in range(2):
        s.step(1 / 60, 2)
        o64.step(1 / 60, 2)
    assert rel_err(s.get_position(), o64.get(0)) < 1e-5


def test_xpbd_batch_equals_scenes_alone_and_the_oracle(ctx):
    """GPU_PBD::step over an XPBD batch (mixed element types, materials, update forms and
    global damping, one launch per group and colour across the scenes) gives each scene's own
    result bit for bit (the elements of a colour share no node, so their order does not
    matter), and matches the oracle."""
    import octopusengine_b200 as ob
    rng = np.random.default_rng(5)
    cases = [(O.TETRA, O.STABLE_NEOHOOKE, O.XPBD_OPTISHARED, 0.0), (O.TETRA10, O.NEOHOOKE, O.XPBD_OPTISHARED, 0.5),
             (O.HEXA, O.STVK, O.XPBD_V0, 0.2), (O.TETRA10, O.COROTATED, O.XPBD_V0, 0.0),
             (O.HEXA27, O.STABLE_NEOHOOKE, O.XPBD_QUADRATURE, 1.0), (O.HEXA, O.STABLE_NEOHOOKE, O.XPBD_OPTIGROUP, 0.0),
             (O.TETRA, O.HOOKE, O.XPBD_OPTISHARED, 0.3)]
    alone, mixed, oracles = [], [], []
    for e, mat, ver, damp in cases:
        cells = (2, 1, 1) if e == O.HEXA27 else (int(rng.integers(2, 5)), 2, int(rng.integers(1, 3)))
        s, o32, o64, mesh = pair(ctx, e, cells=cells, material=mat, solver="xpbd", young=1e5, xpbd_version=ver,
                                 global_damping=damp)
        t, _, _, _ = pair(ctx, e, cells=cells, material=mat, solver="xpbd", young=1e5, xpbd_version=ver,
                          global_damping=damp)
        alone.append(s)
        mixed.append(t)
        oracles.append(o32)
    batch = ob.Batch(ctx, mixed)
    for frame in range(3):
        for s in alone:
            s.step(1 / 60, 5)
        batch.step(1 / 60, 5)
        if frame == 0:   # after one frame within the FP32 parity bar of the XPBD tests
            for o, b in zip(oracles, mixed):
                o.step(1 / 60, 5)
                assert rel_err(b.get_position(), o.get(0)) < 1e-5
    assert (batch.status() == 0).all()
    for a, b in zip(alone, mixed):
        np.testing.assert_array_equal(b.get_position(), a.get_position())
        np.testing.assert_array_equal(b.get_velocity(), a.get_velocity())
    batch.close()


def test_batches_hold_one_solver(ctx):
    import octopusengine_b200 as ob
    a, _, _, _ = pair(ctx, O.TETRA, cells=(2, 1, 1), solver="xpbd")
    b, _, _, _ = pair(ctx, O.TETRA, cells=(2, 1, 1))
    c, _, _, _ = pair(ctx, O.TETRA, cells=(2, 1, 1), solver="explicit")
    with pytest.raises(ob.OctError) as e:
        ob.Batch(ctx, [a, b])
    assert e.value.status == 6   # OCT_ENOTSUP
    with pytest.raises(ob.OctError):
        ob.Batch(ctx, [c])
