"""Failure detection without faulting the GPU: a bounded device wait that runs out is reported
as OCT_ETIMEDOUT and leaves the context usable; a non-finite value forged into the host state
is caught by the FP64 reductions (OCT_ENUMERIC); a scene larger than the context's HBM budget is
refused before anything is allocated; and checkpoint / restore reproduces a run exactly."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import pair

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_context_survives(ctx):
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    st = capi.lib().oct_ctx_wait_probe(ctx.handle, 2000)
    assert st == capi.ETIMEDOUT
    s, o32, o64, mesh = pair(ctx, O.TETRA, cells=(2, 1, 1), iterations=3)
    s.step(1 / 60, 1)   # the context still steps scenes
    assert np.isfinite(s.get_position()).all()


def test_forged_nan_is_detected_by_the_fp64_reductions(ctx):
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    s, o32, o64, mesh = pair(ctx, O.TETRA10, cells=(2, 1, 1), iterations=3)
    good = s.get_position()
    bad = good.copy()
    bad[len(bad) // 2, 1] = np.nan
    s.set_position(bad)
    with pytest.raises(ob.OctError) as e:
        s.residual(1 / 120)
    assert e.value.status == capi.ENUMERIC
    with pytest.raises(ob.OctError) as e:
        s.energy()
    assert e.value.status == capi.ENUMERIC
    s.set_position(good)   # a finite state is accepted again
    assert np.isfinite(s.energy()).all()


def test_over_budget_scene_is_refused_without_allocation(built):
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    c = ob.Context(0, 1 << 20)   # 1 MiB budget
    try:
        used0, budget = c.memory()
        X, T = O.beam_mesh(O.TETRA10, (32, 8, 8), (4.0, 1.0, 1.0))
        with pytest.raises(ob.OctError) as e:
            ob.Scene(c, O.TETRA10, X, T)
        assert e.value.status == capi.ENOMEM_BUDGET
        assert c.memory()[0] == used0
    finally:
        c.close()


@pytest.mark.parametrize("kind", ["vbd_effects", "multigrid", "xpbd"])
def test_checkpoint_restore_reproduces_the_run(ctx, kind):
    from octopusengine_b200 import capi
    import octopusengine_b200 as ob
    if kind == "multigrid":
        X, T = O.beam_mesh(O.TETRA10, (3, 2, 2), (1.0, 0.25, 0.25))
        s = ob.Scene(ctx, O.TETRA10, X, T, fixed_ids=O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0)), young=1e5,
                     iterations=7, gravity=(0.0, 0.0, -9.81), mg_linear=0.4)
    else:
        s, o32, o64, mesh = pair(ctx, O.HEXA, cells=(3, 2, 2), iterations=5, solver="xpbd" if kind == "xpbd" else "vbd")
        if kind == "vbd_effects":
            k = s.add_effect(capi.EFFECT_HIGH_STRETCH, 4, 0.02)
            s.set_effect_active(k, True)
    for _ in range(2):
        s.step(1 / 60, 3)
    snap = s.save()
    for _ in range(2):
        s.step(1 / 60, 3)
    a = s.get_position(), s.get_velocity()
    s.restore(snap)
    for _ in range(2):
        s.step(1 / 60, 3)
    np.testing.assert_array_equal(s.get_position(), a[0])
    np.testing.assert_array_equal(s.get_velocity(), a[1])


def test_restore_refuses_a_checkpoint_of_another_scene(ctx):
    from octopusengine_b200 import capi
    import octopusengine_b200 as ob
    a, _, _, _ = pair(ctx, O.HEXA, cells=(3, 2, 2), iterations=3)
    b, _, _, _ = pair(ctx, O.HEXA, cells=(4, 2, 2), iterations=3)
    a.step(1 / 60, 1)
    snap = a.save()
    assert snap.size == a.save().size
    with pytest.raises(ob.OctError) as e:
        b.restore(snap)
    assert e.value.status == capi.EINVAL
    with pytest.raises(ob.OctError):
        b.restore(np.zeros(b.save().size, np.float32))   # not a checkpoint at all
    before = b.get_position()
    b.step(1 / 60, 1)   # the refused restores left b untouched
    assert np.isfinite(b.get_position()).all() and not np.array_equal(before, b.get_position())
