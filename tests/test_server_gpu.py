"""Serving loop: requests admitted while others run (continuous batching) give the same
result as the same scene stepped alone; HBM-budget admission queues what does not fit and
rejects what never can; p50/p99 step latency is reported."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import rel_err

pytestmark = pytest.mark.gpu


def _spec(i):
    e = [O.TETRA, O.TETRA10, O.HEXA][i % 3]
    cells = (3 + i % 4, 2, 1 + i % 2)
    X, T = O.beam_mesh(e, cells, (cells[0] * 0.1, cells[1] * 0.1, cells[2] * 0.1))
    fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
    kw = dict(density=1000.0, young=float(1e5 * (1 + i)), poisson=0.4, fixed_ids=fixed, gravity=(0.0, 0.0, -9.81))
    return e, X, T, kw


def test_results_equal_alone_and_in_the_mix(ctx):
    import octopusengine_b200 as ob
    srv = ob.Server(ctx, frame_dt=1 / 60, substeps=2, iterations=6, precision=ob.PREC_MIXED, max_scenes=64)
    steps = [3, 7, 5, 9, 4, 6]
    arrive = [0, 0, 1, 2, 4, 6]            # tick at which each request arrives
    ids = {}
    tick = 0
    while len(ids) < len(steps) or any(srv.poll(r) is None for r in ids.values()):
        for i, t in enumerate(arrive):
            if t == tick and i not in ids:
                e, X, T, kw = _spec(i)
                ids[i] = srv.submit(e, X, T, steps[i], **kw)
        srv.tick()
        tick += 1
        assert tick < 100
    st = srv.stats()
    assert st["finished"] == len(steps) and st["rejected"] == 0
    assert st["p99_step_ms"] >= st["p50_step_ms"] > 0
    for i, rid in ids.items():
        e, X, T, kw = _spec(i)
        alone = ob.Scene(ctx, e, X, T, iterations=6, precision=ob.PREC_MIXED, **kw)
        for _ in range(steps[i]):
            alone.step(1 / 60, 2)
        assert rel_err(srv.poll(rid), alone.get_position()) < 1e-6
        alone.close()
    srv.close()


def test_admission_by_hbm_budget(ctx):
    import octopusengine_b200 as ob
    e, X, T, kw = _spec(1)
    d, keep = ob.make_desc(e, X, T, **kw)
    import ctypes as C
    from octopusengine_b200 import capi
    need = C.c_size_t()
    capi.lib().oct_scene_footprint(C.byref(d), C.byref(need))
    # room for two such scenes only
    srv = ob.Server(ctx, frame_dt=1 / 60, substeps=1, iterations=2, hbm_budget=int(need.value * 2.5))
    ids = [srv.submit(e, X, T, 3, **kw) for _ in range(4)]
    srv.tick()
    st = srv.stats()
    assert st["active"] + st["admitted"] - st["active"] <= 4
    assert st["queued"] >= 1 and st["bytes_in_use"] <= need.value * 2.5
    for _ in range(30):
        srv.tick()
    assert all(srv.poll(r) is not None for r in ids)
    # a scene that can never fit is rejected at submit
    big = O.beam_mesh(O.TETRA10, (20, 6, 6), (2, 0.6, 0.6))
    with pytest.raises(ob.OctError) as ei:
        srv.submit(O.TETRA10, big[0], big[1], 2, density=1000.0)
    assert ei.value.status == capi.ENOMEM_BUDGET
    assert srv.stats()["rejected"] == 1
    srv.close()


def _nan_v0(n):
    v0 = np.zeros((n, 3), np.float32)
    v0[n // 2, 1] = np.nan   # a host-side fault: one request's state carries a NaN
    return v0


def test_a_failing_scene_is_reported_alone_in_a_batch(ctx):
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    specs = [_spec(i) for i in range(3)]
    scenes = []
    for i, (e, X, T, kw) in enumerate(specs):
        extra = dict(initial_velocity=_nan_v0(len(X))) if i == 1 else {}
        scenes.append(ob.Scene(ctx, e, X, T, iterations=6, precision=ob.PREC_MIXED, **kw, **extra))
    b = ob.Batch(ctx, scenes)
    b.step(1 / 60, 2)
    np.testing.assert_array_equal(b.status(), [capi.OK, capi.ENUMERIC, capi.OK])
    np.testing.assert_array_equal(b.status(), [capi.OK] * 3)   # reading cleared the flags
    for i in (0, 2):
        e, X, T, kw = specs[i]
        alone = ob.Scene(ctx, e, X, T, iterations=6, precision=ob.PREC_MIXED, **kw)
        alone.step(1 / 60, 2)
        assert alone.status() == capi.OK
        assert rel_err(scenes[i].get_position(), alone.get_position()) < 1e-6
        alone.close()
    b.close()
    # the same scene stepped alone reports the failure through its own status
    e, X, T, kw = specs[1]
    s = ob.Scene(ctx, e, X, T, iterations=6, **kw, initial_velocity=_nan_v0(len(X)))
    s.step(1 / 60, 1)
    assert s.status() == capi.ENUMERIC
    assert s.status() == capi.OK
    s.close()
    for sc in scenes:
        sc.close()


def test_a_failed_request_ends_alone_and_the_others_are_unchanged(ctx):
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    srv = ob.Server(ctx, frame_dt=1 / 60, substeps=2, iterations=6, precision=ob.PREC_MIXED, max_scenes=64)
    steps = [4, 6, 5, 3]
    ids = {}
    for i in range(len(steps)):
        e, X, T, kw = _spec(i)
        ids[i] = srv.submit(e, X, T, steps[i], **kw)
    e, X, T, kw = _spec(1)
    bad = srv.submit(e, X, T, 5, initial_velocity=_nan_v0(len(X)), **kw)
    status = {}
    for _ in range(40):
        srv.tick()
        for i, rid in list(ids.items()) + [("bad", bad)]:
            if i in status:
                continue
            try:
                if srv.poll(rid, fetch=False) is not None:
                    status[i] = capi.OK
            except ob.OctError as err:
                status[i] = err.status
        if len(status) == len(steps) + 1:
            break
    assert status["bad"] == capi.ENUMERIC
    assert all(status[i] == capi.OK for i in range(len(steps)))
    st = srv.stats()
    assert st["failed"] == 1 and st["finished"] == len(steps)
    for i, rid in ids.items():
        e, X, T, kw = _spec(i)
        alone = ob.Scene(ctx, e, X, T, iterations=6, precision=ob.PREC_MIXED, **kw)
        for _ in range(steps[i]):
            alone.step(1 / 60, 2)
        assert rel_err(srv.poll(rid), alone.get_position()) < 1e-6
        alone.close()
    srv.close()
