"""The accuracy measures (octopusengine_b200/csrc/measure.cpp) on the states OctopusEngine itself
wrote in its experiments, against the numpy restatement of the reference's measures
(oracle/measures.py, the checker): the torsion profile of FEM_Torsion_error_recorder
(octopus/src/Script/Record/Recorder.cpp:222-309) on its twisted P1 and Q1 beams, and
MeshDiff_MSE (octopus/include/Script/Measure/MeshDiff.h:64-83) between its small-step runs and
their reference run.  Fixtures: tests/golden/reference_measures.npz
(tests/golden/make_reference_measures.py)."""
import os

import numpy as np
import pytest

from oracle import measures as M

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = np.load(os.path.join(HERE, "golden", "reference_measures.npz"))
NAMES = sorted({k.split("/")[0] for k in FIX.files})


def _state(name):
    import octopusengine_b200 as ob
    import reference_static as RS
    meta = FIX[name + "/meta"]
    e = int(meta[0])
    X, T = ob.beam_mesh(e, tuple(int(v) for v in meta[1:4]), tuple(meta[4:7]), tuple(meta[7:10]))
    assert RS.topology_sha256(T) == str(FIX[name + "/topology_sha256"])   # the reference's own mesh
    return e, X.astype(np.float64), T, FIX[name + "/u"].astype(np.float64)


@pytest.mark.parametrize("name", [n for n in NAMES if n.startswith("torsion")])
@pytest.mark.parametrize("samples", [2, 5])
def test_torsion_profile_of_the_reference_twist(built, name, samples):
    from octopusengine_b200 import capi
    e, X, T, u = _state(name)
    cur = X + u
    d, a = capi.torsion_profile(e, X, cur, T, samples, 2.0)
    rd, ra = M.torsion_profile(e, X, cur, T, samples, 2.0)
    assert len(d) == len(rd) > 8
    np.testing.assert_allclose(d, rd, atol=2e-6)
    np.testing.assert_allclose(a, ra, atol=2e-3)   # degrees; FP32 against FP64 evaluation
    # the profile's ends are the rotations of the beam's end faces (folded into [0, 180] degrees,
    # as the recorder's |atan2| folds them): the controller turned the x = 0 face, x = 2 is held
    for x0, at in ((0.0, a[0]), (2.0, a[-1])):
        face = np.nonzero(np.abs(X[:, 0] - x0) < 1e-6)[0]
        face = face[np.linalg.norm(X[face, 1:] - 0.5, axis=1) > 0.25]
        r0 = X[face, 1:] - 0.5
        r1 = cur[face, 1:] - 0.5
        turn = np.degrees(np.abs(np.arctan2(r0[:, 0] * r1[:, 1] - r0[:, 1] * r1[:, 0], (r0 * r1).sum(1))))
        assert abs(at - np.median(turn)) < 1e-2, (x0, at, np.median(turn))
    assert a.max() > 30.0   # and the beam in between is really twisted


@pytest.mark.parametrize("name", [n for n in NAMES if n.startswith("small_steps_") and not n.endswith("ref")])
def test_mesh_diff_of_the_small_step_runs(built, name):
    from octopusengine_b200 import capi
    e, X, T, u = _state(name)
    er, Xr, Tr, ur = _state("small_steps_ref")
    got = capi.mesh_error((Xr + ur).astype(np.float32), (X + u).astype(np.float32), (Xr[0] - X[0]).astype(np.float32))
    want = M.mesh_diff_mse(Xr + ur, Xr[0], X + u, X[0])
    for k in ("MSE", "RMSE", "MAE", "max", "L1", "L2"):
        assert got[k] == pytest.approx(want[k], rel=1e-5), k
    assert want["max"] > 1e-2   # the runs differ from their reference run: the measure sees it
