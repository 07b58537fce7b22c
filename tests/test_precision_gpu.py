"""Config 3 precision study at test size: a 1 m cube of P3 tetrahedra or Q2 hexahedra with a
per-element Young modulus log-uniform in [1e4, 1e6] Pa (seeded), nu = 0.45, rho = 1000,
bottom face fixed (rigid group 0) and top face moved down by 20 % of the height over 50
steps (rigid group 1, the fixed-node path with a moving target).  The same run in plain FP32
and in mixed precision on the GPU is compared with the FP64 oracle: positions, total energy
and residual.  Full-size (32^3 cells) throughput is measured by bench.py --workload cube_*."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import disp_err, rel_err

pytestmark = pytest.mark.gpu


def cube(element, n, seed=5):
    X, T = O.beam_mesh(element, (n, n, n), (1.0, 1.0, 1.0))
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), len(T))).astype(np.float32)
    bottom = np.nonzero(X[:, 2] < 1e-6)[0]
    top = np.nonzero(X[:, 2] > 1.0 - 1e-6)[0]
    fixed = np.concatenate([bottom, top]).astype(np.int32)
    group = np.concatenate([np.zeros(len(bottom)), np.ones(len(top))]).astype(np.int32)
    order = np.argsort(fixed, kind="stable")   # ascending ids, as GPU_Fix_Constraint collects them
    return X, T, E, fixed[order], group[order]


@pytest.mark.parametrize("element,n", [(O.TETRA20, 3), (O.HEXA27, 3)])
def test_precision_study(ctx, element, n):
    import octopusengine_b200 as ob
    X, T, E, fixed, group = cube(element, n)
    m = O.masses(element, X, T, 1000.0, 1)
    c, nc = O.colour(element, T, len(X), 0)
    common = dict(young_per_element=E, poisson=0.45, gravity=(0.0, 0.0, -9.81), iterations=8)
    runs = {}
    for prec in (ob.PREC_PLAIN, ob.PREC_MIXED):
        runs[prec] = ob.Scene(ctx, element, X, T, masses=m, fixed_ids=fixed, fixed_group=group, precision=prec,
                              young=1e5, **common)
    o64 = O.Solver("vbd", O.Scene(element, X, T, m, fixed=fixed, fixed_group=group, colors=c, n_colors=nc,
                                  in_place=True, young=1e5, **common), fp64=True)
    steps = 50
    energy = {k: [] for k in list(runs) + ["fp64"]}
    for k in range(1, steps + 1):
        off = (0.0, 0.0, -0.2 * k / steps)
        for s in runs.values():
            s.set_fixation(off, group=1)
        o64.set_fixation(off, group=1)
        for s in runs.values():
            s.step(1 / 60, 2)
        o64.step(1 / 60, 2)
        for key, s in runs.items():
            energy[key].append(s.energy()[3])
        energy["fp64"].append(o64.energy()[3])
    ref = o64.get(0)
    top = fixed[group == 1]
    np.testing.assert_allclose(ref[top, 2], X[top, 2] - 0.2, atol=1e-6)   # the top really moved
    eref = np.array(energy["fp64"])
    res = {}
    for key, s in runs.items():
        p = s.get_position()
        res[key] = (rel_err(p, ref), disp_err(p, ref, X), np.abs(np.array(energy[key]) - eref).max() / np.abs(eref).max())
    for key, (pe, de, ee) in res.items():
        assert pe < 1e-5, (key, res)
        assert de < 1e-4, (key, res)   # error relative to the displacement itself
        assert ee < 1e-3, (key, res)
    # both are at the 1e-6 level; mixed precision is not measurably worse than plain FP32
    assert res[ob.PREC_MIXED][1] <= 3.0 * res[ob.PREC_PLAIN][1] + 1e-6, res
    r = runs[ob.PREC_MIXED].residual(1 / 120)
    assert np.isfinite(r).all()
