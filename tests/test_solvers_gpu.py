"""GPU parity of the XPBD coloured element projection and of the explicit integrator
against the CPU oracle (GPU_PBD / kernel_XPBD_V0 and GPU_SemiExplicit /
kernel_fem_eval_force semantics)."""
import numpy as np
import pytest

import oracle_lib as O
from scenes import pair, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10])
@pytest.mark.parametrize("material", [O.STABLE_NEOHOOKE, O.NEOHOOKE, O.STVK, O.HOOKE])
def test_xpbd_parity(ctx, element, material):
    s, o32, o64, mesh = pair(ctx, element, cells=(4, 2, 2), material=material, solver="xpbd", young=1e5,
                             global_damping=0.5)
    for _ in range(3):
        s.step(1 / 60, 5)
        o32.step(1 / 60, 5)
    assert rel_err(s.get_position(), o32.get(0)) < 1e-5
    assert np.isfinite(s.get_velocity()).all()


def test_xpbd_element_colouring_matches_reference_order(ctx):
    import octopusengine_b200 as ob
    X, T = O.beam_mesh(O.TETRA10, (4, 2, 2), (1, 0.25, 0.25))
    c1, n1 = O.colour(O.TETRA10, T, len(X), 2)
    c2, n2, _ = ob.color(O.TETRA10, T, len(X), 2)
    assert n1 == n2 and np.array_equal(c1, c2)


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10])
def test_explicit_parity(ctx, element):
    s, o32, o64, mesh = pair(ctx, element, cells=(4, 2, 2), solver="explicit", young=1e5, damping=1e-4)
    for _ in range(5):
        s.step(1e-3, 20)
        o32.step(1e-3, 20)
    assert rel_err(s.get_position(), o32.get(0)) < 1e-5
    v = s.get_velocity()
    assert np.abs(v - o32.get(1)).max() < 1e-3 * max(1.0, np.abs(o32.get(1)).max())
