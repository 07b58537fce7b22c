"""The product's CUDA kernels against numbers OctopusEngine itself produced: the 16 static-flexion
result files (4 element types x E in {1e6, 1e7} x nu in {0.45, 0.49}, 32 x 8 x 8 beams of up to
18,785 nodes), stored as fixtures by tests/golden/make_reference_static.py.

* The element-diagnostic kernel (GPU_FEM::get_stress / get_volume / get_volume_diff,
  octopus/src/GPU/GPU_FEM.cu:20-85), run at the reference's end state, reproduces the file's
  per-element fields.
* The elastic force pass (the force term of the VBD colour kernel, here through the explicit
  integrator's acceleration: v = (g + f / m) dt from rest) balances gravity at that state: it is
  the stationary point of the product's energy along the reference's displacement.
* One VBD sub-step from a state near it, at these real sizes, matches the FP64 oracle within the
  FP32 oracle's own error, in the drop-in (plain) and the mixed precision.
The bars and why they are what they are: tests/reference_static.py."""
import numpy as np
import pytest

import oracle_lib as O
import reference_static as RS
from scenes import disp_err

pytestmark = pytest.mark.gpu


def _mesh(c):
    import octopusengine_b200 as ob
    X, T = ob.beam_mesh(c["element"], RS.CELLS, RS.SIZE, c["origin"])
    assert RS.topology_sha256(T) == c["topology_sha256"]
    m = ob.lumped_masses(c["element"], X, T, RS.DENSITY, ob.MASS_FEMSHAPE)
    return X, T, m, RS.fixed_ids(X)


def _scene(ctx, c, X, T, m, fixed, **kw):
    import octopusengine_b200 as ob
    return ob.Scene(ctx, c["element"], X, T, masses=m, material=ob.STABLE_NEOHOOKE, young=c["young"],
                    poisson=c["poisson"], gravity=RS.GRAVITY, fixed_ids=fixed, **kw)


def _oracle_stress(c, X, T, m, x):
    out = []
    for fp64 in (True, False):
        sc = O.Scene(c["element"], X, T, m, material=O.STABLE_NEOHOOKE, young=c["young"], poisson=c["poisson"],
                     colors=np.zeros(len(X), np.int32), n_colors=1)
        s = O.Solver("vbd", sc, fp64=fp64)
        s.set(0, x)
        out.append(s.element_data(4))
    return out


@pytest.mark.parametrize("name", RS.NAMES)
def test_element_kernel_reproduces_the_reference_fields(ctx, name):
    import octopusengine_b200 as ob
    c = RS.case(name)
    X, T, m, fixed = _mesh(c)
    s = _scene(ctx, c, X, T, m, fixed, iterations=10)
    x = (X.astype(np.float64) + c["u"]).astype(np.float32)
    s.set_position(x)
    vol = s.element_data(ob.DIAG_VOLUME_ACCUMULATED).astype(np.float64)
    vdiff = s.element_data(ob.DIAG_VOLUME_DIFF_ACCUMULATED).astype(np.float64)
    stress = s.element_data(ob.DIAG_STRESS_ACCUMULATED).astype(np.float64)
    RS.check_volumes(c, vol, vdiff)
    o64, o32 = _oracle_stress(c, X, T, m, x.astype(np.float64))
    RS.check_stress(c, stress, o64, o32)
    # the kernel evaluates the formula in FP64: it equals the FP64 oracle up to its float output
    np.testing.assert_allclose(stress, o64, rtol=2e-6, atol=1e-6 * np.abs(o64).max())


@pytest.mark.parametrize("name", RS.NAMES)
def test_elastic_forces_balance_gravity_at_the_reference_state(ctx, name):
    import octopusengine_b200 as ob
    c = RS.case(name)
    X, T, m, fixed = _mesh(c)
    s = _scene(ctx, c, X, T, m, fixed, solver=ob.SOLVER_EXPLICIT)
    free = np.ones(len(X), bool)
    free[fixed] = False
    h = 1e-4
    zero = np.zeros_like(X)
    works = []
    for a in RS.ALPHAS:
        x = (X.astype(np.float64) + a * c["u"]).astype(np.float32)
        s.set_position(x)
        s.set_velocity(zero)
        s.step(h, 1)
        r = m[:, None].astype(np.float64) * s.get_velocity().astype(np.float64) / h   # f_elastic + m g
        works.append(RS.virtual_work(r, c["u"], m, free))
    RS.check_stationary(c, works)


SOFT = [n for n in RS.NAMES if n.endswith("1e6_045")]


@pytest.mark.parametrize("name", SOFT)
def test_vbd_substep_near_the_reference_state_matches_the_oracle(ctx, name):
    import octopusengine_b200 as ob
    c = RS.case(name)
    X, T, m, fixed = _mesh(c)
    x = (X.astype(np.float64) + 0.98 * c["u"]).astype(np.float32)
    dt, iterations = 1.0 / 300.0, 10
    colors, n_colors = O.colour(c["element"], T, len(X), 0, -1)
    ref = []
    for fp64 in (False, True):
        sc = O.Scene(c["element"], X, T, m, material=O.STABLE_NEOHOOKE, young=c["young"], poisson=c["poisson"],
                     gravity=RS.GRAVITY, fixed=fixed, colors=colors, n_colors=n_colors, in_place=True,
                     iterations=iterations)
        o = O.Solver("vbd", sc, fp64=fp64)
        o.set(0, x)
        o.set(2, x)
        o.step(dt, 1)
        ref.append(o.get(0))
    e32 = disp_err(ref[0], ref[1], x)
    for precision, factor in ((ob.PREC_PLAIN, 4.0), (ob.PREC_MIXED, 2.0)):
        s = _scene(ctx, c, X, T, m, fixed, iterations=iterations, precision=precision)
        np.testing.assert_array_equal(s.coloring()[0], colors)
        s.set_position(x)
        s.set_velocity(np.zeros_like(x))   # at rest: the implicit velocity of the next sub-step is 0
        s.step(dt, 1)
        e = disp_err(s.get_position(), ref[1], x)
        assert e < max(factor * e32, 1e-4), (name, precision, e, e32)
