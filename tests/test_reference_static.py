"""The oracle and the product's host mesh code against the reference's own result files
(CPU; the GPU kernels are checked against the same numbers in test_reference_static_gpu.py).

For each of the 16 static-flexion files (4 element types x E in {1e6, 1e7} x nu in {0.45, 0.49}):
the product's beam generator rebuilds the reference's mesh bit for bit, and the FP64 oracle,
evaluated at the reference's end state, reproduces the file's accumulated volume, volume change
and stress and finds that state to be the static equilibrium of its own elastic forces."""
import numpy as np
import pytest

import oracle_lib as O
import reference_static as RS

DT = 1.0 / 300.0


@pytest.mark.parametrize("name", RS.NAMES)
def test_product_beam_is_the_reference_mesh(built, name):
    import octopusengine_b200 as ob
    c = RS.case(name)
    X, T = ob.beam_mesh(c["element"], RS.CELLS, RS.SIZE, c["origin"])
    assert len(X) == c["n_points"] and len(T) == c["n_elements"]
    assert RS.topology_sha256(T) == c["topology_sha256"]


def _oracle(c, fp64=True):
    X, T = O.beam_mesh(c["element"], RS.CELLS, RS.SIZE, c["origin"])
    m = O.masses(c["element"], X, T, RS.DENSITY, 1)
    fixed = RS.fixed_ids(X)
    # never stepped: one colour stands in for the colouring the solver object needs
    sc = O.Scene(c["element"], X, T, m, material=O.STABLE_NEOHOOKE, young=c["young"], poisson=c["poisson"],
                 gravity=RS.GRAVITY, fixed=fixed, colors=np.zeros(len(X), np.int32), n_colors=1)
    return O.Solver("vbd", sc, fp64=fp64), X, m, fixed, sc


@pytest.mark.parametrize("name", RS.NAMES)
def test_oracle_reproduces_the_reference_fields(built, name):
    c = RS.case(name)
    s64, X, m, fixed, keep = _oracle(c, True)
    s32, *_ = _oracle(c, False)
    x = X.astype(np.float64) + c["u"]
    s64.set(0, x)
    s32.set(0, x)
    RS.check_volumes(c, s64.element_data(5), s64.element_data(6))
    RS.check_stress(c, s64.element_data(4), s64.element_data(4), s32.element_data(4))


@pytest.mark.parametrize("name", RS.NAMES)
def test_reference_state_is_the_oracle_equilibrium(built, name):
    c = RS.case(name)
    s, X, m, fixed, keep = _oracle(c, True)
    free = np.ones(len(X), bool)
    free[fixed] = False
    g = np.asarray(RS.GRAVITY)
    works = []
    for a in RS.ALPHAS:
        x = X.astype(np.float64) + a * c["u"]
        for what in (0, 2, 3):   # p = last_p = y: no inertia, no damping term
            s.set(what, x)
        r = s.forces(DT) + m[:, None] * g
        works.append(RS.virtual_work(r, c["u"], m, free))
    RS.check_stationary(c, works)
