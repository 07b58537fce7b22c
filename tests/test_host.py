"""CPU tests of the product's host side: the C ABI library loads and exports every declared
symbol, and its scene set-up (beam meshes, masses, shape tables, colourings) equals the
oracle's restatement of the reference bit for bit."""
import json
import os
import re

import numpy as np
import pytest

import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHAPES = json.load(open(os.path.join(ROOT, "tests", "golden", "shapes.json")))
ELEMS = [O.TETRA, O.HEXA, O.TETRA10, O.TETRA20, O.HEXA27]
NAMES = {O.TETRA: "Tetra", O.HEXA: "Hexa", O.TETRA10: "Tetra10", O.TETRA20: "Tetra20", O.HEXA27: "Hexa27"}


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "octopus_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(oct_[a-z0-9_]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol(built):
    import ctypes
    from octopusengine_b200 import capi
    lib = ctypes.CDLL(capi.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(lib, s), s
    assert set(capi.EXPORTS) == set(syms)


@pytest.mark.parametrize("e", ELEMS)
def test_shape_tables_match_golden(built, e):
    import octopusengine_b200 as ob
    q, w, d = ob.shape_table(e)
    g = SHAPES[NAMES[e]]
    np.testing.assert_allclose(d, np.array(g["dN"]), atol=1e-13, rtol=0)
    np.testing.assert_allclose(w, np.array(g["weights"]), rtol=1e-14)


@pytest.mark.parametrize("e", ELEMS)
@pytest.mark.parametrize("cells", [(8, 2, 2), (3, 4, 2), (1, 1, 1)])
def test_mesh_masses_colourings_bit_exact(built, e, cells):
    import octopusengine_b200 as ob
    X1, T1 = O.beam_mesh(e, cells, (1.0, 0.25, 0.5), (0.1, -0.2, 0.3))
    X2, T2 = ob.beam_mesh(e, cells, (1.0, 0.25, 0.5), (0.1, -0.2, 0.3))
    assert np.array_equal(X1, X2) and np.array_equal(T1, T2)
    for dist in (0, 1):
        assert np.array_equal(O.masses(e, X1, T1, 1100.0, dist), ob.lumped_masses(e, X2, T2, 1100.0, dist))
    n = len(X1)
    c1, n1 = O.colour(e, T1, n, 0)
    c2, n2, conf = ob.color(e, T2, n, 0)
    assert n1 == n2 and np.array_equal(c1, c2) and conf == 0
    g1, gn1 = O.colour(e, T1, n, 1)
    g2, gn2, _ = ob.color(e, T2, n, 1)
    assert gn1 == gn2 and np.array_equal(g1, g2)
    for target in (2, max(2, n1 - 2)):
        r1, _ = O.colour(e, T1, n, 0, target=target)
        r2, nr2, conf2 = ob.color(e, T2, n, 0, target)
        assert np.array_equal(r1, r2) and nr2 == target
        assert conf2 == O.conflicts(e, T1, n, r1)
    s1, sn1 = O.colour(e, T1, n, 2)
    s2, sn2, _ = ob.color(e, T2, n, 2)
    assert sn1 == sn2 and np.array_equal(s1, s2)


def test_colouring_rejects_bad_topology(built):
    import octopusengine_b200 as ob
    X, T = ob.beam_mesh(O.TETRA, (2, 1, 1), (1, 1, 1))
    T = T.copy()
    T[0, 0] = len(X) + 5
    with pytest.raises(ob.OctError):
        ob.color(O.TETRA, T, len(X), 0)
    with pytest.raises(ob.OctError):
        ob.beam_mesh(O.TETRA, (0, 1, 1), (1, 1, 1))


def test_large_mesh_colouring_is_fast(built):
    """P2 64x16x16 (config 2 size class): host colouring finishes in seconds."""
    import time
    import octopusengine_b200 as ob
    X, T = ob.beam_mesh(O.TETRA10, (32, 8, 8), (2, 0.5, 0.5))
    t = time.time()
    c, n, conf = ob.color(O.TETRA10, T, len(X), 0)
    assert conf == 0 and n > 0
    assert time.time() - t < 30
