"""VTK 5.1 ASCII files (VTK_Formater / VTK_Loader / FEM_VTK_Recorder): the writer reproduces
the reference's own output byte for byte (mesh section and mass block of the reference result
files, pinned by hashes in tests/golden/meshes.json), the reader undoes the Hexa27 node order,
and a written scene frame reads back (GPU test)."""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle_lib as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "meshes.json")))
ELEM = {"Tetra": O.TETRA, "Hexa": O.HEXA, "Tetra10": O.TETRA10, "Hexa27": O.HEXA27}
REFERENCE = os.environ.get("OCTOPUS_REFERENCE", "")   # the reference tree, when mounted (reader test only)


def _sections(path):
    text = open(path, "rb").read()
    a, b = text.index(b"DATASET UNSTRUCTURED_GRID"), text.index(b"POINT_DATA")
    c = text.index(b"SCALARS weights float 1")
    e = text.index(b"\n", text.index(b"LOOKUP_TABLE default", c) + 21) + 1
    return text[a:b], text[c:e]


@pytest.mark.parametrize("name", list(GOLDEN))
def test_writer_reproduces_reference_files(built, tmp_path, name):
    import octopusengine_b200 as ob
    g = GOLDEN[name]
    e = ELEM[name]
    X, T = ob.beam_mesh(e, g["cells"], g["size"], g["origin"])
    m = ob.lumped_masses(e, X, T, g["density"], ob.MASS_FEMSHAPE)
    path = str(tmp_path / ("%s.vtk" % name))
    ob.vtk_write(path, e, X, T, point_fields=[("weights", m)])
    mesh, weights = _sections(path)
    assert hashlib.sha256(mesh).hexdigest() == g["mesh_text_sha256"]
    if name == "Tetra":
        # P1 shape derivatives are exact small integers, so the FemShape masses match the
        # reference's bit for bit and so does the printed block
        assert hashlib.sha256(weights).hexdigest() == g["weights_text_sha256"]
    else:
        # higher-order dN at the quadrature points differ from the reference's FP32 evaluation in
        # the last bit, which moves some masses by ~1e-6 (a few printed last digits)
        w = ob.vtk_read_field(path, "weights", len(X), 1)
        np.testing.assert_allclose(w[::g["point_stride"]], g["mass_sample"], rtol=1e-5)


@pytest.mark.parametrize("element", [O.TETRA, O.HEXA, O.TETRA10, O.TETRA20, O.HEXA27])
def test_round_trip(built, tmp_path, element):
    import octopusengine_b200 as ob
    X, T = ob.beam_mesh(element, (3, 2, 2), (0.75, 0.5, 0.5))
    rng = np.random.default_rng(element)
    u = rng.normal(0, 1, X.shape).astype(np.float32)
    s = rng.normal(0, 1, len(T)).astype(np.float32)
    path = str(tmp_path / "rt.vtk")
    ob.vtk_write(path, element, X, T, point_fields=[("u", u)], cell_fields=[("stress", s)])
    e2, X2, T2 = ob.vtk_read(path)
    assert e2 == element
    np.testing.assert_array_equal(T2, T)
    np.testing.assert_allclose(X2, X, rtol=1e-5, atol=1e-7)   # 6 significant digits, as the reference writes
    np.testing.assert_allclose(ob.vtk_read_field(path, "u", len(X), 3), u, rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(ob.vtk_read_field(path, "stress", len(T), 1), s, rtol=1e-5, atol=1e-6)
    if element == O.HEXA27:   # written in VTK's node order, not the reference's
        text = open(path).read().split("CONNECTIVITY vtktypeint64\n")[1].split("\n")[0].split()
        assert [int(v) for v in text] != list(T[0])


@pytest.mark.skipif(not REFERENCE or not os.path.isdir(REFERENCE), reason="OCTOPUS_REFERENCE not set")
@pytest.mark.parametrize("name", list(GOLDEN))
def test_reader_on_reference_files(built, name):
    import struct

    import octopusengine_b200 as ob
    g = GOLDEN[name]
    path = os.path.join(REFERENCE, g["source"])
    e, X, T = ob.vtk_read(path)
    assert e == ELEM[name] and len(X) == g["n_points"] and len(T) == g["n_elements"]
    flat = T.ravel().tolist()
    assert hashlib.sha256(struct.pack("<%di" % len(flat), *flat)).hexdigest() == g["topology_sha256"]
    w = ob.vtk_read_field(path, "weights", len(X), 1)
    np.testing.assert_allclose(w[::g["point_stride"]], g["mass_sample"], rtol=1e-6)
    u = ob.vtk_read_field(path, "u", len(X), 3)
    assert np.isfinite(u).all() and np.abs(u).max() > 0


@pytest.mark.gpu
def test_scene_frame_reads_back(ctx, tmp_path):
    import octopusengine_b200 as ob
    from scenes import pair
    s, o32, o64, mesh = pair(ctx, O.HEXA27, cells=(2, 1, 1), young=3e4)
    s.step(1 / 60, 2)
    path = str(tmp_path / "frame.vtk")
    s.write_vtk(path)
    e, X, T = ob.vtk_read(path)
    np.testing.assert_array_equal(T, mesh["T"])
    np.testing.assert_allclose(X, mesh["X"], rtol=1e-6, atol=1e-7)
    u = ob.vtk_read_field(path, "u", len(X), 3)
    ref = s.get_position() - mesh["X"]
    assert np.abs(u - ref).max() <= 1e-5 * np.abs(ref).max()
    np.testing.assert_allclose(ob.vtk_read_field(path, "weights", len(X)), s.masses(), rtol=1e-5)
    for name, kind in (("stress", ob.capi.DIAG_STRESS_ACCUMULATED), ("volume", ob.capi.DIAG_VOLUME),
                       ("inverted", ob.capi.DIAG_INVERTED)):
        got = ob.vtk_read_field(path, name, len(T))
        np.testing.assert_allclose(got, s.element_data(kind), rtol=1e-5, atol=1e-12)
    meta = s.metadata()
    assert meta["mesh"] == {"Hexa27": len(T), "vertices": len(X)}
    assert meta["fem"]["material"] == "Stable Neo-Hooke" and meta["fem"]["sub_step"] == 2
