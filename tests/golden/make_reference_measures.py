"""Generate ``reference_measures.npz``: the states OctopusEngine wrote in its torsion and
small-step experiments, for the tests of the accuracy measures on the reference's own data.

Sources (ASCII VTK text only; no reference code is run):
  * ``assets/result/vtk/VBD_Torsion_all/{P1,Q1}_Torsion.vtk``: a 2 x 1 x 1 m beam of
    16 x 8 x 8 cells (P1 6-tet split and Q1), twisted about its axis by the rigid controller
    (FEM_Torsion_error_recorder's experiment, octopus/src/Script/Record/Recorder.cpp:222-309);
  * ``assets/result/vtk/VBD Small Steps/{1..7,ref}_Hexa_16_4_4_4x1x1*.vtk``: a 4 x 1 x 1 m Q1 beam
    of 16 x 4 x 4 cells after 60 s, stepped with 60 sub-steps x 1 iteration ... 1 x 60 and a
    reference run (the MeshDiff_MSE experiment, octopus/include/Script/Measure/MeshDiff.h:64-83).
Per file: ``<name>/u`` (displacement, float32), ``<name>/meta`` [element, cells x3, size x3,
origin x3] and ``<name>/topology_sha256`` (little-endian int32 connectivity).

Usage (build container only; OCTOPUS_REFERENCE overrides the mount point):
    python tests/golden/make_reference_measures.py
"""
import glob
import hashlib
import os
import struct
import sys

import numpy as np

from make_reference_static import REF, _read

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    root = os.path.join(REF, "assets/result/vtk")
    if not os.path.isdir(root):
        sys.exit("reference tree not found at %s" % REF)
    files = [("torsion_P1", "VBD_Torsion_all/P1_Torsion.vtk", (16, 8, 8), (2.0, 1.0, 1.0)),
             ("torsion_Q1", "VBD_Torsion_all/Q1_Torsion.vtk", (16, 8, 8), (2.0, 1.0, 1.0))]
    for path in sorted(glob.glob(os.path.join(root, "VBD Small Steps", "*_Hexa_16_4_4_4x1x1*.vtk"))):
        base = os.path.basename(path)[:-4]
        if "Graphic" in base:
            continue
        files.append(("small_steps_" + base.split("_")[0] + ("_" + "_".join(base.split("_")[-2:]) if base[0] != "r" else ""),
                      os.path.relpath(path, root), (16, 4, 4), (4.0, 1.0, 1.0)))
    out = {}
    for name, rel, cells, size in files:
        element, X, T, field = _read(os.path.join(root, rel))
        flat = T.astype(np.int32).ravel().tolist()
        out[name + "/topology_sha256"] = np.array(hashlib.sha256(struct.pack("<%di" % len(flat), *flat)).hexdigest())
        out[name + "/meta"] = np.array([element, *cells, *size, *X[0]], np.float64)
        out[name + "/u"] = field("u", 3, len(X)).astype(np.float32)
        print(name, rel, element, len(X), len(T))
    np.savez_compressed(os.path.join(HERE, "reference_measures.npz"), **out)


if __name__ == "__main__":
    main()
