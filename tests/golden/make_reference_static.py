"""Generate ``reference_static.npz``: the fields OctopusEngine itself computed and wrote into its
result files ``assets/result/vtk/References/{1_Tetra,2_Hexa,3_Tetra10,4_Hexa27}_32_8_8_4x1x1_
{1e6,1e7}_{045,049}.vtk`` (16 files).

Each file is one 4 x 1 x 1 m beam of 32 x 8 x 8 cells (P1 6-tet split, Q1, P2, Q2), fixed at
x < 0.01 and hanging under gravity -y (BaseScene.h:34-51,72-73,157-166), Stable Neo-Hookean with
the Young modulus and Poisson ratio of the file name, density 1000 and FemShape masses.  The
recorder (FEM_VTK_Recorder::save, octopus/src/Script/Record/Recorder.cpp:117-168) wrote the rest
mesh, the masses ("weights"), the displacement ``u`` of the reference's simulated end state, and
per element the ``stress`` / ``volume`` / ``volume_diff`` the reference's GPU_FEM kernels
(octopus/src/GPU/GPU_FEM.cu:20-85) evaluated at that state.

The script parses the ASCII text only (it runs no reference code) and stores, per file:
  * ``<name>/u``           n_points x 3 float32 (the printed 6-digit values)
  * ``<name>/stress``, ``<name>/volume``, ``<name>/volume_diff``   n_elements float32
  * ``<name>/meta``        [element id, young, poisson, origin x, y, z, n_points, n_elements]
  * ``<name>/topology_sha256``  SHA-256 of the connectivity (little-endian int32) in the
                           reference's node order (the writer's Hexa27 reorder undone)
so that the tests can rebuild the same beam with the product's mesh generator, put it in the
reference's state and compare the product's own kernels with the reference's numbers.

Usage (build container only; OCTOPUS_REFERENCE overrides the mount point):
    python tests/golden/make_reference_static.py
"""
import glob
import hashlib
import os
import struct
import sys

import numpy as np

REF = os.environ.get("OCTOPUS_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))
ELEMENT = {"Tetra": 3, "Hexa": 6, "Tetra10": 7, "Hexa27": 9}
VTK_CELL = {10: 3, 12: 6, 24: 7, 29: 9}
# The writer swaps these Hexa27 node positions (VTK_Formater.cpp:55-90: VTK's tri-quadratic
# hexahedron orders the mid-edge and face nodes differently); a swap table is its own inverse.
HEXA27_VTK_SWAP = {20: 24, 24: 20, 21: 22, 22: 21, 12: 16, 16: 12, 13: 17, 17: 13, 14: 18, 18: 14, 15: 19, 19: 15}


def _read(path):
    tok = open(path).read().split()
    i = tok.index("POINTS")
    n = int(tok[i + 1])
    X = np.array(tok[i + 3:i + 3 + 3 * n], np.float64).reshape(n, 3)
    i = tok.index("OFFSETS")
    ne = int(tok[tok.index("CELLS") + 1]) - 1
    off = np.array(tok[i + 2:i + 2 + ne + 1], np.int64)
    i = tok.index("CONNECTIVITY")
    conn = np.array(tok[i + 2:i + 2 + off[-1]], np.int64)
    i = tok.index("CELL_TYPES")
    types = set(int(t) for t in tok[i + 2:i + 2 + ne])
    assert len(types) == 1, "one element type per file"
    element = VTK_CELL[types.pop()]
    nen = int(off[1] - off[0])
    T = conn.reshape(ne, nen)

    def field(name, comps, count):
        j = tok.index(name)
        # "SCALARS name float 1 LOOKUP_TABLE default v..." or "VECTORS name float v..."
        k = j + (5 if tok[j - 1] == "SCALARS" else 2)
        return np.array(tok[k:k + comps * count], np.float64).reshape(count, comps) if comps > 1 else \
            np.array(tok[k:k + count], np.float64)

    return element, X, T, field


def main():
    d = os.path.join(REF, "assets/result/vtk/References")
    if not os.path.isdir(d):
        sys.exit("reference tree not found at %s" % REF)
    out = {}
    for path in sorted(glob.glob(os.path.join(d, "*_32_8_8_4x1x1_*.vtk"))):
        name = os.path.basename(path)[:-4]
        element, X, T, field = _read(path)
        if element == 9:
            T = T[:, [HEXA27_VTK_SWAP.get(k, k) for k in range(27)]]
        parts = name.split("_")
        young, poisson = float(parts[-2]), float("0." + parts[-1][1:])
        flat = T.astype(np.int32).ravel().tolist()
        out[name + "/topology_sha256"] = np.array(hashlib.sha256(struct.pack("<%di" % len(flat), *flat)).hexdigest())
        out[name + "/meta"] = np.array([element, young, poisson, X[0, 0], X[0, 1], X[0, 2], len(X), len(T)], np.float64)
        out[name + "/u"] = field("u", 3, len(X)).astype(np.float32)
        for k in ("stress", "volume", "volume_diff"):
            out[name + "/" + k] = field(k, 1, len(T)).astype(np.float32)
        print(name, element, len(X), len(T))
    np.savez_compressed(os.path.join(HERE, "reference_static.npz"), **out)


if __name__ == "__main__":
    main()
