"""Generate the golden fixtures under tests/golden/ from the OctopusEngine sources.

This script is the only committed code that reads the reference tree, and it runs
only where that tree is mounted (the build container).  It never compiles or runs
reference code: it reads two kinds of text.

1. ``octopus/include/Dynamic/FEM/FEM_Shape.h`` — the shape-function derivative
   expressions, quadrature coordinates and weights of Tetra_4 (:36-66),
   Pyramid_5 (:69-125), Prism_6 (:127-173), Hexa_8 (:175-224), Tetra_10 (:227-272),
   Tetra_20 (:274-482) and Hexa_27 (:483-690).  The C++ initializer lists are
   evaluated in IEEE double by Python (the expressions are plain arithmetic), and the
   post-scaling loops of Prism_6 (x0.5) and Hexa_8 (x1/8) are applied.  Output:
   ``shapes.json`` with, per element, the quadrature points, weights and dN[q][i][3].

2. ``assets/result/vtk/References/*_1e6_045.vtk`` — meshes the reference's own
   beam generator wrote (TetraBeamGenerator 6-tet split, HexaBeamGenerator,
   tetra4_to_tetra10, hexa_to_hexa27, and the FemShape lumped masses as the
   ``weights`` point field).  Output: ``meshes.json`` with the SHA-256 of the
   connectivity in the reference's internal node order (the VTK writer's Hexa27
   reorder, VTK_Formater.cpp:55-90, is undone), the point count, a subsample of the
   points and of the masses, and the mass total.

Usage (build container only):  python tests/golden/make_golden.py
"""
import hashlib
import json
import math
import os
import re
import sys

# The reference tree; OCTOPUS_REFERENCE overrides the build container's mount point.
REF = os.environ.get("OCTOPUS_REFERENCE", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))


# --------------------------------------------------------------------------- shapes
def _strip_comments(src):
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return re.sub(r"//[^\n]*", "", src)


def _struct_body(src, name):
    m = re.search(r"struct\s+%s\b[^{]*\{" % name, src)
    if not m:
        raise RuntimeError("struct %s not found" % name)
    i = m.end()
    depth = 1
    while depth:
        c = src[i]
        depth += (c == "{") - (c == "}")
        i += 1
    return src[m.end():i - 1]


def _func_body(body, fname):
    m = re.search(r"%s\s*\(([^)]*)\)[^{]*\{" % fname, body)
    if not m:
        raise RuntimeError("function %s not found" % fname)
    params = [p.strip().split()[-1] for p in m.group(1).split(",") if p.strip()]
    i = m.end()
    depth = 1
    while depth:
        c = body[i]
        depth += (c == "{") - (c == "}")
        i += 1
    return params, body[m.end():i - 1]


def _split_top(s):
    out, depth, cur = [], 0, ""
    for c in s:
        if c in "([{":
            depth += 1
        elif c in ")]}":
            depth -= 1
        if c == "," and depth == 0:
            out.append(cur)
            cur = ""
        else:
            cur += c
    if cur.strip():
        out.append(cur)
    return [x.strip() for x in out if x.strip()]


def _py_expr(e):
    e = " ".join(e.split())
    e = re.sub(r"(\d+\.\d*|\d*\.\d+|\d+)f\b", r"\1", e)           # float suffix
    e = e.replace("std::sqrt", "math.sqrt").replace("sqrt", "math.sqrt")
    e = e.replace("math.math.sqrt", "math.sqrt")
    e = re.sub(r"static_cast<\w+>", "", e)
    return e


def _eval(e, env):
    return float(eval(_py_expr(e), {"math": math}, dict(env)))


def _locals(body, env):
    """Evaluate `scalar name = expr;` / `constexpr scalar ...` declarations in order."""
    for m in re.finditer(r"(?:constexpr\s+)?(?:const\s+)?scalar\s+([^;]+);", body):
        for decl in _split_top(m.group(1)):
            if "=" not in decl:
                continue
            name, expr = decl.split("=", 1)
            name = name.strip()
            if "[" in name:
                continue
            env[name] = _eval(expr, env)
    return env


def _init_list(body):
    m = re.search(r"\{(.*)\}", body, flags=re.S)
    return _split_top(m.group(1))


def extract_shapes():
    src = _strip_comments(open(os.path.join(REF, "octopus/include/Dynamic/FEM/FEM_Shape.h")).read())
    spec = {  # struct, element enum value, nodes, post-scale of dN
        "Tetra": ("Tetra_4", 3, 4, 1.0),
        "Pyramid": ("Pyramid_5", 4, 5, 1.0),
        "Prism": ("Prism_6", 5, 6, 0.5),
        "Hexa": ("Hexa_8", 6, 8, 1.0 / 8.0),
        "Tetra10": ("Tetra_10", 7, 10, 1.0),
        "Tetra20": ("Tetra_20", 8, 20, 1.0),
        "Hexa27": ("Hexa_27", 9, 27, 1.0),
    }
    out = {}
    for key, (struct, enum, nb, scale) in spec.items():
        body = _struct_body(src, struct)
        # quadrature coordinates
        _, qb = _func_body(body, "get_quadrature_coordinates")
        env = _locals(qb, {})
        if "std::vector(3, 0.25" in qb.replace(" ", "").replace("std::vector(3,0.25", "std::vector(3, 0.25"):
            coords = [0.25, 0.25, 0.25]
        else:
            ret = qb[qb.index("return") if "return" in qb and "{" in qb[qb.index("return"):] else 0:]
            if "coords" in qb and "return coords" in qb:
                lst = re.search(r"coords\s*=\s*\{(.*?)\};", qb, flags=re.S).group(1)
            else:
                lst = re.search(r"return\s*\{(.*?)\};", qb, flags=re.S).group(1)
            coords = [_eval(x, env) for x in _split_top(lst)]
        # weights
        _, wb = _func_body(body, "get_weights")
        wenv = _locals(wb, {})
        mv = re.search(r"std::vector(?:<scalar>)?\((\d+),\s*([^;]+)\);", wb)
        if mv and "{" not in wb.split("return", 1)[1].split(";")[0]:
            n = int(mv.group(1))
            weights = [_eval(mv.group(2), wenv)] * n
        else:
            lst = re.search(r"(?:w\s*=\s*|return\s*)\{(.*?)\};", wb, flags=re.S).group(1)
            weights = [_eval(x, wenv) for x in _split_top(lst)]
        nq = len(weights)
        assert len(coords) == 3 * nq, (key, len(coords), nq)
        # derivatives
        params, db = _func_body(body, "build_shape_derivatives")
        terms = _init_list(re.search(r"dN\s*\[[^\]]*\]\s*(=\s*)?\{.*?\};", db, flags=re.S).group(0))
        assert len(terms) == 3 * nb, (key, len(terms))
        dN = []
        for q in range(nq):
            env = dict(zip(params, coords[3 * q:3 * q + 3]))
            vals = [_eval(t, env) * scale for t in terms]
            # convert_dN_to_vector3 (FEM_Shape.cpp:18-28): component d of node i at i + d*nb
            dN.append([[vals[i], vals[i + nb], vals[i + 2 * nb]] for i in range(nb)])
        out[key] = {"element": enum, "nodes": nb, "quadrature": [coords[3 * q:3 * q + 3] for q in range(nq)],
                    "weights": weights, "dN": dN}
    return out


# --------------------------------------------------------------------------- meshes
HEXA27_VTK_SWAP = {20: 24, 24: 20, 21: 22, 22: 21, 12: 16, 16: 12, 13: 17, 17: 13, 14: 18, 18: 14, 15: 19, 19: 15}


def read_vtk(path):
    lines = open(path).read().split("\n")
    i = 0
    pts, conn, offs, weights = [], [], [], []
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("POINTS"):
            n = int(ln.split()[1])
            vals = []
            i += 1
            while len(vals) < 3 * n:
                vals += [float(v) for v in lines[i].split()]
                i += 1
            pts = [vals[3 * k:3 * k + 3] for k in range(n)]
            continue
        if ln.startswith("OFFSETS"):
            i += 1
            while not lines[i].startswith("CONNECTIVITY"):
                offs += [int(v) for v in lines[i].split()]
                i += 1
            continue
        if ln.startswith("CONNECTIVITY"):
            i += 1
            while not lines[i].startswith("CELL_TYPES"):
                conn += [int(v) for v in lines[i].split()]
                i += 1
            continue
        if ln.startswith("SCALARS weights"):
            i += 2
            while len(weights) < len(pts):
                weights += [float(v) for v in lines[i].split()]
                i += 1
            continue
        i += 1
    return pts, conn, offs, weights


def extract_meshes():
    d = os.path.join(REF, "assets/result/vtk/References")
    spec = [("1_Tetra_32_8_8_4x1x1_1e6_045.vtk", "Tetra", 4),
            ("2_Hexa_32_8_8_4x1x1_1e6_045.vtk", "Hexa", 8),
            ("3_Tetra10_32_8_8_4x1x1_1e6_045.vtk", "Tetra10", 10),
            ("4_Hexa27_32_8_8_4x1x1_1e6_045.vtk", "Hexa27", 27)]
    out = {}
    for fname, elem, ne in spec:
        pts, conn, offs, weights = read_vtk(os.path.join(d, fname))
        assert len(conn) % ne == 0
        topo = list(conn)
        if elem == "Hexa27":
            topo = []
            for c in range(len(conn) // 27):
                cell = conn[27 * c:27 * c + 27]
                topo += [cell[HEXA27_VTK_SWAP.get(k, k)] for k in range(27)]
        import struct
        blob = struct.pack("<%di" % len(topo), *topo)
        text = open(os.path.join(d, fname), "rb").read()
        a = text.index(b"DATASET UNSTRUCTURED_GRID")
        b = text.index(b"POINT_DATA")
        c = text.index(b"SCALARS weights float 1")
        e = text.index(b"\n", text.index(b"LOOKUP_TABLE default", c) + 21) + 1   # end of the values line
        step = 97
        out[elem] = {
            "source": "assets/result/vtk/References/" + fname,
            "cells": [32, 8, 8], "size": [4.0, 1.0, 1.0], "density": 1000.0, "distribution": "FemShape",
            "n_points": len(pts), "n_elements": len(topo) // ne,
            "topology_sha256": hashlib.sha256(blob).hexdigest(),
            "topology_head": topo[:4 * ne],
            "origin": pts[0],
            "point_stride": step,
            "points_sample": pts[::step],
            "mass_sample": weights[::step],
            "mass_sum": sum(weights),
            # the reference's own VTK text (VTK_Formater::save_mesh and the masses block of
            # FEM_VTK_Recorder::save): a writer with the same formatting reproduces it byte for byte
            "mesh_text_sha256": hashlib.sha256(text[a:b]).hexdigest(),
            "weights_text_sha256": hashlib.sha256(text[c:e]).hexdigest(),
        }
    return out


def main():
    if not os.path.isdir(REF):
        sys.exit("reference tree not mounted; the committed fixtures stand")
    shapes = extract_shapes()
    with open(os.path.join(HERE, "shapes.json"), "w") as f:
        json.dump(shapes, f, separators=(",", ":"))
    meshes = extract_meshes()
    with open(os.path.join(HERE, "meshes.json"), "w") as f:
        json.dump(meshes, f, separators=(",", ":"))
    print("wrote shapes.json (%s) and meshes.json (%s)" % (", ".join(shapes), ", ".join(meshes)))


if __name__ == "__main__":
    main()
