"""The reference's own numbers at the end states of its static-flexion runs, and the checks that
compare a solver with them (shared by the oracle test and the GPU test).

``golden/reference_static.npz`` (written by ``golden/make_reference_static.py`` from the 16
result files ``assets/result/vtk/References/*_32_8_8_4x1x1_*.vtk``) holds, per file, the
displacement ``u`` the reference's simulation reached and the per-element ``stress``, ``volume``
and ``volume_diff`` its GPU_FEM kernels (octopus/src/GPU/GPU_FEM.cu:20-85) evaluated there.
The scene is BaseScene's beam (octopus/include/Scene/BaseScene.h:34-51,72-73,157-166): 4 x 1 x 1 m,
32 x 8 x 8 cells, nodes with x < 0.01 fixed, gravity -9.81 y, density 1000 with FemShape masses,
Stable Neo-Hookean with the file's Young modulus and Poisson ratio.

What the fields pin, and how closely they can:
  * ``volume`` / ``volume_diff``: the shape-function derivatives, the quadrature weights, the rest
    volumes V and the mesh.  The files carry the volume with the Jacobian accumulated over the
    quadrature points (as kernel_compute_stress accumulates it), so they are compared with that
    form.  Printed to 6 digits, so 5e-4 relative per element.
  * ``stress``: the material's PK1 stress, its Cauchy form and von Mises norm, JX_inv.  The
    accumulated Jacobian makes F grow with the point index, and for Hexa27 (27 points) and the
    stiffer files the von Mises norm of the reference's FP32 evaluation is dominated by
    rounding of a large hydrostatic part: the FP32 and FP64 evaluations of the same formula
    differ by a median 30 % to 1600 % there.  The bar is therefore per file: the error
    against the file may not exceed the spread between the FP32 and the FP64 evaluation of the
    formula (median and 90th percentile) plus the printing error.
  * ``u`` at static equilibrium: the elastic force of the solver balances gravity.  With u
    printed to 6 digits the force residual itself is dominated by rounding for the stiff
    files, so the check is the virtual work along the reference's own displacement,
    W(a) = sum_free r(X + a u) . u / sum_free |m g . u| with r = f_elastic + m g: the
    reference's state is the stationary point, W(a*) = 0, at a* = 1 to within STATIONARY_TOL,
    while W(0.98) and W(1.02) are of order one.
"""
import hashlib
import os
import struct

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = np.load(os.path.join(HERE, "golden", "reference_static.npz"))
NAMES = sorted({k.split("/")[0] for k in FIXTURE.files})
CELLS, SIZE = (32, 8, 8), (4.0, 1.0, 1.0)
DENSITY = 1000.0
GRAVITY = (0.0, -9.81, 0.0)
FIX_X = 0.01
STATIONARY_TOL = 2.5e-3
VOLUME_RTOL = 5e-4
PRINT_RTOL = 2e-4
ALPHAS = (0.98, 1.0, 1.02)


def case(name):
    meta = FIXTURE[name + "/meta"]
    return dict(name=name, element=int(meta[0]), young=float(meta[1]), poisson=float(meta[2]),
                origin=tuple(float(v) for v in meta[3:6]), n_points=int(meta[6]), n_elements=int(meta[7]),
                topology_sha256=str(FIXTURE[name + "/topology_sha256"]),
                u=FIXTURE[name + "/u"].astype(np.float64),
                stress=FIXTURE[name + "/stress"].astype(np.float64),
                volume=FIXTURE[name + "/volume"].astype(np.float64),
                volume_diff=FIXTURE[name + "/volume_diff"].astype(np.float64))


def topology_sha256(T):
    flat = np.ascontiguousarray(T, np.int32).ravel().tolist()
    return hashlib.sha256(struct.pack("<%di" % len(flat), *flat)).hexdigest()


def fixed_ids(X):
    return np.where(np.asarray(X)[:, 0] < FIX_X)[0].astype(np.int32)


def check_volumes(c, volume, volume_diff):
    """Accumulated-Jacobian volume and volume change against the file."""
    rel = np.abs(volume - c["volume"]) / np.abs(c["volume"])
    assert rel.max() < VOLUME_RTOL, (c["name"], rel.max())
    # volume_diff is a difference of near-equal printed numbers for the linear elements
    err = np.abs(volume_diff - c["volume_diff"]).max() / np.abs(c["volume_diff"]).max()
    assert err < 2e-3, (c["name"], err)
    return float(rel.max()), float(err)


def check_stress(c, stress, stress64, stress32):
    """Stress against the file, within the FP32-vs-FP64 spread of the reference's formula."""
    err = np.abs(stress - c["stress"]) / np.abs(c["stress"])
    spread = np.abs(stress32 - stress64) / np.abs(stress64)
    med, p90 = np.median(err), np.percentile(err, 90)
    assert med <= np.median(spread) + PRINT_RTOL, (c["name"], med, np.median(spread))
    assert p90 <= 1.2 * np.percentile(spread, 90) + 1e-2, (c["name"], p90, np.percentile(spread, 90))
    return float(med), float(p90)


def virtual_work(r, u, m, free):
    g = np.asarray(GRAVITY)
    den = np.abs((m[:, None] * g * u)[free].sum(1)).sum()
    return float((r * u)[free].sum() / den)


def stationary_point(works):
    """Root nearest 1 of the quadratic through W(0.98), W(1), W(1.02)."""
    p = np.polyfit(ALPHAS, works, 2)
    roots = np.roots(p)
    roots = roots[np.abs(roots.imag) < 1e-12].real
    return float(roots[np.argmin(np.abs(roots - 1.0))])


def check_stationary(c, works):
    a = stationary_point(works)
    assert abs(a - 1.0) < STATIONARY_TOL, (c["name"], a, works)
    assert works[0] > 0.0 > works[2], (c["name"], works)   # a minimum of the energy along u
    return a
