"""ctypes bindings of the CPU oracle (oracle/liboracle.so) for the tests and the CPU
baseline.  The oracle is the checker: nothing in the product imports this module."""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
LIB_PATH = os.path.join(ORACLE_DIR, "liboracle.so")

TETRA, PYRAMID, PRISM, HEXA, TETRA10, TETRA20, HEXA27 = 3, 4, 5, 6, 7, 8, 9
ELEMENT_NODES = {TETRA: 4, HEXA: 8, TETRA10: 10, TETRA20: 20, HEXA27: 27}
HOOKE, STVK, NEOHOOKE, STABLE_NEOHOOKE, COROTATED, FIXED_COROTATED = 0, 1, 2, 3, 4, 5
XPBD_V0, XPBD_QUADRATURE, XPBD_OPTISHARED, XPBD_OPTIGROUP = 0, 1, 2, 3


class OrcDesc(C.Structure):
    _fields_ = [
        ("element", C.c_int32), ("n_nodes", C.c_int32), ("positions", C.POINTER(C.c_float)),
        ("n_elements", C.c_int32), ("topology", C.POINTER(C.c_int32)), ("masses", C.POINTER(C.c_float)),
        ("material", C.c_int32), ("young", C.c_float), ("poisson", C.c_float),
        ("young_per_element", C.POINTER(C.c_float)), ("damping", C.c_float), ("gravity", C.c_float * 3),
        ("n_fixed", C.c_int32), ("fixed_ids", C.POINTER(C.c_int32)), ("fixed_group", C.POINTER(C.c_int32)),
        ("initial_velocity", C.POINTER(C.c_float)),
        ("iterations", C.c_int32), ("rho", C.c_float), ("in_place", C.c_int32), ("n_colors", C.c_int32),
        ("colors", C.POINTER(C.c_int32)), ("order_mode", C.c_int32), ("seed", C.c_uint64),
        ("box_limit", C.c_int32), ("box_min", C.c_float * 3), ("box_max", C.c_float * 3),
        ("global_damping", C.c_float), ("xpbd_version", C.c_int32),
        ("mg_linear", C.c_float), ("mg_masses", C.POINTER(C.c_float)),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
        L = C.CDLL(LIB_PATH)
        vp, ip, fp, dp = C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_double)
        L.orc_beam_counts.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_int)] * 2
        L.orc_beam_mesh.argtypes = [C.c_int] * 4 + [C.c_float] * 6 + [fp, ip]
        L.orc_shape.argtypes = [C.c_int, C.POINTER(C.c_int), dp, dp, dp]
        L.orc_masses.argtypes = [C.c_int, fp, C.c_int, ip, C.c_int, C.c_float, C.c_int, fp]
        L.orc_precompute.argtypes = [C.c_int, fp, ip, C.c_int, C.c_int, dp, dp]
        L.orc_colour.argtypes = [C.c_int, ip, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip]
        L.orc_conflicts.argtypes = [C.c_int, ip, C.c_int, C.c_int, ip]
        for k in ("vbd", "xpbd", "explicit"):
            getattr(L, "orc_%s_create" % k).argtypes = [C.POINTER(OrcDesc), C.c_int]
            getattr(L, "orc_%s_create" % k).restype = vp
            getattr(L, "orc_%s_step" % k).argtypes = [vp, C.c_float, C.c_int]
            getattr(L, "orc_%s_get" % k).argtypes = [vp, C.c_int, dp]
            getattr(L, "orc_%s_destroy" % k).argtypes = [vp]
        L.orc_vbd_set.argtypes = [vp, C.c_int, dp]
        L.orc_set_fixation.argtypes = [vp, C.c_int, fp, fp]
        L.orc_vbd_energy.argtypes = [vp, dp]
        L.orc_vbd_residual.argtypes = [vp, C.c_float, dp]
        L.orc_cpuvbd_create.argtypes = [C.POINTER(OrcDesc)]
        L.orc_cpuvbd_create.restype = vp
        L.orc_cpuvbd_step.argtypes = [vp, C.c_float, C.c_int, C.c_int]
        L.orc_cpuvbd_get.argtypes = [vp, C.c_int, dp]
        L.orc_cpuvbd_destroy.argtypes = [vp]
        L.orc_cpuvbd_run_many.argtypes = [C.POINTER(vp), C.c_int, C.c_float, C.c_int, C.c_int, C.c_int]
        L.orc_cpuvbd_run_many.restype = C.c_double
        L.orc_polar.argtypes = [dp, C.c_int, dp, dp]
        L.orc_element_data.argtypes = [vp, C.c_int, dp]
        L.orc_add_effect.argtypes = [vp, C.c_int, fp, ip, C.c_int]
        L.orc_set_effect_active.argtypes = [vp, C.c_int, C.c_int]
        L.orc_vbd_forces.argtypes = [vp, C.c_float, dp]
        L.orc_xpbd_pair.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, dp, dp, dp]
        L.orc_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def set_threads(n=None):
    """Host threads for one colour's vertices in the oracle's VBD sweep (None: all cores)."""
    lib().orc_set_threads(int(n if n is not None else (os.cpu_count() or 1)))


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


def polar(F, fp64=True):
    """(R, S) of the reference polar decomposition of a 3x3 matrix (row-major numpy in and out)."""
    Fc = np.ascontiguousarray(np.asarray(F, np.float64).T)   # column-major
    R, S = np.zeros(9), np.zeros(9)
    lib().orc_polar(_p(Fc.ravel(), C.c_double), int(fp64), _p(R, C.c_double), _p(S, C.c_double))
    return R.reshape(3, 3).T, S.reshape(3, 3).T


def xpbd_pair(material, m, lam, mu, F):
    """(P, C) of one XPBD constraint of eval_material (row-major numpy in and out)."""
    Fc = np.ascontiguousarray(np.asarray(F, np.float64).T)
    P, c = np.zeros(9), C.c_double()
    rc = lib().orc_xpbd_pair(material, m, lam, mu, _p(Fc.ravel(), C.c_double), _p(P, C.c_double), C.byref(c))
    assert rc == 0
    return P.reshape(3, 3).T, c.value


def beam_mesh(element, cells, size, offset=(0.0, 0.0, 0.0)):
    L = lib()
    nn, ne = C.c_int(), C.c_int()
    if L.orc_beam_counts(element, cells[0], cells[1], cells[2], C.byref(nn), C.byref(ne)):
        raise ValueError("unsupported beam element")
    X = np.zeros((nn.value, 3), np.float32)
    T = np.zeros((ne.value, ELEMENT_NODES[element]), np.int32)
    L.orc_beam_mesh(element, cells[0], cells[1], cells[2], *[float(v) for v in size], *[float(v) for v in offset],
                    _p(X, C.c_float), _p(T, C.c_int32))
    return X, T


def shape(element):
    L = lib()
    nq = C.c_int()
    q = np.zeros(27 * 3)
    w = np.zeros(27)
    d = np.zeros(27 * 27 * 3)
    if L.orc_shape(element, C.byref(nq), _p(q, C.c_double), _p(w, C.c_double), _p(d, C.c_double)):
        raise ValueError("unknown element")
    n = nq.value
    ne = ELEMENT_NODES[element]
    return q[:3 * n].reshape(n, 3), w[:n], d[:n * ne * 3].reshape(n, ne, 3)


def masses(element, X, T, density, distribution):
    m = np.zeros(len(X), np.float32)
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.int32)
    lib().orc_masses(element, _p(X, C.c_float), len(X), _p(T, C.c_int32), len(T), density, distribution, _p(m, C.c_float))
    return m


def precompute(element, X, T, fp64=True):
    nq = shape(element)[1].size
    JX = np.zeros((len(T), nq, 3, 3))
    V = np.zeros((len(T), nq))
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.int32)
    lib().orc_precompute(element, _p(X, C.c_float), _p(T, C.c_int32), len(T), int(fp64), _p(JX, C.c_double), _p(V, C.c_double))
    return JX, V   # JX[e, q, column j, row i]


def colour(element, T, n_nodes, algo=0, target=-1):
    T = np.ascontiguousarray(T, np.int32)
    n = len(T) if algo == 2 else n_nodes
    c = np.zeros(n, np.int32)
    nc = C.c_int32()
    r = lib().orc_colour(element, _p(T, C.c_int32), len(T), n_nodes, algo, target, _p(c, C.c_int32), C.byref(nc))
    if r:
        raise ValueError("colouring failed %d" % r)
    return c, nc.value


def conflicts(element, T, n_nodes, colors):
    T = np.ascontiguousarray(T, np.int32)
    colors = np.ascontiguousarray(colors, np.int32)
    return lib().orc_conflicts(element, _p(T, C.c_int32), len(T), n_nodes, _p(colors, C.c_int32))


class Scene:
    """Holds the numpy arrays an OrcDesc points into, so they outlive the solver."""

    def __init__(self, element, X, T, m, material=STABLE_NEOHOOKE, young=1e5, poisson=0.45, damping=0.0,
                 gravity=(0, 0, -9.81), fixed=(), v0=None, iterations=20, rho=0.0, in_place=False, colors=None,
                 n_colors=0, order_mode=0, seed=0, young_per_element=None, box=None, global_damping=0.0,
                 fixed_group=None, xpbd_version=2, mg_linear=0.0, mg_masses=None):
        self.arrays = dict(X=np.ascontiguousarray(X, np.float32), T=np.ascontiguousarray(T, np.int32),
                           m=np.ascontiguousarray(m, np.float32), fixed=np.ascontiguousarray(fixed, np.int32),
                           v0=None if v0 is None else np.ascontiguousarray(v0, np.float32),
                           colors=None if colors is None else np.ascontiguousarray(colors, np.int32),
                           ype=None if young_per_element is None else np.ascontiguousarray(young_per_element, np.float32),
                           fgroup=None if fixed_group is None else np.ascontiguousarray(fixed_group, np.int32),
                           mgm=None if mg_masses is None else np.ascontiguousarray(mg_masses, np.float32))
        a = self.arrays
        d = OrcDesc()
        d.element = element
        d.n_nodes = len(a["X"])
        d.positions = _p(a["X"], C.c_float)
        d.n_elements = len(a["T"])
        d.topology = _p(a["T"], C.c_int32)
        d.masses = _p(a["m"], C.c_float)
        d.material = material
        d.young = young
        d.poisson = poisson
        d.young_per_element = _p(a["ype"], C.c_float)
        d.damping = damping
        d.gravity = (C.c_float * 3)(*gravity)
        d.n_fixed = len(a["fixed"])
        d.fixed_ids = _p(a["fixed"], C.c_int32) if len(a["fixed"]) else None
        d.fixed_group = _p(a["fgroup"], C.c_int32)
        d.initial_velocity = _p(a["v0"], C.c_float)
        d.iterations = iterations
        d.rho = rho
        d.in_place = int(in_place)
        d.n_colors = n_colors
        d.colors = _p(a["colors"], C.c_int32)
        d.order_mode = order_mode
        d.seed = seed
        if box is not None:
            d.box_limit = 1
            d.box_min = (C.c_float * 3)(*box[0])
            d.box_max = (C.c_float * 3)(*box[1])
        d.global_damping = global_damping
        d.xpbd_version = xpbd_version
        d.mg_linear = mg_linear
        d.mg_masses = _p(a["mgm"], C.c_float)
        self.desc = d
        self.n = d.n_nodes


class Solver:
    def __init__(self, kind, scene, fp64=False):
        self.kind = kind
        self.scene = scene
        L = lib()
        self.h = getattr(L, "orc_%s_create" % kind)(C.byref(scene.desc), int(fp64))
        if not self.h:
            raise ValueError("oracle %s create failed" % kind)

    def step(self, frame_dt, substeps=1):
        getattr(lib(), "orc_%s_step" % self.kind)(self.h, frame_dt, substeps)

    def get(self, what=0):
        out = np.zeros((self.scene.n, 3)) if what != 4 else np.zeros(self.scene.n)
        getattr(lib(), "orc_%s_get" % self.kind)(self.h, what, _p(out, C.c_double))
        return out

    def set_fixation(self, offset=(0, 0, 0), rotation=None, group=0):
        off = np.asarray(offset, np.float32)
        rot = np.eye(3, dtype=np.float32) if rotation is None else np.asarray(rotation, np.float32)
        rot = np.ascontiguousarray(rot.T)
        lib().orc_set_fixation(self.h, group, _p(off, C.c_float), _p(rot, C.c_float))

    def energy(self):
        e = np.zeros(4)
        lib().orc_vbd_energy(self.h, _p(e, C.c_double))
        return e

    def add_effect(self, kind, params=(0.0, 0.0), ids=()):
        p = np.asarray(list(params) + [0.0] * 2, np.float32)
        i = np.ascontiguousarray(ids, np.int32)
        k = lib().orc_add_effect(self.h, kind, _p(p, C.c_float), _p(i, C.c_int32) if len(i) else None, len(i))
        assert k >= 0
        return k

    def set_effect_active(self, index, active=True):
        assert lib().orc_set_effect_active(self.h, index, int(active)) == 0

    def set(self, what, values):
        """VBD state write (what: 0 p, 1 v, 2 last_p, 3 y)."""
        a = np.ascontiguousarray(values, np.float64)
        assert lib().orc_vbd_set(self.h, what, _p(a, C.c_double)) == 0

    def element_data(self, kind):
        out = np.zeros(self.scene.desc.n_elements)
        assert lib().orc_element_data(self.h, kind, _p(out, C.c_double)) == 0
        return out

    def forces(self, dt):
        out = np.zeros((self.scene.n, 3))
        assert lib().orc_vbd_forces(self.h, dt, _p(out, C.c_double)) == 0
        return out

    def residual(self, dt):
        r = np.zeros(2)
        lib().orc_vbd_residual(self.h, dt, _p(r, C.c_double))
        return r

    def __del__(self):
        try:
            if self.h:
                getattr(lib(), "orc_%s_destroy" % self.kind)(self.h)
        except Exception:
            pass


class CpuVBD:
    """The reference's CPU VBD path (single-thread Gauss-Seidel), restated."""

    def __init__(self, scene):
        self.scene = scene
        self.h = lib().orc_cpuvbd_create(C.byref(scene.desc))
        if not self.h:
            raise ValueError("cpu vbd create failed")

    def step(self, frame_dt, substeps=1, residual_pass=True):
        lib().orc_cpuvbd_step(self.h, frame_dt, substeps, int(residual_pass))

    def get(self, what=0):
        out = np.zeros((self.scene.n, 3))
        lib().orc_cpuvbd_get(self.h, what, _p(out, C.c_double))
        return out

    def __del__(self):
        try:
            lib().orc_cpuvbd_destroy(self.h)
        except Exception:
            pass


def run_cpu_many(solvers, frame_dt, substeps, residual_pass=True, threads=1):
    arr = (C.c_void_p * len(solvers))(*[s.h for s in solvers])
    return lib().orc_cpuvbd_run_many(arr, len(solvers), frame_dt, substeps, int(residual_pass), threads)


def fixed_by_plane(X, origin, normal):
    """Area::Plane::inside (Tools/Area.h:52-54): dot(p - o, n) > 0, evaluated in float32."""
    X = np.asarray(X, np.float32)
    d = ((X - np.float32(origin)) * np.float32(normal)).astype(np.float32)
    s = (d[:, 0] + d[:, 1]) + d[:, 2]
    return np.nonzero(s > 0)[0].astype(np.int32)
