"""ctypes binding of liboctb.so (the C ABI declared in include/octopus_b200.h).

There is no fallback: if the library is missing or a CUDA device is absent, the calls
raise.  The compute runs in the library's own CUDA kernels.
"""
import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "liboctb.so")

OK, EINVAL, ENOMEM_BUDGET, ETIMEDOUT, ENUMERIC, ECUDA, ENOTSUP = range(7)
STATUS = {0: "OCT_OK", 1: "OCT_EINVAL", 2: "OCT_ENOMEM_BUDGET", 3: "OCT_ETIMEDOUT", 4: "OCT_ENUMERIC",
          5: "OCT_ECUDA", 6: "OCT_ENOTSUP"}
TETRA, HEXA, TETRA10, TETRA20, HEXA27 = 3, 6, 7, 8, 9
ELEMENT_NODES = {TETRA: 4, HEXA: 8, TETRA10: 10, TETRA20: 20, HEXA27: 27}
ELEMENT_QUADRATURE = {TETRA: 1, HEXA: 8, TETRA10: 4, TETRA20: 11, HEXA27: 27}
HOOKE, STVK, NEOHOOKE, STABLE_NEOHOOKE, COROTATED, FIXED_COROTATED = 0, 1, 2, 3, 4, 5
XPBD_XPBD, XPBD_QUADRATURE, XPBD_OPTISHARED, XPBD_OPTIGROUP = 0, 1, 2, 3
DIAG_STRESS, DIAG_VOLUME, DIAG_VOLUME_DIFF, DIAG_INVERTED, DIAG_STRESS_ACCUMULATED = 0, 1, 2, 3, 4
DIAG_VOLUME_ACCUMULATED, DIAG_VOLUME_DIFF_ACCUMULATED = 5, 6
EFFECT_CRUSH, EFFECT_RANDOM_SPHERE, EFFECT_HIGH_STRETCH = 0, 1, 2
MASS_UNIFORM, MASS_FEMSHAPE = 0, 1
SOLVER_VBD, SOLVER_XPBD, SOLVER_EXPLICIT = 0, 1, 2
VBD_BASE, VBD_THREADED_QUADRATURE, VBD_REDUCTION_SYMMETRY, VBD_BETTER_COLORATION = 0, 1, 2, 3
COLOR_DSAT, COLOR_GREEDY = 0, 1
ORDER_ASCENDING, ORDER_SHUFFLED = 0, 1
PREC_PLAIN, PREC_MIXED = 0, 1

EXPORTS = [
    "oct_ctx_create", "oct_ctx_destroy", "oct_last_error", "oct_ctx_memory", "oct_desc_init",
    "oct_scene_create", "oct_scene_destroy", "oct_scene_step", "oct_scene_sync", "oct_scene_set_capture",
    "oct_scene_get_positions",
    "oct_scene_get_velocities", "oct_scene_set_positions", "oct_scene_set_velocities", "oct_scene_info",
    "oct_scene_get_coloring", "oct_scene_get_masses", "oct_scene_set_fixation", "oct_scene_energy",
    "oct_scene_residual", "oct_batch_create", "oct_batch_step", "oct_batch_destroy", "oct_batch_set_state",
    "oct_batch_get_state", "oct_batch_state_size", "oct_beam_mesh", "oct_lumped_masses", "oct_shape_table",
    "oct_color", "oct_last_step_ms", "oct_launch_count", "oct_ctx_stream", "oct_fp32_peak",
    "oct_batch_group_info", "oct_batch_time_group", "oct_scene_set_precision", "oct_scene_footprint",
    "oct_server_create", "oct_server_submit", "oct_server_tick", "oct_server_poll", "oct_server_get_stats",
    "oct_server_destroy", "oct_elastic_energy_noalloc", "oct_scene_set_fixation_group",
    "oct_scene_element_data", "oct_scene_vertex_residuals", "oct_scene_set_mapping", "oct_scene_get_mapping", "oct_autotune_mapping",
    "oct_batch_prepare", "oct_scene_element_type", "oct_scene_get_rest_positions", "oct_scene_get_topology",
    "oct_scene_metadata_json", "oct_vtk_write", "oct_vtk_read_mesh", "oct_vtk_read_field", "oct_scene_write_vtk",
    "oct_shape_values", "oct_reference_nodes", "oct_mesh_error", "oct_beam_sampler_create", "oct_beam_sampler_info",
    "oct_beam_sampler_error", "oct_beam_sampler_destroy", "oct_flexion_error", "oct_torsion_profile",
    "oct_scene_add_effect", "oct_scene_set_effect_active", "oct_scene_effect_ids", "oct_surface_nodes",
    "oct_scene_state_size", "oct_scene_save", "oct_scene_restore", "oct_ctx_wait_probe",
    "oct_scene_status", "oct_batch_status",
]


class VtkField(C.Structure):
    _fields_ = [("name", C.c_char_p), ("location", C.c_int32), ("components", C.c_int32), ("data", C.POINTER(C.c_float))]


VTK_POINT, VTK_CELL = 0, 1


class ServerConfig(C.Structure):
    _fields_ = [("hbm_budget", C.c_size_t), ("max_scenes", C.c_int32), ("frame_dt", C.c_float),
                ("substeps", C.c_int32), ("iterations", C.c_int32), ("precision", C.c_int32),
                ("setup_threads", C.c_int32)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("admitted", C.c_int64), ("finished", C.c_int64),
                ("rejected", C.c_int64), ("queued", C.c_int64), ("active", C.c_int64), ("frames", C.c_int64),
                ("p50_step_ms", C.c_double), ("p99_step_ms", C.c_double), ("mean_step_ms", C.c_double),
                ("vertex_iterations", C.c_double), ("busy_ms", C.c_double), ("bytes_in_use", C.c_size_t),
                ("gap_ms", C.c_double), ("failed", C.c_int64)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("solver", C.c_int32), ("element", C.c_int32), ("n_nodes", C.c_int32), ("positions", C.POINTER(C.c_float)),
        ("n_elements", C.c_int32), ("topology", C.POINTER(C.c_int32)), ("masses", C.POINTER(C.c_float)),
        ("density", C.c_float), ("mass_distribution", C.c_int32), ("material", C.c_int32),
        ("young", C.c_float), ("poisson", C.c_float), ("young_per_element", C.POINTER(C.c_float)),
        ("damping", C.c_float), ("gravity", C.c_float * 3), ("n_fixed", C.c_int32),
        ("fixed_ids", C.POINTER(C.c_int32)), ("fixed_group", C.POINTER(C.c_int32)), ("fix_by_plane", C.c_int32), ("plane_origin", C.c_float * 3),
        ("plane_normal", C.c_float * 3), ("initial_velocity", C.POINTER(C.c_float)), ("iterations", C.c_int32),
        ("rho", C.c_float), ("vbd_version", C.c_int32), ("target_color", C.c_int32), ("color_algo", C.c_int32),
        ("order_mode", C.c_int32), ("seed", C.c_uint64), ("global_damping", C.c_float), ("precision", C.c_int32),
        ("box_limit", C.c_int32), ("box_min", C.c_float * 3), ("box_max", C.c_float * 3),
        ("threads_per_vertex", C.c_int32), ("xpbd_version", C.c_int32), ("mg_linear", C.c_float),
    ]


class OctError(RuntimeError):
    def __init__(self, status, where, detail=""):
        self.status = status
        super().__init__("%s failed: %s %s" % (where, STATUS.get(status, status), detail))


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("liboctb.so is not built (run octopusengine_b200.build.build())")
        L = C.CDLL(LIB_PATH)
        vp, ip, fp, dp = C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_float), C.POINTER(C.c_double)
        pp = C.POINTER(C.c_void_p)
        sig = {
            "oct_ctx_create": ([C.c_int, C.c_size_t, pp], C.c_int),
            "oct_ctx_destroy": ([vp], C.c_int),
            "oct_last_error": ([vp], C.c_char_p),
            "oct_ctx_memory": ([vp, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)], C.c_int),
            "oct_desc_init": ([C.POINTER(SceneDesc)], None),
            "oct_scene_create": ([vp, C.POINTER(SceneDesc), pp], C.c_int),
            "oct_scene_destroy": ([vp], C.c_int),
            "oct_scene_step": ([vp, C.c_float, C.c_int], C.c_int),
            "oct_scene_sync": ([vp], C.c_int),
            "oct_scene_set_capture": ([vp, C.c_int], C.c_int),
            "oct_scene_element_data": ([vp, C.c_int, C.POINTER(C.c_float)], C.c_int),
            "oct_scene_set_mapping": ([vp, C.c_int], C.c_int),
            "oct_scene_get_mapping": ([vp, ip], C.c_int),
            "oct_batch_prepare": ([vp, C.c_float, C.c_int], C.c_int),
            "oct_scene_element_type": ([vp, C.POINTER(C.c_int32)], C.c_int),
            "oct_scene_get_rest_positions": ([vp, C.POINTER(C.c_float)], C.c_int),
            "oct_scene_get_topology": ([vp, C.POINTER(C.c_int32)], C.c_int),
            "oct_scene_metadata_json": ([vp, C.c_char_p, C.c_size_t, C.POINTER(C.c_size_t)], C.c_int),
            "oct_vtk_write": ([C.c_char_p, C.POINTER(C.c_float), C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.c_int32,
                               C.POINTER(VtkField), C.c_int32], C.c_int),
            "oct_vtk_read_mesh": ([C.c_char_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_float), C.POINTER(C.c_int32)], C.c_int),
            "oct_vtk_read_field": ([C.c_char_p, C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.c_float)], C.c_int),
            "oct_scene_write_vtk": ([vp, C.c_char_p], C.c_int),
            "oct_shape_values": ([C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
            "oct_scene_add_effect": ([vp, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_int32)], C.c_int),
            "oct_scene_state_size": ([vp, C.POINTER(C.c_size_t)], C.c_int),
            "oct_scene_save": ([vp, C.POINTER(C.c_float)], C.c_int),
            "oct_scene_restore": ([vp, C.POINTER(C.c_float)], C.c_int),
            "oct_ctx_wait_probe": ([vp, C.c_int32], C.c_int),
            "oct_scene_set_effect_active": ([vp, C.c_int32, C.c_int], C.c_int),
            "oct_scene_effect_ids": ([vp, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)], C.c_int),
            "oct_surface_nodes": ([C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
                                  C.c_int),
            "oct_reference_nodes": ([C.c_int32, C.POINTER(C.c_double)], C.c_int),
            "oct_mesh_error": ([C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32, C.POINTER(C.c_float),
                                C.POINTER(C.c_double)], C.c_int),
            "oct_beam_sampler_create": ([C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.POINTER(C.c_float)),
                                         C.POINTER(C.c_int32), C.POINTER(C.POINTER(C.c_int32)), C.c_int32, C.c_int32,
                                         C.POINTER(vp)], C.c_int),
            "oct_beam_sampler_info": ([vp, C.POINTER(C.c_int32)], C.c_int),
            "oct_beam_sampler_error": ([vp, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_double)],
                                       C.c_int),
            "oct_beam_sampler_destroy": ([vp], C.c_int),
            "oct_flexion_error": ([C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32, C.POINTER(C.c_float),
                                   C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int32)], C.c_int),
            "oct_torsion_profile": ([C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32, C.POINTER(C.c_int32),
                                     C.c_int32, C.c_int32, C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32,
                                     C.POINTER(C.c_int32)], C.c_int),
            "oct_autotune_mapping": ([vp, C.POINTER(vp), C.c_int, C.c_float, C.c_int, C.POINTER(C.c_int32)], C.c_int),
            "oct_scene_vertex_residuals": ([vp, C.c_float, C.POINTER(C.c_float)], C.c_int),
            "oct_scene_get_positions": ([vp, fp], C.c_int),
            "oct_scene_get_velocities": ([vp, fp], C.c_int),
            "oct_scene_set_positions": ([vp, fp], C.c_int),
            "oct_scene_set_velocities": ([vp, fp], C.c_int),
            "oct_scene_info": ([vp, ip, ip, ip, ip], C.c_int),
            "oct_scene_get_coloring": ([vp, ip, ip], C.c_int),
            "oct_scene_get_masses": ([vp, fp], C.c_int),
            "oct_scene_set_fixation": ([vp, fp, fp], C.c_int),
            "oct_scene_set_fixation_group": ([vp, C.c_int, fp, fp], C.c_int),
            "oct_scene_energy": ([vp, dp], C.c_int),
            "oct_scene_residual": ([vp, C.c_float, dp], C.c_int),
            "oct_batch_create": ([vp, pp, C.c_int, pp], C.c_int),
            "oct_batch_step": ([vp, C.c_float, C.c_int], C.c_int),
            "oct_batch_destroy": ([vp], C.c_int),
            "oct_scene_status": ([vp], C.c_int),
            "oct_batch_status": ([vp, ip], C.c_int),
            "oct_batch_set_state": ([vp, fp], C.c_int),
            "oct_batch_get_state": ([vp, fp], C.c_int),
            "oct_batch_state_size": ([vp, C.POINTER(C.c_size_t)], C.c_int),
            "oct_beam_mesh": ([C.c_int, C.c_int, C.c_int, C.c_int, fp, fp, ip, ip, fp, ip], C.c_int),
            "oct_lumped_masses": ([C.c_int, fp, C.c_int, ip, C.c_int, C.c_float, C.c_int, fp], C.c_int),
            "oct_shape_table": ([C.c_int, ip, dp, dp, dp], C.c_int),
            "oct_color": ([C.c_int, ip, C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, C.POINTER(C.c_int64)], C.c_int),
            "oct_last_step_ms": ([vp, fp], C.c_int),
            "oct_launch_count": ([vp, C.POINTER(C.c_uint64)], C.c_int),
            "oct_ctx_stream": ([vp, pp], C.c_int),
            "oct_fp32_peak": ([vp, dp], C.c_int),
            "oct_batch_group_info": ([vp, C.c_int, ip, ip, dp, dp, ip, C.POINTER(C.c_int64)], C.c_int),
            "oct_batch_time_group": ([vp, C.c_int, C.c_int, C.c_float, fp], C.c_int),
            "oct_scene_set_precision": ([vp, C.c_int], C.c_int),
            "oct_scene_footprint": ([C.POINTER(SceneDesc), C.POINTER(C.c_size_t)], C.c_int),
            "oct_server_create": ([vp, C.POINTER(ServerConfig), pp], C.c_int),
            "oct_server_submit": ([vp, C.POINTER(SceneDesc), C.c_int32, C.POINTER(C.c_int64)], C.c_int),
            "oct_server_tick": ([vp, ip], C.c_int),
            "oct_server_poll": ([vp, C.c_int64, ip, fp], C.c_int),
            "oct_server_get_stats": ([vp, C.POINTER(ServerStats)], C.c_int),
            "oct_server_destroy": ([vp], C.c_int),
            "oct_elastic_energy_noalloc": ([C.c_int, C.c_int, vp, vp, vp, C.c_int, C.c_float, C.c_float, vp, vp],
                                           C.c_int),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def ptr(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def check(status, where, ctx=None):
    if status != OK:
        detail = ""
        if ctx is not None:
            try:
                detail = lib().oct_last_error(ctx).decode()
            except Exception:
                pass
        raise OctError(status, where, detail)


# ----------------------------------------------------------------------------- host helpers
def beam_mesh(element, cells, size, offset=(0.0, 0.0, 0.0)):
    L = lib()
    nn, ne = C.c_int32(0), C.c_int32(0)
    sz = np.asarray(size, np.float32)
    off = np.asarray(offset, np.float32)
    check(L.oct_beam_mesh(element, cells[0], cells[1], cells[2], ptr(sz, C.c_float), ptr(off, C.c_float),
                          C.byref(nn), C.byref(ne), None, None), "oct_beam_mesh")
    X = np.zeros((nn.value, 3), np.float32)
    T = np.zeros((ne.value, ELEMENT_NODES[element]), np.int32)
    check(L.oct_beam_mesh(element, cells[0], cells[1], cells[2], ptr(sz, C.c_float), ptr(off, C.c_float),
                          C.byref(nn), C.byref(ne), ptr(X, C.c_float), ptr(T, C.c_int32)), "oct_beam_mesh")
    return X, T


def surface_nodes(element, T):
    T = np.ascontiguousarray(T, np.int32)
    n = C.c_int32()
    check(lib().oct_surface_nodes(element, ptr(T, C.c_int32), len(T), None, C.byref(n)), "oct_surface_nodes")
    out = np.zeros(n.value, np.int32)
    check(lib().oct_surface_nodes(element, ptr(T, C.c_int32), len(T), ptr(out, C.c_int32), C.byref(n)), "oct_surface_nodes")
    return out


def vtk_write(path, element, X, T, point_fields=(), cell_fields=()):
    """VTK 5.1 ASCII file of one mesh; fields are (name, array) with 1 or 3 values per point/cell."""
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.int32)
    keep, fs = [], []
    for loc, group in ((VTK_POINT, point_fields), (VTK_CELL, cell_fields)):
        for name, a in group:
            a = np.ascontiguousarray(a, np.float32)
            keep.append(a)
            comps = 3 if a.ndim == 2 and a.shape[1] == 3 else 1
            fs.append(VtkField(name.encode(), loc, comps, ptr(a, C.c_float)))
    arr = (VtkField * max(len(fs), 1))(*fs)
    check(lib().oct_vtk_write(path.encode(), ptr(X, C.c_float), len(X), element, ptr(T, C.c_int32), len(T), arr, len(fs)),
          "oct_vtk_write")


def vtk_read(path):
    """(element, X, T) of a VTK 5.1 ASCII unstructured grid with one element type."""
    e, nn, ne = C.c_int32(), C.c_int32(), C.c_int32()
    check(lib().oct_vtk_read_mesh(path.encode(), C.byref(e), C.byref(nn), C.byref(ne), None, None), "oct_vtk_read_mesh")
    X = np.zeros((nn.value, 3), np.float32)
    T = np.zeros((ne.value, ELEMENT_NODES.get(e.value, 1)), np.int32)
    check(lib().oct_vtk_read_mesh(path.encode(), C.byref(e), C.byref(nn), C.byref(ne), ptr(X, C.c_float),
                                  ptr(T, C.c_int32)), "oct_vtk_read_mesh")
    return e.value, X, T


def vtk_read_field(path, name, n, components=1):
    out = np.zeros((n, components) if components == 3 else n, np.float32)
    check(lib().oct_vtk_read_field(path.encode(), name.encode(), components, n, ptr(out, C.c_float)), "oct_vtk_read_field")
    return out


ERROR_KEYS = ("MSE", "RMSE", "MAE", "max", "L1", "L2")


def shape_values(element, x):
    N = np.zeros(ELEMENT_NODES[element])
    xx = np.ascontiguousarray(x, np.float64)
    check(lib().oct_shape_values(element, ptr(xx, C.c_double), ptr(N, C.c_double)), "oct_shape_values")
    return N


def reference_nodes(element):
    X = np.zeros((ELEMENT_NODES[element], 3))
    check(lib().oct_reference_nodes(element, ptr(X, C.c_double)), "oct_reference_nodes")
    return X


def mesh_error(a, b, offset=None):
    """MeshDiff_MSE error between two same-topology node sets: dict MSE, RMSE, MAE, max, L1, L2."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    out = np.zeros(6)
    off = None if offset is None else np.ascontiguousarray(offset, np.float32)
    check(lib().oct_mesh_error(ptr(a, C.c_float), ptr(b, C.c_float), len(a), ptr(off, C.c_float) if off is not None else None,
                               ptr(out, C.c_double)), "oct_mesh_error")
    return dict(zip(ERROR_KEYS, out))


class BeamSampler:
    """Beam_MSE_Sampling over meshes [(element, rest X, T), ...] against meshes[reference]."""

    def __init__(self, meshes, reference=0, nb_sample=4):
        self._keep = [(np.ascontiguousarray(X, np.float32), np.ascontiguousarray(T, np.int32)) for _, X, T in meshes]
        n = len(meshes)
        el = (C.c_int32 * n)(*[e for e, _, _ in meshes])
        nn = (C.c_int32 * n)(*[len(X) for X, _ in self._keep])
        ne = (C.c_int32 * n)(*[len(T) for _, T in self._keep])
        xs = (C.POINTER(C.c_float) * n)(*[ptr(X, C.c_float) for X, _ in self._keep])
        ts = (C.POINTER(C.c_int32) * n)(*[ptr(T, C.c_int32) for _, T in self._keep])
        self._h = C.c_void_p()
        check(lib().oct_beam_sampler_create(n, el, nn, xs, ne, ts, reference, nb_sample, C.byref(self._h)),
              "oct_beam_sampler_create")
        k = C.c_int32()
        lib().oct_beam_sampler_info(self._h, C.byref(k))
        self.n_samples = k.value

    def error(self, mesh, positions, reference_positions):
        p = np.ascontiguousarray(positions, np.float32)
        r = np.ascontiguousarray(reference_positions, np.float32)
        out = np.zeros(6)
        check(lib().oct_beam_sampler_error(self._h, mesh, ptr(p, C.c_float), ptr(r, C.c_float), ptr(out, C.c_double)),
              "oct_beam_sampler_error")
        return dict(zip(ERROR_KEYS, out))

    def close(self):
        if self._h:
            lib().oct_beam_sampler_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def flexion_error(rest, current, follow, target):
    rest = np.ascontiguousarray(rest, np.float32)
    cur = np.ascontiguousarray(current, np.float32)
    f = np.ascontiguousarray(follow, np.float32)
    t = np.ascontiguousarray(target, np.float32)
    err, pid = C.c_double(), C.c_int32()
    check(lib().oct_flexion_error(ptr(rest, C.c_float), ptr(cur, C.c_float), len(rest), ptr(f, C.c_float),
                                  ptr(t, C.c_float), C.byref(err), C.byref(pid)), "oct_flexion_error")
    return err.value, pid.value


def torsion_profile(element, rest, current, T, samples_per_edge, beam_length):
    rest = np.ascontiguousarray(rest, np.float32)
    cur = np.ascontiguousarray(current, np.float32)
    T = np.ascontiguousarray(T, np.int32)
    n = C.c_int32()
    args = (element, ptr(rest, C.c_float), ptr(cur, C.c_float), len(rest), ptr(T, C.c_int32), len(T), samples_per_edge,
            beam_length)
    check(lib().oct_torsion_profile(*args, None, None, 0, C.byref(n)), "oct_torsion_profile")
    d, a = np.zeros(n.value, np.float32), np.zeros(n.value, np.float32)
    check(lib().oct_torsion_profile(*args, ptr(d, C.c_float), ptr(a, C.c_float), n.value, C.byref(n)), "oct_torsion_profile")
    return d, a


def lumped_masses(element, X, T, density, distribution=MASS_FEMSHAPE):
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.int32)
    m = np.zeros(len(X), np.float32)
    check(lib().oct_lumped_masses(element, ptr(X, C.c_float), len(X), ptr(T, C.c_int32), len(T), density,
                                  distribution, ptr(m, C.c_float)), "oct_lumped_masses")
    return m


def shape_table(element):
    nq = ELEMENT_QUADRATURE[element]
    ne = ELEMENT_NODES[element]
    q = np.zeros(nq * 3)
    w = np.zeros(nq)
    d = np.zeros(nq * ne * 3)
    n = C.c_int32(0)
    check(lib().oct_shape_table(element, C.byref(n), ptr(q, C.c_double), ptr(w, C.c_double), ptr(d, C.c_double)),
          "oct_shape_table")
    return q.reshape(nq, 3), w, d.reshape(nq, ne, 3)


def color(element, T, n_nodes, algo=COLOR_DSAT, target=-1):
    T = np.ascontiguousarray(T, np.int32)
    n = len(T) if algo == 2 else n_nodes
    c = np.zeros(n, np.int32)
    nc = C.c_int32(0)
    conf = C.c_int64(0)
    check(lib().oct_color(element, ptr(T, C.c_int32), len(T), n_nodes, algo, target, ptr(c, C.c_int32),
                          C.byref(nc), C.byref(conf)), "oct_color")
    return c, nc.value, conf.value


def fixed_by_plane(X, origin, normal):
    """Nodes with dot(p - origin, normal) > 0 in float32 (Area::Plane::inside)."""
    X = np.asarray(X, np.float32)
    d = ((X - np.float32(origin)) * np.float32(normal)).astype(np.float32)
    return np.nonzero((d[:, 0] + d[:, 1]) + d[:, 2] > 0)[0].astype(np.int32)
