"""octopusengine_b200 — Blackwell-native soft-body FEM time step (VBD / XPBD / explicit).

Python host-side handle on the C ABI (include/octopus_b200.h).  The classes mirror the
reference's GPU solver objects and their host caller:

    Context                 one device, one stream, one HBM budget
    Scene                   GPU_ParticleSystem + GPU_VBD / GPU_PBD / GPU_SemiExplicit +
                            GPU_VBD_FEM / GPU_PBD_FEM / GPU_FEM_Explicit + GPU_Fix_Constraint
                            (octopus/include/Script/Dynamic/Cuda_FEM_Dynamic.h:18-25)
    Scene.step(dt, n)       Cuda_ParticleSystem_Dynamics::update: n sub-steps of dt/n
                            (octopus/src/Script/Dynamic/Cuda_ParticleSystem_Dynamic.cpp:17-31)
    Scene.get_position()    GPU_ParticleSystem::get_position (octopus/include/GPU/GPU_ParticleSystem.h:54-61)
    Batch                   many VBD scenes stepped by one launch per (element type, colour)

Errors raise OctError with the library's status, as the C ABI returns it.
"""
import ctypes as C

import numpy as np

from . import capi
from .capi import (COLOR_DSAT, COLOR_GREEDY, COROTATED, DIAG_INVERTED, DIAG_STRESS, DIAG_STRESS_ACCUMULATED,
                   DIAG_VOLUME, DIAG_VOLUME_ACCUMULATED, DIAG_VOLUME_DIFF, DIAG_VOLUME_DIFF_ACCUMULATED,
                   ELEMENT_NODES, FIXED_COROTATED, HEXA, HEXA27, HOOKE,
                   MASS_FEMSHAPE, MASS_UNIFORM, NEOHOOKE, ORDER_ASCENDING, ORDER_SHUFFLED, PREC_MIXED, PREC_PLAIN,
                   SOLVER_EXPLICIT, SOLVER_VBD, SOLVER_XPBD, STABLE_NEOHOOKE, STVK, TETRA, TETRA10, TETRA20, VBD_BASE,
                   VBD_BETTER_COLORATION, VBD_REDUCTION_SYMMETRY, XPBD_OPTIGROUP, XPBD_OPTISHARED, XPBD_QUADRATURE,
                   XPBD_XPBD, OctError, beam_mesh, color, fixed_by_plane, lumped_masses, shape_table, vtk_read,
                   vtk_read_field, vtk_write)

__all__ = ["Context", "Scene", "Batch", "Server", "make_desc", "autotune_mapping", "vtk_read", "vtk_read_field", "vtk_write", "OctError", "beam_mesh", "color", "lumped_masses", "shape_table",
           "fixed_by_plane", "library_path"]


def library_path():
    return capi.LIB_PATH


class Context:
    def __init__(self, device=0, hbm_budget=0):
        self._h = C.c_void_p()
        capi.check(capi.lib().oct_ctx_create(device, hbm_budget, C.byref(self._h)), "oct_ctx_create")
        self._objs = []

    @property
    def handle(self):
        return self._h

    def memory(self):
        used, budget = C.c_size_t(), C.c_size_t()
        capi.check(capi.lib().oct_ctx_memory(self._h, C.byref(used), C.byref(budget)), "oct_ctx_memory")
        return used.value, budget.value

    def last_step_ms(self):
        v = C.c_float()
        capi.lib().oct_last_step_ms(self._h, C.byref(v))
        return v.value

    def launch_count(self):
        v = C.c_uint64()
        capi.lib().oct_launch_count(self._h, C.byref(v))
        return v.value

    def close(self):
        if self._h:
            for o in reversed(self._objs):
                o.close()
            self._objs = []
            capi.lib().oct_ctx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_desc(element, positions, topology, **kw):
    """Builds an oct_scene_desc; returns (desc, arrays kept alive while the desc is used)."""
    X = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
    T = np.ascontiguousarray(topology, np.int32).reshape(-1, ELEMENT_NODES[element])
    d = capi.SceneDesc()
    capi.lib().oct_desc_init(C.byref(d))
    keep = [X, T]
    d.element = element
    d.n_nodes = len(X)
    d.positions = capi.ptr(X, C.c_float)
    d.n_elements = len(T)
    d.topology = capi.ptr(T, C.c_int32)
    for k, v in kw.items():
        if k in ("masses", "young_per_element", "initial_velocity"):
            a = np.ascontiguousarray(v, np.float32).ravel()
            keep.append(a)
            setattr(d, k, capi.ptr(a, C.c_float))
        elif k == "fixed_ids":
            a = np.ascontiguousarray(v, np.int32).ravel()
            keep.append(a)
            d.fixed_ids = capi.ptr(a, C.c_int32) if len(a) else None
            d.n_fixed = len(a)
        elif k == "fixed_group":
            a = np.ascontiguousarray(v, np.int32).ravel()
            keep.append(a)
            d.fixed_group = capi.ptr(a, C.c_int32) if len(a) else None
        elif k in ("gravity", "plane_origin", "plane_normal", "box_min", "box_max"):
            setattr(d, k, (C.c_float * 3)(*v))
        else:
            setattr(d, k, v)
    return d, keep


class Scene:
    """One simulated object.  Keyword arguments map 1:1 onto oct_scene_desc fields."""

    def __init__(self, ctx, element, positions, topology, **kw):
        self.ctx = ctx
        d, keep = make_desc(element, positions, topology, **kw)
        self._h = C.c_void_p()
        capi.check(capi.lib().oct_scene_create(ctx.handle, C.byref(d), C.byref(self._h)), "oct_scene_create",
                   ctx.handle)
        ctx._objs.append(self)
        nn, ne, nc, nf = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        capi.lib().oct_scene_info(self._h, C.byref(nn), C.byref(ne), C.byref(nc), C.byref(nf))
        self.n_nodes, self.n_elements, self.n_colors, self.n_fixed = nn.value, ne.value, nc.value, nf.value
        self.element = element
        self.solver = kw.get("solver", SOLVER_VBD)

    @property
    def handle(self):
        return self._h

    def set_mapping(self, threads_per_vertex):
        """Lane mapping of the vertex kernel (-1 packed, 0 default, 1..32 lanes per vertex)."""
        capi.check(capi.lib().oct_scene_set_mapping(self._h, int(threads_per_vertex)), "oct_scene_set_mapping",
                   self.ctx.handle)

    def mapping(self):
        """Lane mapping in effect (-1 packed, else lanes per vertex; 0 for XPBD scenes)."""
        t = C.c_int32()
        capi.check(capi.lib().oct_scene_get_mapping(self._h, C.byref(t)), "oct_scene_get_mapping", self.ctx.handle)
        return t.value

    def set_capture(self, on=True):
        """Replay each frame's sub-steps from a captured CUDA graph (oct_scene_set_capture)."""
        capi.check(capi.lib().oct_scene_set_capture(self._h, int(on)), "oct_scene_set_capture", self.ctx.handle)

    def step(self, frame_dt, substeps=1, sync=True):
        capi.check(capi.lib().oct_scene_step(self._h, frame_dt, substeps), "oct_scene_step", self.ctx.handle)
        if sync:
            self.sync()

    def sync(self):
        capi.check(capi.lib().oct_scene_sync(self._h), "oct_scene_sync", self.ctx.handle)

    def _get(self, fn):
        out = np.zeros((self.n_nodes, 3), np.float32)
        capi.check(fn(self._h, capi.ptr(out, C.c_float)), fn.__name__, self.ctx.handle)
        return out

    def get_position(self):
        return self._get(capi.lib().oct_scene_get_positions)

    def get_velocity(self):
        return self._get(capi.lib().oct_scene_get_velocities)

    def set_position(self, p):
        p = np.ascontiguousarray(p, np.float32)
        capi.check(capi.lib().oct_scene_set_positions(self._h, capi.ptr(p, C.c_float)), "oct_scene_set_positions")

    def set_velocity(self, v):
        v = np.ascontiguousarray(v, np.float32)
        capi.check(capi.lib().oct_scene_set_velocities(self._h, capi.ptr(v, C.c_float)), "oct_scene_set_velocities")

    def coloring(self):
        c = np.zeros(self.n_nodes, np.int32)
        o = np.zeros(self.n_nodes, np.int32)
        capi.check(capi.lib().oct_scene_get_coloring(self._h, capi.ptr(c, C.c_int32), capi.ptr(o, C.c_int32)),
                   "oct_scene_get_coloring")
        return c, o

    def masses(self):
        m = np.zeros(self.n_nodes, np.float32)
        capi.check(capi.lib().oct_scene_get_masses(self._h, capi.ptr(m, C.c_float)), "oct_scene_get_masses")
        return m

    def set_fixation(self, offset=(0, 0, 0), rotation=None, group=0):
        off = np.asarray(offset, np.float32)
        rot = np.eye(3, dtype=np.float32) if rotation is None else np.asarray(rotation, np.float32)
        rot = np.ascontiguousarray(rot.T)   # column-major
        capi.check(capi.lib().oct_scene_set_fixation_group(self._h, group, capi.ptr(off, C.c_float),
                                                           capi.ptr(rot, C.c_float)), "oct_scene_set_fixation_group")

    def set_precision(self, precision):
        capi.check(capi.lib().oct_scene_set_precision(self._h, precision), "oct_scene_set_precision")

    def energy(self):
        e = np.zeros(4)
        capi.check(capi.lib().oct_scene_energy(self._h, capi.ptr(e, C.c_double)), "oct_scene_energy",
                   self.ctx.handle)
        return e

    def save(self):
        """Checkpoint of the scene state (oct_scene_save)."""
        n = C.c_size_t()
        capi.lib().oct_scene_state_size(self._h, C.byref(n))
        out = np.zeros(n.value, np.float32)
        capi.check(capi.lib().oct_scene_save(self._h, capi.ptr(out, C.c_float)), "oct_scene_save", self.ctx.handle)
        return out

    def restore(self, state):
        a = np.ascontiguousarray(state, np.float32)
        capi.check(capi.lib().oct_scene_restore(self._h, capi.ptr(a, C.c_float)), "oct_scene_restore", self.ctx.handle)

    def add_effect(self, kind, *params):
        """Scripted effect (capi.EFFECT_*), created inactive; returns its index."""
        idx = C.c_int32()
        p = np.asarray(params if params else [0.0], np.float32)
        capi.check(capi.lib().oct_scene_add_effect(self._h, kind, capi.ptr(p, C.c_float), C.byref(idx)),
                   "oct_scene_add_effect", self.ctx.handle)
        return idx.value

    def set_effect_active(self, index, active=True):
        capi.check(capi.lib().oct_scene_set_effect_active(self._h, index, int(active)), "oct_scene_set_effect_active",
                   self.ctx.handle)

    def effect_ids(self, index):
        n = C.c_int32()
        capi.check(capi.lib().oct_scene_effect_ids(self._h, index, None, C.byref(n)), "oct_scene_effect_ids")
        out = np.zeros(n.value, np.int32)
        capi.check(capi.lib().oct_scene_effect_ids(self._h, index, capi.ptr(out, C.c_int32), C.byref(n)),
                   "oct_scene_effect_ids")
        return out

    def write_vtk(self, path):
        """One FEM_VTK_Recorder frame of this scene (oct_scene_write_vtk)."""
        capi.check(capi.lib().oct_scene_write_vtk(self._h, path.encode()), "oct_scene_write_vtk", self.ctx.handle)

    def metadata(self):
        """Run metadata (mesh counts, material) as the reference's recorders write it, parsed."""
        import json
        n = C.c_size_t()
        capi.check(capi.lib().oct_scene_metadata_json(self._h, None, 0, C.byref(n)), "oct_scene_metadata_json")
        buf = C.create_string_buffer(n.value + 1)
        capi.check(capi.lib().oct_scene_metadata_json(self._h, buf, n.value + 1, C.byref(n)), "oct_scene_metadata_json")
        return json.loads(buf.value.decode())

    def topology(self):
        out = np.zeros((self.n_elements, ELEMENT_NODES[self.element]), np.int32)
        capi.check(capi.lib().oct_scene_get_topology(self._h, capi.ptr(out, C.c_int32)), "oct_scene_get_topology")
        return out

    def status(self):
        """Failure state of the scene's own steps (oct_scene_status): the oct_status value."""
        return capi.lib().oct_scene_status(self._h)

    def element_data(self, kind):
        """Per-element diagnostic (capi.DIAG_STRESS / VOLUME / VOLUME_DIFF / INVERTED)."""
        out = np.zeros(self.n_elements, np.float32)
        capi.check(capi.lib().oct_scene_element_data(self._h, kind, capi.ptr(out, C.c_float)),
                   "oct_scene_element_data", self.ctx.handle)
        return out

    def vertex_residuals(self, dt):
        """Per-vertex VBD residual force for sub-step dt (GPU_VBD_FEM::get_forces)."""
        out = np.zeros((self.n_nodes, 3), np.float32)
        capi.check(capi.lib().oct_scene_vertex_residuals(self._h, dt, capi.ptr(out, C.c_float)),
                   "oct_scene_vertex_residuals", self.ctx.handle)
        return out

    def residual(self, dt):
        r = np.zeros(2)
        capi.check(capi.lib().oct_scene_residual(self._h, dt, capi.ptr(r, C.c_double)), "oct_scene_residual",
                   self.ctx.handle)
        return r

    def close(self):
        if self._h:
            capi.lib().oct_scene_destroy(self._h)
            self._h = C.c_void_p()


def autotune_mapping(ctx, scenes, dt, sweeps=3):
    """Times every lane mapping per element type over the scenes and keeps the fastest
    (oct_autotune_mapping); returns {element: mapping} (-1 = packed pairs)."""
    arr = (C.c_void_p * len(scenes))(*[s.handle.value for s in scenes])
    chosen = (C.c_int32 * 10)()
    capi.check(capi.lib().oct_autotune_mapping(ctx.handle, arr, len(scenes), dt, sweeps, chosen),
               "oct_autotune_mapping", ctx.handle)
    present = {s.element for s in scenes}
    return {e: int(chosen[e]) for e in present}


class Batch:
    """Many VBD scenes stepped together (one launch per element type and colour, CUDA graph)."""

    def __init__(self, ctx, scenes):
        self.ctx = ctx
        self.scenes = list(scenes)
        arr = (C.c_void_p * len(self.scenes))(*[s.handle.value for s in self.scenes])
        self._h = C.c_void_p()
        capi.check(capi.lib().oct_batch_create(ctx.handle, arr, len(self.scenes), C.byref(self._h)),
                   "oct_batch_create", ctx.handle)
        ctx._objs.append(self)
        n = C.c_size_t()
        capi.lib().oct_batch_state_size(self._h, C.byref(n))
        self.state_size = n.value

    def step(self, frame_dt, substeps=1):
        capi.check(capi.lib().oct_batch_step(self._h, frame_dt, substeps), "oct_batch_step", self.ctx.handle)

    def status(self):
        """Per-scene failure state of the batch's frames (oct_batch_status), read and cleared."""
        out = np.zeros(len(self.scenes), np.int32)
        capi.check(capi.lib().oct_batch_status(self._h, capi.ptr(out, C.c_int32)), "oct_batch_status",
                   self.ctx.handle)
        return out

    def set_state(self, host):
        capi.check(capi.lib().oct_batch_set_state(self._h, capi.ptr(host, C.c_float)), "oct_batch_set_state")

    def get_state(self, host):
        capi.check(capi.lib().oct_batch_get_state(self._h, capi.ptr(host, C.c_float)), "oct_batch_get_state")

    def close(self):
        if self._h:
            capi.lib().oct_batch_destroy(self._h)
            self._h = C.c_void_p()


class Server:
    """Continuous-batching request loop (oct_server_*): submit (scene, steps) requests, tick
    frames, poll results."""

    def __init__(self, ctx, frame_dt=1 / 60, substeps=4, iterations=20, max_scenes=1024, hbm_budget=0,
                 precision=PREC_MIXED, setup_threads=0):
        self.ctx = ctx
        cfg = capi.ServerConfig(hbm_budget, max_scenes, frame_dt, substeps, iterations, precision, setup_threads)
        self._h = C.c_void_p()
        capi.check(capi.lib().oct_server_create(ctx.handle, C.byref(cfg), C.byref(self._h)), "oct_server_create")
        ctx._objs.append(self)
        self.n_nodes = {}

    def submit(self, element, positions, topology, steps, **kw):
        d, keep = make_desc(element, positions, topology, **kw)
        rid = C.c_int64()
        capi.check(capi.lib().oct_server_submit(self._h, C.byref(d), steps, C.byref(rid)), "oct_server_submit")
        self.n_nodes[rid.value] = d.n_nodes
        return rid.value

    def tick(self):
        n = C.c_int32()
        capi.check(capi.lib().oct_server_tick(self._h, C.byref(n)), "oct_server_tick", self.ctx.handle)
        return n.value

    def poll(self, rid, fetch=True):
        """None while the request runs; then its final positions (or True with fetch=False)."""
        done = C.c_int32()
        out = np.zeros((self.n_nodes[rid], 3), np.float32) if fetch else None
        st = capi.lib().oct_server_poll(self._h, rid, C.byref(done), capi.ptr(out, C.c_float) if fetch else None)
        if st != capi.OK:
            raise OctError(st, "oct_server_poll")
        if not done.value:
            return None
        return out if fetch else True

    def stats(self):
        s = capi.ServerStats()
        capi.check(capi.lib().oct_server_get_stats(self._h, C.byref(s)), "oct_server_get_stats")
        return {k: getattr(s, k) for k, _ in capi.ServerStats._fields_}

    def close(self):
        if self._h:
            capi.lib().oct_server_destroy(self._h)
            self._h = C.c_void_p()
