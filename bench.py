"""Benchmark of the batched VBD time step (one JSON line on rank 0).

Workload (default, "batched"): 256 seeded beam scenes, hex-grid dims nx in [4, 96],
ny, nz in [2, 24] (cell edge 1/16 m), element type uniform over {P1 tet (6-tet split),
P2 tet, Q1 hex}, E log-uniform in [1e4, 1e7] Pa, nu uniform in [0.30, 0.49], rho = 1000,
stable Neo-Hookean, x = 0 face fixed, gravity -z, each scene with its own DSAT colouring;
one step = one 1/60 s frame of 4 sub-steps x 20 VBD iterations over all scenes, batched
mixed precision (one launch per element type and colour, the sub-step as a CUDA graph).
Synthetic data; the state (~1 GB) is larger than L2, so no flush is needed between steps.

metric: vertex-iterations/s = sum over scenes of free nodes x iterations x sub-steps per
step, / time.  Also reported: the plain single-scene drop-in path (each scene stepped on
its own, FP32, one launch per colour, no graph) on the same scenes and GPU, p50/p99 step
latency, the end-to-end number through the C ABI with host buffers, the roofline of the
dominant kernel (algorithmic flops and bytes of the reference algorithm: Jx, F, dF/dx, PK1,
the six symmetric Hessian blocks and their assembly; the executed-flop rate beside them), the reference CPU VBD path timed on the host cores (one thread, as the reference runs;
all threads as an extension), the timed run's error against the FP64 oracle on a sample of
its scenes (`parity`), and, on the same GPU, config 2 as a single scene (`p2_single`), config
3's P3 and Q2 cubes at 32^3 cells (`cube`), the same 256 beams as XPBD scenes in one batch
(`xpbd_batched`, element-projections/s) and a
15 s Poisson request stream at 4 requests/s through the request loop (`served`, p50/p99
frame and request latency).  --no-extra skips the last four, --no-cpu the CPU legs.

Single-scene solver workloads of the P2 beam (64x16x16 hex grid x 6 tets = 98,304 P2 elements,
140,481 nodes, E=1e6, nu=0.49, rho=1100, x = 0 fixed, v0 ~ N(0, 0.05) from the seed):
  xpbd_p2      one step = one 1/60 s frame of 5 XPBD sub-steps (the GPU XPBD has no inner
               iterations), frame captured as a CUDA graph; metric element-projections/s
               (one projection = both constraints of one element)
  explicit_p2  one step = 100 symplectic-Euler sub-steps of dt = 1e-5 s, captured as a CUDA
               graph; metric vertex-steps/s

Served stream ("served"): Poisson arrivals at each rate of --rates (requests/s, wall clock);
each request is a seeded beam scene as in the batched workload with element count
log-uniform in [1e3, 5e5] and step count uniform in [10, 200], admitted by the request loop
(oct_server_*) under a 150 GB budget; one JSON line with, per rate, the aggregate
vertex-iterations/s, p50/p99 device frame time, p50/p99 wall time per tick and per request,
and the plain single-scene path on a sample of the same requests.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload batched|p2|cfg1|cube_p3|cube_q2|xpbd_p2|explicit_p2|served]
                    [--scenes N] [--no-plain] [--no-cpu] [--no-extra]
"""
import argparse
import concurrent.futures as cf
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FRAME_DT = 1.0 / 60.0


# ---- replicas over ranks: one process per GPU, no data-path collective; only the timing is
# combined (max over ranks) and the aggregate counts every rank's work
def init_ranks(world, local, timeout_s=600):
    """Process group for the replicas (NCCL on GPUs; gloo when no GPU is visible, for tests)."""
    if world <= 1:
        return None
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(x, world):
    """The largest of the ranks' values (each rank's device-timed milliseconds)."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(units_per_step, steps, world, max_ms):
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return units_per_step * steps * world / (max_ms * 1e-3)


def barrier_ranks(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def workload_specs(name, seed):
    """List of scene specs: (element, cells, size, young, poisson, density, gravity, iterations, substeps, dt)."""
    import octopusengine_b200 as ob
    rng = np.random.default_rng(seed)
    specs = []
    if name == "batched":
        for _ in range(256):
            nx, ny, nz = int(rng.integers(4, 97)), int(rng.integers(2, 25)), int(rng.integers(2, 25))
            e = [ob.TETRA, ob.TETRA10, ob.HEXA][int(rng.integers(0, 3))]
            young = float(np.exp(rng.uniform(np.log(1e4), np.log(1e7))))
            nu = float(rng.uniform(0.30, 0.49))
            specs.append(dict(element=e, cells=(nx, ny, nz), size=(nx / 16.0, ny / 16.0, nz / 16.0), young=young,
                              poisson=nu, density=1000.0))
        return specs, 20, 4, FRAME_DT
    if name == "p2":   # config 2: P2 beam 64x16x16 over 4x1x1 m, E=1e6, nu=0.49, rho=1100
        return [dict(element=ob.TETRA10, cells=(64, 16, 16), size=(4.0, 1.0, 1.0), young=1e6, poisson=0.49,
                     density=1100.0, v0_sigma=0.05)], 10, 5, FRAME_DT
    if name in ("cube_p3", "cube_q2"):   # config 3: 1 m cube 32^3, per-element E, top moved down 20 %
        e = ob.TETRA20 if name == "cube_p3" else ob.HEXA27
        E = np.exp(rng.uniform(np.log(1e4), np.log(1e6), 32 ** 3 * (6 if e == ob.TETRA20 else 1)))
        return [dict(element=e, cells=(32, 32, 32), size=(1.0, 1.0, 1.0), young=1e5, poisson=0.45, density=1000.0,
                     young_per_element=E.astype(np.float32), cube=True)], 10, 2, FRAME_DT
    if name in ("xpbd_p2", "explicit_p2"):
        return [dict(element=ob.TETRA10, cells=(64, 16, 16), size=(4.0, 1.0, 1.0), young=1e6, poisson=0.49,
                     density=1100.0, v0_sigma=0.05)], 1, (5 if name == "xpbd_p2" else 100), \
            (FRAME_DT if name == "xpbd_p2" else 100 * 1e-5)
    if name == "cfg1":  # config 1: 8x2x2 P1 beam, E=1e5, nu=0.45, dt=0.01, 1 x 20
        return [dict(element=ob.TETRA, cells=(8, 2, 2), size=(1.0, 0.25, 0.25), young=1e5, poisson=0.45,
                     density=1000.0)], 20, 1, 0.01
    raise SystemExit("unknown workload " + name)


def build_scene(ctx, spec, iterations, precision, seed, tpv=0, solver=None):
    import octopusengine_b200 as ob
    X, T = ob.beam_mesh(spec["element"], spec["cells"], spec["size"])
    group = None
    if spec.get("cube"):   # bottom face: rigid group 0 (static); top face: group 1 (moved)
        bottom = np.nonzero(X[:, 2] < 1e-6)[0]
        top = np.nonzero(X[:, 2] > spec["size"][2] - 1e-6)[0]
        fixed = np.concatenate([bottom, top]).astype(np.int32)
        group = np.concatenate([np.zeros(len(bottom)), np.ones(len(top))]).astype(np.int32)
        order = np.argsort(fixed, kind="stable")
        fixed, group = fixed[order], group[order]
    else:
        fixed = ob.fixed_by_plane(X, (0.01, 0.0, 0.0), (-1.0, 0.0, 0.0))
    kw = dict(density=spec["density"], mass_distribution=ob.MASS_FEMSHAPE, material=ob.STABLE_NEOHOOKE,
              young=spec["young"], poisson=spec["poisson"], fixed_ids=fixed, iterations=iterations,
              gravity=(0.0, 0.0, -9.81), precision=precision, threads_per_vertex=tpv)
    if solver is not None:
        kw["solver"] = solver
    if group is not None:
        kw["fixed_group"] = group
    if spec.get("young_per_element") is not None:
        kw["young_per_element"] = spec["young_per_element"]
    if spec.get("v0_sigma"):
        kw["initial_velocity"] = np.random.default_rng(seed).normal(0, spec["v0_sigma"], X.shape).astype(np.float32)
    return ob.Scene(ctx, spec["element"], X, T, **kw)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.device = device
        self.proc = None
        # raw samples (the JSON line carries their summary); OCTB_CLOCKS_DIR keeps them elsewhere
        self.path = os.path.join(os.environ.get("OCTB_CLOCKS_DIR", tempfile.gettempdir()),
                                 "clocks_bench_%d_%d.csv" % (device, os.getpid()))

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().split("\n") if r.strip()]
            if not rows:
                out["note"] = "timed region shorter than the 100 ms sampling period: no sample"
                return out
            sm = [float(r[1]) for r in rows]
            out["sm_mhz"] = float(np.median(sm))
            out["sm_max_mhz"] = float(rows[0][2])
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for k, n in enumerate(names):
                if any(r[5 + k].strip() == "Active" for r in rows):
                    out["reasons"].append(n)
            out["samples"] = len(rows)
            out["power_w_max"] = max(float(r[3]) for r in rows)
        except Exception:
            pass
        return out


def cpu_reference(specs, iterations, substeps, dt, threads, sample_every, sample_iters):
    """The reference CPU VBD (single-thread Gauss-Seidel per scene, as shipped, with its
    per-iteration force pass) over a sample of the workload's scenes, scenes spread over
    the host threads.  Returns vertex-iterations/s and the sample description."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    import octopusengine_b200 as ob
    sel = specs[::sample_every]
    keep, solvers, vit = [], [], 0
    for sp in sel:
        X, T = O.beam_mesh(sp["element"], sp["cells"], sp["size"])
        m = O.masses(sp["element"], X, T, sp["density"], 1)
        fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
        s = O.Scene(sp["element"], X, T, m, young=sp["young"], poisson=sp["poisson"], fixed=fixed,
                    iterations=sample_iters, gravity=(0, 0, -9.81))
        keep.append(s)
        solvers.append(O.CpuVBD(s))
        vit += (len(X) - len(fixed)) * sample_iters
    secs = O.run_cpu_many(solvers, dt / substeps, 1, True, threads)
    desc = ("%d of %d scenes (every %d-th), 1 sub-step x %d iterations of dt=%.5f s, %d host threads, "
            "reference CPU VBD restated in C++ (oracle/), per-iteration force pass included"
            % (len(sel), len(specs), sample_every, sample_iters, dt / substeps, threads))
    return vit / secs, secs, desc


SOLVER_WORKLOADS = {"xpbd_p2": "xpbd", "explicit_p2": "explicit"}


def solver_units(name, scene_or_spec, substeps):
    """Work units per step of a single-solver workload: element projections or vertex steps."""
    if SOLVER_WORKLOADS[name] == "xpbd":
        return scene_or_spec["n_elements"] * substeps
    return scene_or_spec["free_nodes"] * substeps


def cpu_solver_reference(name, spec, substeps, frame_dt, seed):
    """The workload's solver restated on the CPU (oracle/, GPU semantics, one thread), timed on a
    bounded sample: one XPBD sub-step or five explicit sub-steps of the full scene."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    X, T = O.beam_mesh(spec["element"], spec["cells"], spec["size"])
    m = O.masses(spec["element"], X, T, spec["density"], 1)
    fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
    v0 = np.random.default_rng(seed).normal(0, spec["v0_sigma"], X.shape).astype(np.float32)
    sc = O.Scene(spec["element"], X, T, m, young=spec["young"], poisson=spec["poisson"], fixed=fixed,
                 gravity=(0, 0, -9.81), v0=v0)
    kind = SOLVER_WORKLOADS[name]
    solver = O.Solver(kind, sc)
    n = 1 if kind == "xpbd" else 5
    sub = frame_dt / substeps
    t0 = time.perf_counter()
    solver.step(sub * n, n)
    secs = time.perf_counter() - t0
    units = (len(T) if kind == "xpbd" else len(X) - len(fixed)) * n
    desc = ("%d %s sub-step(s) of the full scene (%d elements, %d nodes), 1 host thread, the GPU %s path "
            "restated in C++ (oracle/)" % (n, kind, len(T), len(X), kind))
    return units / secs, secs, desc


def bench_solver(args, world, rank, local, threads):
    """xpbd_p2 / explicit_p2: one scene, frames replayed from a CUDA graph."""
    import ctypes as C

    import torch
    specs, iterations, substeps, frame_dt = workload_specs(args.workload, args.seed)
    spec = specs[0]
    kind = SOLVER_WORKLOADS[args.workload]
    unit = "element-projections/s" if kind == "xpbd" else "vertex-steps/s"
    metric = "element_projections_per_s" if kind == "xpbd" else "vertex_steps_per_s"
    if args.impl == "reference":
        if rank != 0:
            return
        vals = []
        for _ in range(args.warmup + args.steps):
            v, secs, desc = cpu_solver_reference(args.workload, spec, substeps, frame_dt, args.seed)
            vals.append(v)
        v = float(np.median(vals[args.warmup:]))
        print(json.dumps({"impl": "reference", "metric": metric, "value": v, "unit": unit, "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                          "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                          "config": {"workload": args.workload, "scenes": 1, "seed": args.seed},
                          "cpu_baseline": {"value": v, "unit": unit, "cores": 1, "kind": "port", "sample": desc},
                          "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    init_ranks(world, local)
    torch.cuda.set_device(local)
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    ctx = ob.Context(local, 0)
    solver = ob.SOLVER_XPBD if kind == "xpbd" else ob.SOLVER_EXPLICIT
    scene = build_scene(ctx, spec, iterations, ob.PREC_PLAIN, args.seed, solver=solver)
    scene.set_capture(True)
    info = dict(n_elements=scene.n_elements, free_nodes=scene.n_nodes - scene.n_fixed)
    units = solver_units(args.workload, info, substeps)
    stream_ptr = C.c_void_p()
    capi.lib().oct_ctx_stream(ctx.handle, C.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value, device=local)
    for _ in range(args.warmup):
        scene.step(frame_dt, substeps, sync=False)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    l0 = ctx.launch_count()
    barrier_ranks(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        ev[0].record(stream)
        for k in range(args.steps):
            scene.step(frame_dt, substeps, sync=False)
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
    barrier_ranks(world)
    launches = ctx.launch_count() - l0
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = max_over_ranks(ev[0].elapsed_time(ev[-1]), world)
    value = aggregate_rate(units, args.steps, world, total_ms)
    # end to end: positions and velocities in from pinned host memory, positions out, each step
    n = scene.n_nodes
    host_p = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    host_v = torch.empty((n, 3), dtype=torch.float32, pin_memory=True).numpy()
    host_p[:] = scene.get_position()
    host_v[:] = scene.get_velocity()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        scene.set_position(host_p)
        scene.set_velocity(host_v)
        scene.step(frame_dt, substeps, sync=False)
        host_p[:] = scene.get_position()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    e2e_value = units * args.steps * world / (e2e_ms * 1e-3)
    # roofline of the frame: algorithmic flops and bytes per unit.  Element projection:
    # 2 Q (36 n_e + 160) + 24 n_e flops.  Explicit vertex step (vertex-centric force): for each
    # of the vertex's (owner, quadrature point) pairs Jx 18 n_e, F 48, dF/dx 15, P ~45, f 21.
    ne, nq = 10, 4
    fp32_peak = C.c_double()
    capi.lib().oct_fp32_peak(ctx.handle, C.byref(fp32_peak))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    if kind == "xpbd":
        flops_unit = 2 * nq * (36 * ne + 160) + 24 * ne
        bytes_unit = 4 * ne + 48 + 2 * 16 * ne   # topology, one affine record, node gather + write-back
    else:
        flops_unit = (info["n_elements"] * ne / n) * nq * (18 * ne + 129)
        bytes_unit = 16 * 4 + 4 * 2   # u, v, y, u_new per node + owner entry stream (amortised)
    sec = total_ms * 1e-3 / (args.steps * world)
    ach_tf = flops_unit * units / sec / 1e12
    ach_gb = bytes_unit * units / sec / 1e9
    roofline = {"bound": "hbm", "achieved": ach_gb, "peak": hbm_peak, "unit": "GB/s", "frac": ach_gb / hbm_peak,
                "traffic": None, "kernel": "whole frame graph (%s)" % ("k_xpbd colour launches" if kind == "xpbd"
                                                                      else "k_vertex force + integrate"),
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s",
                "binding_roof": "fp32",
                "fp32": {"achieved_tflops": ach_tf, "peak_tflops": fp32_peak.value, "frac": ach_tf / fp32_peak.value,
                         "flops_per_unit": flops_unit}}
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        v, secs, desc = cpu_solver_reference(args.workload, spec, substeps, frame_dt, args.seed)
        cpu = {"value": v, "unit": unit, "cores": 1, "kind": "port", "sample": desc}
    if rank == 0:
        print(json.dumps({
            "metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "scenes": 1, "elements": info["n_elements"],
                       "free_nodes": info["free_nodes"], "substeps": substeps, "frame_dt": frame_dt,
                       "seed": args.seed, "l2": "scene state below L2 size; no flush (single-scene workload)",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "p50_step_ms": float(np.percentile(step_ms, 50)), "p99_step_ms": float(np.percentile(step_ms, 99)),
            "e2e": {"value": e2e_value, "unit": unit, "h2d_bytes_per_step": 2 * n * 12, "d2h_bytes_per_step": n * 12},
            "gpu_launches": int(launches), "roofline": roofline, "clocks": clocks.summary(), "cpu_baseline": cpu}))
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def served_request(rng):
    """One request of the served stream: (element, cells, size, young, poisson, steps)."""
    import octopusengine_b200 as ob
    e = [ob.TETRA, ob.TETRA10, ob.HEXA][int(rng.integers(0, 3))]
    target = float(np.exp(rng.uniform(np.log(1e3), np.log(5e5))))
    cells = target / (1.0 if e == ob.HEXA else 6.0)
    ny = max(2, int(round((cells / 4.0) ** (1.0 / 3.0))))
    nx = max(4, int(round(cells / (ny * ny))))
    young = float(np.exp(rng.uniform(np.log(1e4), np.log(1e7))))
    nu = float(rng.uniform(0.30, 0.49))
    return dict(element=e, cells=(nx, ny, ny), size=(nx / 16.0, ny / 16.0, ny / 16.0), young=young, poisson=nu,
                density=1000.0, steps=int(rng.integers(10, 201)))


def served_stream(ctx, rate, seconds, seed, threads, iterations=20, substeps=4, frame_dt=FRAME_DT):
    """One Poisson request stream at `rate` requests/s for `seconds` of arrivals through the
    request loop (oct_server_*), drained afterwards; returns its throughput and latencies."""
    import octopusengine_b200 as ob
    rng = np.random.default_rng(seed)
    srv = ob.Server(ctx, frame_dt=frame_dt, substeps=substeps, iterations=iterations, max_scenes=1024,
                    hbm_budget=150 * 10 ** 9, precision=ob.PREC_MIXED, setup_threads=max(1, threads - 2))
    # the request stream is generated before the clock starts (arrival times and meshes), so
    # the loop below only submits, ticks and polls
    arrivals_at, reqs, t = [], [], rng.exponential(1.0 / rate)
    while t < seconds:
        r = served_request(rng)
        X, T = ob.beam_mesh(r["element"], r["cells"], r["size"])
        fixed = ob.fixed_by_plane(X, (0.01, 0.0, 0.0), (-1.0, 0.0, 0.0))
        reqs.append((r, X, T, fixed))
        arrivals_at.append(t)
        t += rng.exponential(1.0 / rate)
    outstanding, latencies, tick_ms, nxt = {}, [], [], 0
    finished_seen = 0
    t_start = time.perf_counter()
    with ClockSampler(0) as clocks:
        while True:
            now = time.perf_counter() - t_start
            while nxt < len(reqs) and arrivals_at[nxt] <= now:
                r, X, T, fixed = reqs[nxt]
                rid = srv.submit(r["element"], X, T, r["steps"], density=1000.0, mass_distribution=ob.MASS_FEMSHAPE,
                                 material=ob.STABLE_NEOHOOKE, young=r["young"], poisson=r["poisson"],
                                 fixed_ids=fixed, gravity=(0.0, 0.0, -9.81))
                outstanding[rid] = t_start + arrivals_at[nxt]
                nxt += 1
            if nxt >= len(reqs) and not outstanding:
                break
            if now > seconds * 4:   # drain limit
                break
            t0 = time.perf_counter()
            st0 = srv.stats()
            srv.tick()
            st1 = srv.stats()
            if st1["frames"] > st0["frames"]:   # ticks that ran a frame
                tick_ms.append((time.perf_counter() - t0) * 1e3)
            if st1["finished"] + st1["rejected"] + st1["failed"] > finished_seen:
                finished_seen = st1["finished"] + st1["rejected"] + st1["failed"]
                for rid in list(outstanding):
                    if srv.poll(rid, fetch=False) is not None:
                        latencies.append(time.perf_counter() - outstanding.pop(rid))
            if not st1["active"]:
                time.sleep(0.001)   # idle: waiting for arrivals or set-up
    wall = time.perf_counter() - t_start
    st = srv.stats()
    out = {
        "rate_per_s": rate, "arrival_window_s": seconds, "arrived": nxt, "finished": int(st["finished"]),
        "rejected": int(st["rejected"]), "failed": int(st["failed"]),
        "frames": int(st["frames"]), "wall_s": wall,
        "vertex_iter_per_s": st["vertex_iterations"] / wall,
        "vertex_iter_per_busy_s": st["vertex_iterations"] / max(st["busy_ms"] * 1e-3, 1e-9),
        "gpu_busy_frac": st["busy_ms"] * 1e-3 / wall,
        "gap_ms_per_frame": st["gap_ms"] / max(st["frames"], 1),
        "p50_step_ms": st["p50_step_ms"], "p99_step_ms": st["p99_step_ms"], "mean_step_ms": st["mean_step_ms"],
        "p50_tick_wall_ms": float(np.percentile(tick_ms, 50)) if tick_ms else None,
        "p99_tick_wall_ms": float(np.percentile(tick_ms, 99)) if tick_ms else None,
        "p50_request_s": float(np.percentile(latencies, 50)) if latencies else None,
        "p99_request_s": float(np.percentile(latencies, 99)) if latencies else None,
        "clocks": clocks.summary()}
    srv.close()
    return out


def single_scene_p2(ctx, seed, stream, warmup=3, steps=5):
    """Config 2 alone: the P2 beam (140,481 nodes), 5 sub-steps x 10 iterations per 1/60 s frame,
    mixed precision with the autotuned mapping (a batch of one scene, sub-steps from a CUDA
    graph), and the plain drop-in path (FP32, per-colour launches) on the same scene."""
    import torch
    import octopusengine_b200 as ob
    specs, iterations, substeps, frame_dt = workload_specs("p2", seed)
    sc = build_scene(ctx, specs[0], iterations, ob.PREC_MIXED, seed)
    mapping = ob.autotune_mapping(ctx, [sc], frame_dt / substeps, sweeps=3)
    b = ob.Batch(ctx, [sc])
    vit = (sc.n_nodes - sc.n_fixed) * iterations * substeps

    def timed(step, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(n):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    for _ in range(warmup):
        b.step(frame_dt, substeps)
    ms = timed(lambda: b.step(frame_dt, substeps), steps)
    b.close()
    sc.set_precision(ob.PREC_PLAIN)
    sc.step(frame_dt, substeps, sync=False)
    plain_ms = timed(lambda: sc.step(frame_dt, substeps, sync=False), 3)
    out = {"value": vit / (ms * 1e-3), "unit": "vertex-iter/s", "ms_per_frame": ms, "frames": steps,
           "nodes": sc.n_nodes, "mapping": mapping.get(ob.TETRA10),
           "plain_dropin": {"value": vit / (plain_ms * 1e-3), "ms_per_frame": plain_ms}}
    sc.close()
    return out


def single_cube(ctx, name, seed, stream, warmup=3, steps=3):
    """Config 3 at full size: the 1 m cube of 32^3 cells as P3 (912,673 nodes) or Q2 (274,625
    nodes), per-element Young modulus, bottom fixed and top moved down 20 % over 50 frames;
    2 sub-steps x 10 iterations per 1/60 s frame, mixed precision, autotuned mapping."""
    import torch
    import octopusengine_b200 as ob
    specs, iterations, substeps, frame_dt = workload_specs(name, seed)
    t0 = time.time()
    sc = build_scene(ctx, specs[0], iterations, ob.PREC_MIXED, seed)
    setup_s = time.time() - t0
    mapping = ob.autotune_mapping(ctx, [sc], frame_dt / substeps, sweeps=2)
    b = ob.Batch(ctx, [sc])
    frame = [0]

    def step():
        frame[0] += 1
        sc.set_fixation((0.0, 0.0, -0.2 * min(frame[0], 50) / 50.0), group=1)
        b.step(frame_dt, substeps)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    vit = (sc.n_nodes - sc.n_fixed) * iterations * substeps
    out = {"value": vit / (ms * 1e-3), "unit": "vertex-iter/s", "ms_per_frame": ms, "frames": steps,
           "nodes": sc.n_nodes, "elements": sc.n_elements, "mapping": mapping.get(specs[0]["element"]),
           "setup_s": setup_s, "status": int(b.status()[0])}
    b.close()
    sc.close()
    return out


def batched_xpbd(ctx, specs, seed, stream, threads, warmup=3, steps=5, substeps=5, frame_dt=FRAME_DT):
    """The batched workload's scenes as XPBD scenes (reference default OptiShared: V0 for P1, the
    raw V2 update for P2/Q1) in one batch: per 1/60 s frame 5 sub-steps of GPU_PBD::step over
    all scenes, one launch per (element type, material, update form, colour) across the scenes,
    the sub-step a CUDA graph.  Metric: element projections/s (both constraints of one
    element, every element once per sub-step)."""
    import torch
    import octopusengine_b200 as ob
    t0 = time.time()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        scenes = list(ex.map(lambda a: build_scene(ctx, a[1], 1, ob.PREC_PLAIN, seed + a[0], solver=ob.SOLVER_XPBD),
                             enumerate(specs)))
    setup_s = time.time() - t0
    b = ob.Batch(ctx, scenes)
    units = sum(s.n_elements for s in scenes) * substeps
    for _ in range(warmup):
        b.step(frame_dt, substeps)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(steps + 1)]
    l0 = ctx.launch_count()
    ev[0].record(stream)
    for k in range(steps):
        b.step(frame_dt, substeps)
        ev[k + 1].record(stream)
    torch.cuda.synchronize()
    launches = ctx.launch_count() - l0
    ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(steps)]
    total = ev[0].elapsed_time(ev[-1])
    status = b.status()
    b.close()
    for s in scenes:
        s.close()
    return {"value": units * steps / (total * 1e-3), "unit": "element-projections/s", "scenes": len(specs),
            "elements": units // substeps, "substeps": substeps, "frame_dt": frame_dt, "ms_per_frame": total / steps,
            "p50_frame_ms": float(np.percentile(ms, 50)), "p99_frame_ms": float(np.percentile(ms, 99)),
            "gpu_launches": int(launches), "failed_scenes": int((status != 0).sum()), "setup_s": setup_s}


def bench_served(args, threads):
    """Continuous batching of a Poisson request stream through oct_server_* (one GPU)."""
    import ctypes as C

    import torch
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    torch.cuda.set_device(0)
    iterations, substeps, frame_dt = 20, 4, FRAME_DT
    rates = [float(x) for x in args.rates.split(",") if x]
    ctx = ob.Context(0, 0)
    results = [served_stream(ctx, rate, args.serve_seconds, args.seed + ri, threads, iterations, substeps, frame_dt)
               for ri, rate in enumerate(rates)]
    # plain single-scene path on a sample of the same request stream: each scene stepped alone
    rng = np.random.default_rng(args.seed)
    sample = [served_request(rng) for _ in range(12)]
    scenes = []
    for r in sample:
        X, T = ob.beam_mesh(r["element"], r["cells"], r["size"])
        fixed = ob.fixed_by_plane(X, (0.01, 0.0, 0.0), (-1.0, 0.0, 0.0))
        scenes.append(ob.Scene(ctx, r["element"], X, T, density=1000.0, mass_distribution=ob.MASS_FEMSHAPE,
                               material=ob.STABLE_NEOHOOKE, young=r["young"], poisson=r["poisson"], fixed_ids=fixed,
                               gravity=(0.0, 0.0, -9.81), iterations=iterations, precision=ob.PREC_PLAIN))
    stream_ptr = C.c_void_p()
    capi.lib().oct_ctx_stream(ctx.handle, C.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value, device=0)
    for sc in scenes:
        sc.step(frame_dt, substeps, sync=False)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(2):
        for sc in scenes:
            sc.step(frame_dt, substeps, sync=False)
    p1.record(stream)
    torch.cuda.synchronize()
    vit = 2 * sum(sc.n_nodes - sc.n_fixed for sc in scenes) * iterations * substeps
    plain = vit / (p0.elapsed_time(p1) * 1e-3)
    for sc in scenes:
        sc.close()
    top = max(results, key=lambda x: x["vertex_iter_per_s"])
    print(json.dumps({
        "metric": "vertex_iterations_per_s", "value": top["vertex_iter_per_s"], "unit": "vertex-iter/s", "n_gpus": 1,
        "steps": int(top["frames"]), "warmup": 0, "ms_per_step": top["mean_step_ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "served", "rates_per_s": rates, "serve_seconds": args.serve_seconds,
                   "iterations": iterations, "substeps": substeps, "frame_dt": frame_dt, "budget_bytes": 150 * 10 ** 9,
                   "seed": args.seed, "precision": "mixed"},
        "p50_step_ms": top["p50_step_ms"], "p99_step_ms": top["p99_step_ms"],
        "served": results,
        "plain_dropin": {"value": plain, "unit": "vertex-iter/s",
                         "path": "12 requests of the stream, each scene stepped alone (FP32, per-colour launches)"},
        "batched_over_plain": top["vertex_iter_per_busy_s"] / plain,
        "gpu_launches": None}))
    ctx.close()


def vertex_kernel_label(group, scenes):
    """Name of the colour kernel a batch group launches (its element's lane mapping in effect)."""
    tpv = next((s.mapping() for s in scenes if s.element == group["element"]), 0)
    if tpv == -1:
        return "k_vertex_packed<%d,%d> (VBD colour sweep, element %d, one lane per (vertex, owner) pair)" % (
            group["element"], group["material"], group["element"])
    return "k_vertex<%d,%d> (VBD colour sweep, element %d, %d lanes per vertex, wider on colours of more than %d owners per lane)" % (
        group["element"], group["material"], group["element"], tpv, 8)


def parity_sample(scenes, specs, positions, frames, iterations, substeps, frame_dt, threads):
    """Error of the timed run against the FP64 oracle (the checker, on the host): the sampled
    scenes' positions after the run's frames, against the FP64 restatement of the same scenes
    stepped through the same frames from rest.  The sample is the two smallest scenes of at
    least 500 nodes of each element type; the scenes run on parallel host threads."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as O
    sel = sorted(positions)
    jobs = []
    for i in sel:
        sp, sc = specs[i], scenes[i]
        X, T = O.beam_mesh(sp["element"], sp["cells"], sp["size"])
        m = O.masses(sp["element"], X, T, sp["density"], 1)
        fixed = O.fixed_by_plane(X, (0.01, 0, 0), (-1, 0, 0))
        colors = sc.coloring()[0]
        o = O.Scene(sp["element"], X, T, m, young=sp["young"], poisson=sp["poisson"], fixed=fixed, gravity=(0, 0, -9.81),
                    iterations=iterations, colors=colors, n_colors=int(colors.max()) + 1, in_place=True)
        jobs.append((i, X, o, O.Solver("vbd", o, fp64=True)))

    def run(job):
        for _ in range(frames):
            job[3].step(frame_dt, substeps)
        return job[3].get(0)

    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=max(1, min(threads, len(jobs)))) as ex:
        refs = list(ex.map(run, jobs))
    rows = []
    for (i, X, o, solver), ref in zip(jobs, refs):
        p = positions[i].astype(np.float64)
        err = np.abs(p - ref).max()
        rows.append({"scene": i, "element": specs[i]["element"], "nodes": len(X),
                     "pos_rel_err": float(err / np.abs(ref).max()),
                     "disp_rel_err": float(err / max(np.abs(ref - X).max(), 1e-30))})
    return {"against": "FP64 oracle (GPU semantics restated in C++), same scenes, colourings and frames from rest",
            "frames": frames, "scenes": rows,
            "max_pos_rel_err": max(r["pos_rel_err"] for r in rows),
            "max_disp_rel_err": max(r["disp_rel_err"] for r in rows),
            "oracle_s": time.perf_counter() - t0}


def parity_indices(scenes):
    """Two smallest scenes of at least 500 nodes per element type."""
    out = []
    for e in sorted({s.element for s in scenes}):
        cand = sorted((s.n_nodes, i) for i, s in enumerate(scenes) if s.element == e and s.n_nodes >= 500)
        out += [i for _, i in cand[:2]]
    return out


def survey_counts(scenes, element):
    """Algorithmic work of one colour sweep over the scenes of one element type, by the
    reference algorithm's per-unit figures: per (vertex, owner element, quadrature point)
    triple 18 n_e + 480 FP32 flops (Jx, F, dF/dx, PK1, symmetric Hessian blocks and their
    assembly, accumulation: compute_f_H_sym with eval_pk1_stress / eval_hessian_sym /
    assemble_sub_hessian_sym), and per sweep 40 B per node (p, y, mass read, p written) plus per
    element 4 n_e B of topology and 40 B per quadrature point (JX_inv and V) as minimal DRAM
    bytes.  Free vertices only: fixed ones are skipped by the sweep."""
    from octopusengine_b200 import capi
    ne, nq = capi.ELEMENT_NODES[element], capi.ELEMENT_QUADRATURE[element]
    fl = by = 0.0
    for s in scenes:
        if s.element != element:
            continue
        free = s.n_nodes - s.n_fixed
        fl += s.n_elements * ne * nq * free / s.n_nodes * (18.0 * ne + 480.0)
        by += 40.0 * s.n_nodes + s.n_elements * (4.0 * ne + 40.0 * nq)
    return fl, by


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "p2", "cfg1", "cube_p3", "cube_q2", "xpbd_p2", "explicit_p2", "served",
                             "xpbd_batched"])
    ap.add_argument("--rates", default="4,8,16", help="served: Poisson arrival rates (requests/s)")
    ap.add_argument("--serve-seconds", type=float, default=20.0, help="served: arrival window per rate")
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--tpv", type=int, default=0, help="lanes per vertex (0 = measured default, -1 = packed pair-per-lane mapping)")
    ap.add_argument("--tpv-elem", default="", help="per-element lanes per vertex, e.g. 3:4,7:-1")
    ap.add_argument("--no-autotune", action="store_true", help="keep the measured default mapping")
    ap.add_argument("--scenes", type=int, default=0,
                    help="batched: only the first N scenes of the draw (a smaller case for profiling)")
    ap.add_argument("--no-extra", action="store_true",
                    help="batched: skip the single-scene config-2 figure and the short served stream")
    ap.add_argument("--serve-rate", type=float, default=4.0, help="batched: rate of the short served stream")
    ap.add_argument("--serve-window", type=float, default=15.0, help="batched: arrival window of the served stream")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    threads = os.cpu_count() or 1
    if args.workload in SOLVER_WORKLOADS:
        bench_solver(args, world, rank, local, threads)
        return
    if args.workload == "xpbd_batched":   # the batched workload's scenes as XPBD scenes, alone
        if args.impl == "reference" or rank != 0:
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference's XPBD path is GPU-only; "
                                  "its CPU VBD path is timed by the batched workload"}))
            return
        import torch
        torch.cuda.set_device(local)
        import octopusengine_b200 as ob
        specs, _, _, _ = workload_specs("batched", args.seed)
        if args.scenes > 0:
            specs = specs[:args.scenes]
        from octopusengine_b200 import capi
        import ctypes as C
        ctx = ob.Context(local, 0)
        stream_ptr = C.c_void_p()
        capi.lib().oct_ctx_stream(ctx.handle, C.byref(stream_ptr))
        stream = torch.cuda.ExternalStream(stream_ptr.value, device=local)
        line = batched_xpbd(ctx, specs, args.seed, stream, threads, warmup=args.warmup, steps=args.steps)
        ctx.close()
        print(json.dumps({"metric": "element_projections_per_s", "value": line["value"], "unit": line["unit"],
                          "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                          "ms_per_step": line["ms_per_frame"], "config": {"workload": "xpbd_batched",
                          "scenes": len(specs)}, "xpbd_batched": line}))
        return
    if args.workload == "served":
        if args.impl == "reference" or rank != 0:
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "the reference has no request loop; "
                                  "its CPU VBD path is timed by the batched workload"}))
            return
        bench_served(args, threads)
        return
    specs, iterations, substeps, frame_dt = workload_specs(args.workload, args.seed)
    if args.scenes > 0:
        specs = specs[:args.scenes]

    if args.impl == "reference":
        if rank != 0:
            return
        every = 4 if args.workload == "batched" else 1
        its = 4 if args.workload == "batched" else (2 if args.workload == "p2" else iterations)
        vals = []
        for _ in range(args.warmup + args.steps):
            v, secs, desc = cpu_reference(specs, iterations, substeps, frame_dt, threads, every, its)
            vals.append(v)
        v = float(np.median(vals[args.warmup:]))
        line = {"impl": "reference", "metric": "vertex_iterations_per_s", "value": v, "unit": "vertex-iter/s",
                "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": {"workload": args.workload, "scenes": len(specs), "seed": args.seed},
                "cpu_baseline": {"value": v, "unit": "vertex-iter/s", "cores": threads, "kind": "port",
                                 "sample": desc},
                "e2e": {"value": v, "unit": "vertex-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    init_ranks(world, local)
    device = local
    torch.cuda.set_device(device)
    import octopusengine_b200 as ob
    from octopusengine_b200 import capi
    import ctypes as C

    ctx = ob.Context(device, 0)
    # scene set-up (host colouring etc.) in parallel host threads
    t0 = time.time()
    with cf.ThreadPoolExecutor(max_workers=threads) as ex:
        per_elem = {int(k): int(v) for k, v in (x.split(":") for x in args.tpv_elem.split(",") if x)}
        scenes = list(ex.map(lambda a: build_scene(ctx, a[1], iterations, ob.PREC_MIXED, args.seed + a[0],
                                                   per_elem.get(a[1]["element"], args.tpv)), enumerate(specs)))
    setup_s = time.time() - t0
    # lane mapping per element type: the autotuner times every candidate on these scenes
    # (state untouched) unless a mapping was forced on the command line
    mapping, tune_s = None, None
    if not args.no_autotune and args.tpv == 0 and not args.tpv_elem:
        t0 = time.time()
        mapping = ob.autotune_mapping(ctx, scenes, frame_dt / substeps, sweeps=3)
        tune_s = time.time() - t0
    batch = ob.Batch(ctx, scenes)
    free_nodes = sum(s.n_nodes - s.n_fixed for s in scenes)
    vit_per_step = free_nodes * iterations * substeps

    stream_ptr = C.c_void_p()
    capi.lib().oct_ctx_stream(ctx.handle, C.byref(stream_ptr))
    stream = torch.cuda.ExternalStream(stream_ptr.value, device=device)

    def barrier():
        barrier_ranks(world)

    cube = bool(specs[0].get("cube"))
    frame = [0]

    def step_all():
        if cube:   # top face moved down 20 % of the height over 50 frames, then held
            frame[0] += 1
            for s in scenes:
                s.set_fixation((0.0, 0.0, -0.2 * min(frame[0], 50) / 50.0), group=1)
        batch.step(frame_dt, substeps)

    for _ in range(args.warmup):
        step_all()
    torch.cuda.synchronize()

    # ---- timed region: K batched steps, per-step events on the library's stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    launches0 = ctx.launch_count()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(device) as clocks:
        ev[0].record(stream)
        for k in range(args.steps):
            step_all()
            ev[k + 1].record(stream)
        torch.cuda.synchronize()
    barrier()
    launches = ctx.launch_count() - launches0
    sample_pos = {}
    if rank == 0 and world == 1 and not args.no_cpu and args.workload == "batched":
        sample_pos = {i: scenes[i].get_position() for i in parity_indices(scenes)}
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps)]
    total_ms = max_over_ranks(ev[0].elapsed_time(ev[-1]), world)
    value = aggregate_rate(vit_per_step, args.steps, world, total_ms)

    # ---- end to end through the C ABI with pinned host buffers
    n_state = batch.state_size
    host = torch.empty(n_state, dtype=torch.float32, pin_memory=True)
    host_np = host.numpy()
    batch.get_state(host_np)
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    e_start.record(stream)
    for _ in range(args.steps):
        batch.set_state(host_np)
        step_all()
        batch.get_state(host_np)
    e_end.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e_start.elapsed_time(e_end), world)
    e2e_value = aggregate_rate(vit_per_step, args.steps, world, e2e_ms)
    bytes_state = n_state * 4

    # ---- roofline of the dominant kernel (the VBD colour kernel of the heaviest group)
    groups = []
    g = 0
    while True:
        el, mat, nl = C.c_int32(), C.c_int32(), C.c_int32()
        fl, by = C.c_double(), C.c_double()
        nv = C.c_int64()
        if capi.lib().oct_batch_group_info(batch._h, g, C.byref(el), C.byref(mat), C.byref(fl), C.byref(by),
                                           C.byref(nl), C.byref(nv)) != 0:
            break
        groups.append(dict(g=g, element=el.value, material=mat.value, flops=fl.value, bytes=by.value,
                           launches=nl.value, vertices=nv.value))
        g += 1
    dom = max(groups, key=lambda x: x["flops"])
    sweeps = 10
    ms = C.c_float()
    for gi in groups:   # every group alone: per-sweep time and algorithmic rates
        capi.check(capi.lib().oct_batch_time_group(batch._h, gi["g"], 2, frame_dt / substeps, C.byref(ms)), "warm")
        capi.check(capi.lib().oct_batch_time_group(batch._h, gi["g"], 5, frame_dt / substeps, C.byref(ms)), "time")
        gi["ms_per_sweep"] = ms.value / 5
        gi["tflops"] = gi["flops"] / (gi["ms_per_sweep"] * 1e-3) / 1e12
        gi["gvit_per_s"] = gi["vertices"] / (gi["ms_per_sweep"] * 1e-3) / 1e9
    capi.check(capi.lib().oct_batch_time_group(batch._h, dom["g"], 2, frame_dt / substeps, C.byref(ms)), "warm")
    capi.check(capi.lib().oct_batch_time_group(batch._h, dom["g"], sweeps, frame_dt / substeps, C.byref(ms)),
               "oct_batch_time_group")
    per_launch_s = ms.value * 1e-3 / (sweeps * dom["launches"])
    survey_fl, survey_by = survey_counts(scenes, dom["element"])
    flops_per_launch = survey_fl / dom["launches"]
    bytes_per_launch = survey_by / dom["launches"]
    executed_flops_per_launch = dom["flops"] / dom["launches"]
    fp32_peak = C.c_double()
    capi.lib().oct_fp32_peak(ctx.handle, C.byref(fp32_peak))
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    achieved_gbs = bytes_per_launch / per_launch_s / 1e9
    achieved_tflops = flops_per_launch / per_launch_s / 1e12
    executed_tflops = executed_flops_per_launch / per_launch_s / 1e12
    traffic = None
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "vbd_dram_traffic.json")))
        traffic = prof.get("bytes_per_launch_scaled", {}).get(args.workload)
    except Exception:
        pass
    roofline = {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                "frac": achieved_gbs / hbm_peak, "traffic": traffic,
                "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured)" if peaks else "fallback 6650 GB/s",
                "kernel": vertex_kernel_label(dom, scenes),
                "launch_ms": per_launch_s * 1e3,
                "algorithmic": {"bytes_per_launch": bytes_per_launch, "flops_per_launch": flops_per_launch,
                                "per_unit": "reference algorithm: 18 n_e + 480 flops per (vertex, owner, quadrature point); "
                                            "40 B per node + (4 n_e + 40 Q) B per element per sweep"},
                "binding_roof": "fp32",
                "fp32": {"achieved_tflops": achieved_tflops, "peak_tflops": fp32_peak.value,
                         "frac": achieved_tflops / fp32_peak.value,
                         "peak_source": "oct_fp32_peak FMA loop, measured in this run",
                         "executed": {"tflops": executed_tflops, "frac": executed_tflops / fp32_peak.value,
                                      "note": "flops the kernel executes: the closed-form Hessian contraction "
                                              "needs about half the reference algorithm's count"}}}

    # ---- plain single-scene drop-in path on the same scenes (FP32, per-colour launches)
    plain = None
    if not args.no_plain:
        for s in scenes:
            s.set_precision(ob.PREC_PLAIN)
        for s in scenes:
            s.step(frame_dt, substeps, sync=False)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for s in scenes:
            s.step(frame_dt, substeps, sync=False)
        p1.record(stream)
        torch.cuda.synchronize()
        plain_ms = p0.elapsed_time(p1)
        plain = {"value": vit_per_step / (plain_ms * 1e-3), "unit": "vertex-iter/s", "ms_per_step": plain_ms,
                 "path": "each scene stepped alone through oct_scene_step: FP32, one launch per colour, no graph"}

    # ---- the rest of the metric on the same GPU: config 2 alone, and a short served stream
    p2_line, served_line, xpbd_line, cube_lines = None, None, None, None
    if rank == 0 and world == 1 and args.workload == "batched" and not args.no_extra:
        p2_line = single_scene_p2(ctx, args.seed, stream)
        cube_lines = {w: single_cube(ctx, w, args.seed, stream) for w in ("cube_p3", "cube_q2")}
        xpbd_line = batched_xpbd(ctx, specs, args.seed, stream, threads)
        served_line = served_stream(ctx, args.serve_rate, args.serve_window, args.seed, threads)

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        every = 4 if args.workload == "batched" else 1
        its = 4 if args.workload == "batched" else (2 if args.workload == "p2" else iterations)
        # the reference's CPU VBD is single-threaded, as shipped: timed on one thread (every
        # 16th scene of the batched workload); the same code over all host threads, one scene
        # per thread, is a labelled extension
        v1, secs1, desc1 = cpu_reference(specs, iterations, substeps, frame_dt, 1, 4 * every, its)
        cpu = {"value": v1, "unit": "vertex-iter/s", "cores": 1, "kind": "port", "sample": desc1}
        v, secs, desc = cpu_reference(specs, iterations, substeps, frame_dt, threads, every, its)
        cpu["all_threads"] = {"value": v, "cores": threads, "sample": desc,
                              "note": "extension: independent scenes on parallel host threads"}
        if sample_pos:
            parity = parity_sample(scenes, specs, sample_pos, args.warmup + args.steps, iterations, substeps,
                                   frame_dt, threads)

    if rank == 0:
        line = {
            "metric": "vertex_iterations_per_s", "value": value, "unit": "vertex-iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "scenes": len(scenes), "free_nodes": free_nodes,
                       "iterations": iterations, "substeps": substeps, "frame_dt": frame_dt,
                       "precision": "mixed (FP32 bulk, compensated sums, FP64 ill-conditioned solves)",
                       "seed": args.seed, "l2": "state larger than L2 (126 MB); no flush",
                       "mapping": ({str(k): v for k, v in mapping.items()} if mapping is not None else
                                   "fixed (--tpv / --tpv-elem / --no-autotune)"),
                       "autotune_s": tune_s,
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "p50_step_ms": float(np.percentile(step_ms, 50)), "p99_step_ms": float(np.percentile(step_ms, 99)),
            "plain_dropin": plain,
            "batched_over_plain": (value / world) / plain["value"] if plain else None,
            "e2e": {"value": e2e_value, "unit": "vertex-iter/s", "h2d_bytes_per_step": bytes_state,
                    "d2h_bytes_per_step": bytes_state},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "groups": [{k: g[k] for k in ("element", "vertices", "launches", "ms_per_sweep", "tflops", "gvit_per_s")}
                       for g in groups],
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "parity": parity,
            "p2_single": p2_line,
            "cube": cube_lines,
            "xpbd_batched": xpbd_line,
            "served": served_line,
            "setup_s": setup_s,
        }
        print(json.dumps(line))
    batch.close()
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
