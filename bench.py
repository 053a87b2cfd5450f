"""Throughput of the boundary-integral hot path on the large 2-D scene.

    python bench.py [--gpus N --steps K --warmup W] [--impl ours|reference] [--precision mixed|fp64] [--route fused|plain]

Workload (one step): lambda + the twelve moments of every particle of the large 2-D scene (2^20 particles uniform in
[0, 4]^2, h = 0.02, 64 seeded star polygons in one multi-loop surface, near-tangent particles) for each of the kernels
cubic, w2, w4, w6.  Metric: particle-edge neighbour pairs per second (pairs = pairs passing the float64 neighbour
predicate, counted once, times the number of kernels).  `value` is measured with inputs resident on the device;
`e2e` through the public provider API with host buffers (pinned host -> device copy of positions and supports, device
-> host copy of lam, G, Cov, m1, m2 of every kernel) inside the timed region.  Between timed steps L2 is flushed by
writing a 256 MiB buffer (outside the events).  `routes` compares the plain float64 route, the fused float64 pass and
the fused mixed pass on the same scene.  Multi-GPU: one process per GPU, each its own particle set of the same size
over the same geometry (weak scaling, no data-path collective); time = max over ranks.

--impl reference times the reference algorithm on the host cores: the oracle port (oracle/edge2d.py, a CPU
restatement of the reference's numpy path, with the cell list and y bins built once as the reference caches them) over
a fixed seeded sample of 2^16 rows per step, the four kernels each, all cores in spawned worker processes; its
`ms_per_step` is the measured time of that sample (nothing is extrapolated).  `cpu_baseline` of the GPU line is the
same measurement.
"""
import argparse
import json
import math
import os

# expandable segments: the serving stream allocates buffers of widely varying sizes on several streams; without them
# the caching allocator falls back to cudaMalloc (a device synchronisation) on most of those allocations
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

KERNELS = ["cubic", "w2", "w4", "w6"]
METRIC = "particle-edge pairs/s (lambda + 12 moments, 4 kernels, 2^20-particle 2-D scene)"
UNIT = "pairs/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--precision", default="fp64", choices=["mixed", "fp64", "fp32"],
                   help="route of the headline (fp64: the one within 1e-6 relative of the oracle at full size)")
    p.add_argument("--route", default="fused", choices=["fused", "plain"])
    p.add_argument("--particles", type=int, default=1 << 20)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-mesh", action="store_true", help="skip the 3-D closed-surface leg")
    p.add_argument("--leg", choices=["all", "radial", "mesh3d", "serving", "disks"], default="all",
                   help="run one side leg alone (prints its JSON object; for profiling)")
    p.add_argument("--mesh-particles", type=int, default=1 << 21, help="particles of the 3-D closed-surface leg")
    p.add_argument("--no-routes", action="store_true", help="skip the plain / fused fp64 / mixed comparison")
    p.add_argument("--serve-requests", type=int, default=10000,
                   help="requests of the serving stream measured after the main workload (0: skip)")
    return p.parse_args()


WORKLOAD = ("c2: 2^20 particles uniform in [0,4]^2, h=0.02, 64 star polygons (32-512 vertices, one multi-loop "
            "surface), kernels cubic/w2/w4/w6, lambda + 12 moments")


def workload(n, rank):
    """the rank's shard of the 2-D workload: the c2 geometry on every rank, rank 0 the c2 particles, the other ranks
    their own seeded particle sets of the same size (weak scaling)."""
    from warpsphboundaries_b200 import shard, workloads
    loops, X, h = workloads.c2(n_particles=n, seed=0)
    return loops, shard.rank_particles(len(X), rank, X), h


# ----------------------------------------------------------------------------------------------- reference (CPU) arm
def config(n):
    """the workload as both arms report it (the reference arm times a fixed sample of it, stated in `cpu_baseline`)."""
    return {"workload": WORKLOAD, "particles_per_gpu": n, "kernels": KERNELS,
            "l2": "flushed between steps (256 MiB write, untimed)"}


CPU_SAMPLE_ROWS = 1 << 16        # rows of the 2-D scene one reference step evaluates (4 kernels each)
CPU_CHUNK = 4096                 # rows a worker takes at a time

_CPU = {}


def _cpu_init(n):
    """worker set-up: the scene, its cell list and y bins once per process (the reference caches both per surface
    and support, scene.py:273-279, 318-336)."""
    from oracle import edge2d as O
    from warpsphboundaries_b200 import workloads
    loops, X, h = workload(n, 0)
    V, E = workloads.edges_of(loops)
    _CPU.update(X=X, h=h, V=V, E=E, cl=O.build_cell_list(V, E, h), bins=O.ybins(V, E))


def _cpu_chunk(rows):
    """the reference algorithm on one chunk of rows: indicator once, then the four kernels' channels (neighbour slots,
    per-pair closed forms, fixed-order row sums, indicator times the plane constants, physical scaling)."""
    from oracle import edge2d as O
    c = _CPU
    X, h = c["X"][rows], c["h"]
    hs = np.full(len(rows), h)
    ind = O.indicator_binned(c["V"], c["E"], 0, X, hs, c["cl"], c["bins"])
    pairs = 0
    for k in KERNELS:
        _, slots, _ = O.local_twelve(c["V"], c["E"], 0, X, hs, k, h, ind=ind, cl=c["cl"], return_slots=True)
        pairs += sum(len(s) for s in slots)
    return pairs


class CpuReference:
    """the oracle port (oracle/edge2d.py, the reference's numpy algorithm restated) over a fixed seeded sample of the
    scene's rows, in worker processes on the host cores (spawned before any CUDA work)."""

    def __init__(self, n, procs=None):
        import multiprocessing as mp
        self.procs = procs or os.cpu_count() or 1
        rows = np.sort(np.random.default_rng(7).choice(n, min(CPU_SAMPLE_ROWS, n), replace=False))
        self.chunks = [rows[i:i + CPU_CHUNK] for i in range(0, len(rows), CPU_CHUNK)]
        self.pool = mp.get_context("spawn").Pool(self.procs, initializer=_cpu_init, initargs=(n,))
        self.sample = (f"a fixed seeded sample of {len(rows)} of the {n} rows per step, the four kernels each "
                       f"({len(self.chunks)} chunks of {CPU_CHUNK} rows over {self.procs} worker processes)")

    def step(self):
        """(pair evaluations, seconds) of one step."""
        t0 = time.perf_counter()
        pairs = sum(self.pool.map(_cpu_chunk, self.chunks, chunksize=1))
        return pairs, time.perf_counter() - t0

    def close(self):
        self.pool.close()
        self.pool.join()


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    ref = CpuReference(args.particles)
    for _ in range(args.warmup):
        ref.step()
    pairs, secs = 0, 0.0
    for _ in range(args.steps):
        p, t = ref.step()
        pairs += p
        secs += t
    ref.close()
    value = pairs / secs
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)", "config": config(args.particles),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ref.procs, "kind": "port", "sample": ref.sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------------------------- clocks
class Clocks:
    def __init__(self):
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"wsb_clocks_{os.getpid()}.csv")

    def start(self, index):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(index), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], [], set()
        for ln in open(self.path):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------------------------- serving stream
def serving_run(n_requests, dev, pair_density, seed=0, start_load=0.9, max_streams=6):
    """Poisson stream of boundary queries over 32 resident scenes: 16 of the large 2-D kind (64 star polygons each,
    h = 0.02) and 16 of the 3-D kind, as the 3-D configuration has them: 8 closed icospheres of 20480 faces (radius
    U(0.3, 0.8), 5 % jitter, h = 0.03) and 8 solid-sphere scenes whose requests are (query, sphere) rows (radii
    exp U(ln 0.2h, ln 50h), signed distances U(-1.2h, 1.2h) clipped at -R).  Sizes log-uniform in [1e3, 1e6]
    (particles uniform in [0, 4]^2 or [-1, 1]^3, or sphere rows: slices of resident rings), kernels uniform in
    {w2, w4, w6}, 25 % of the 2-D requests with the adjoint.  The arrival rate is a load factor times the capacity
    measured on a saturating run of one request a batch, starting at `start_load` and scaled from the measured busy
    fraction until the device is 80-90 % busy (`max_streams` streams at most; every one tried is reported).  Returns p50 / p99 latency overall and per request class, rates and the
    device busy fraction."""
    import torch
    from warpsphboundaries_b200 import workloads
    from warpsphboundaries_b200.scene import Body, Scene, SurfaceRep
    from warpsphboundaries_b200.serve import BoundaryServer
    h, h3 = 0.02, 0.03
    rng = np.random.default_rng(seed + 77)
    srv = BoundaryServer(dev, streams=4)
    for k in range(16):
        sc = Scene([Body(reps=[SurfaceRep.loops(workloads.stars(64, (32, 512), seed=100 + k))])], dev)
        srv.register(f"scene{k}", sc, h)
    for k in range(8):
        V, Fc = workloads.icosphere(5, float(rng.uniform(0.3, 0.8)), 0.05, seed=200 + k)
        srv.register_mesh(f"mesh{k}", V, Fc, h3)
    for k in range(8):
        srv.register_spheres(f"spheres{k}", h3)
    names = [f"scene{k}" for k in range(16)] + [f"mesh{k}" for k in range(8)] + [f"spheres{k}" for k in range(8)]
    specs = []
    for _ in range(n_requests):
        sid = names[rng.integers(0, 32)]
        rows = int(round(np.exp(rng.uniform(np.log(1e3), np.log(1e6)))))
        kern = ["w2", "w4", "w6"][rng.integers(0, 3)]
        grad = bool(rng.uniform() < 0.25) and sid.startswith("scene")
        specs.append((sid, rows, kern, grad))
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    # the clients' particle positions: slices of resident rings of positions (a simulation's state is resident)
    ring2 = torch.rand((1 << 22, 2), dtype=torch.float64, device=dev, generator=gen) * 4.0
    ring3 = torch.rand((1 << 22, 3), dtype=torch.float64, device=dev, generator=gen) * 2.0 - 1.0
    rr = np.random.default_rng(seed + 78)
    ns_ = 1 << 22
    R = np.exp(rr.uniform(np.log(0.2 * h3), np.log(50 * h3), ns_))
    nv = rr.normal(size=(ns_, 3))
    nv /= np.linalg.norm(nv, axis=1, keepdims=True)
    ringS = torch.tensor(np.concatenate([np.maximum(rr.uniform(-1.2 * h3, 1.2 * h3, ns_), -R)[:, None], nv, R[:, None]],
                                        1), dtype=torch.float64, device=dev)
    cursor = [0, 0, 0]

    def make(sid, rows):
        kind = 2 if sid.startswith("spheres") else int(sid.startswith("mesh"))
        ring = (ring2, ring3, ringS)[kind]
        c = cursor[kind]
        start = c if c + rows <= len(ring) else 0
        cursor[kind] = start + rows
        return ring[start:start + rows], (h if kind == 0 else h3)

    def submit(sid, rows, k, g, arrival=None):
        p, hh = make(sid, rows)
        return srv.submit(sid, p, hh, k, grad=g, arrival=arrival)

    # saturation probes (every request submitted as soon as the previous submit returns, polling in between, as in the
    # stream): the first warms workspaces; the second measures the capacity in rows/s with one request a batch -- a
    # saturated queue merges requests into larger batches than a stream below saturation ever forms, so the merged
    # rate would overstate what a stream can sustain
    burst = specs[: min(600, n_requests)]
    batch_rows = srv.max_batch_rows
    for rep in range(2):
        srv.max_batch_rows = batch_rows if rep == 0 else 1      # a batch takes at least one request
        srv.reset_stats()
        t0 = time.perf_counter()
        done = 0
        for sid, rows, k, g in burst:
            submit(sid, rows, k, g)
            srv.poll()
            for r in srv.completed[done:]:                     # results taken as they complete
                srv.release(r.rid)
            done = len(srv.completed)
        srv.run()
        torch.cuda.synchronize()
        cap_rows = sum(r for _, r, _, _ in burst) / (time.perf_counter() - t0)
        sat = srv.stats()
        for r in srv.completed[done:]:
            srv.release(r.rid)
        srv.completed.clear()
    srv.max_batch_rows = batch_rows
    mean_rows = float(np.mean([r for _, r, _, _ in specs]))
    unit = rng.exponential(1.0, n_requests)                   # inter-arrival times in units of the mean

    def stream(load, count=n_requests):
        rate = load * cap_rows / mean_rows                     # requests per second
        arrivals = np.cumsum(unit[:count] / rate)
        srv.completed.clear()                                  # every request of an earlier stream is released
        srv.reset_stats()
        start = time.perf_counter()
        i = 0
        released = [0]
        while i < count or srv.poll():
            now = time.perf_counter() - start
            while i < count and arrivals[i] <= now:
                sid, rows, k, g = specs[i]
                submit(sid, rows, k, g, arrival=start + arrivals[i])
                i += 1
                while released[0] < len(srv.completed):       # a client takes its results as soon as they are done
                    srv.release(srv.completed[released[0]].rid)
                    released[0] += 1
            srv.poll()
            while released[0] < len(srv.completed):           # the clients take their results and free them
                srv.release(srv.completed[released[0]].rid)
                released[0] += 1
        torch.cuda.synchronize()
        wall = time.perf_counter() - start
        st = srv.stats()
        while released[0] < len(srv.completed):               # the ones completed by the last poll
            srv.release(srv.completed[released[0]].rid)
            released[0] += 1
        return rate, wall, st

    # a warm-up stream of the whole request set (not measured for the report): every (scene, kernel, bucket) key the
    # streams meet runs here first -- the small-batch keys reach their capture threshold and are captured, first-use
    # costs are paid -- so that no measured stream holds a one-off stall
    _, _, warm = stream(start_load, n_requests)
    # the arrival rate is chosen so the device is 80-90 % busy: the first measured stream runs at start_load of the
    # burst capacity; while a stream leaves the device outside that window, the next one's rate is scaled by the busy
    # fraction towards 84 % (at most 6x a step, max_streams streams in all).  The burst's capacity is only a starting point: with several streams and
    # the host issuing one batch at a time it understates what the device absorbs under a stream.
    tried = []
    load = start_load
    for attempt in range(max_streams):
        rate, wall, st = stream(load)
        busy = st.get("gpu_busy") or 0.0
        tried.append({"offered_load": load, "arrival_rate_per_s": rate, "gpu_busy": busy,
                      "p50_ms": st.get("p50_ms"), "p99_ms": st.get("p99_ms"), "classes": st.get("classes"),
                      "host": st.get("host")})
        if 0.8 <= busy <= 0.9:
            break
        # busy is close to proportional to the arrival rate below saturation; above 90 % the queue grows (an overloaded
        # stream's latencies say nothing of the server), so the rate comes down again
        load *= min(6.0, 0.84 / max(busy, 0.05))
    rows_total = sum(r for _, r, _, _ in specs)
    rows_2d = sum(r for sid, r, _, _ in specs if sid.startswith("scene"))
    return {"requests": n_requests, "scenes": 32, "p50_ms": st.get("p50_ms"), "p99_ms": st.get("p99_ms"),
            "classes": st.get("classes"), "graphs": srv.use_graphs,
            "mean_ms": st.get("mean_ms"), "arrival_rate_per_s": rate, "wall_s": wall, "loads_tried": tried,
            "rows_per_s": rows_total / wall, "pairs_per_s_est": rows_2d * pair_density / wall,
            "rows_3d_per_s": (rows_total - rows_2d) / wall,
            "capacity_rows_per_s": cap_rows, "offered_load": load, "gpu_busy": st.get("gpu_busy"),
            "host": st.get("host"), "saturation": {"gpu_busy": sat.get("gpu_busy"), "host": sat.get("host")},
            "warmup": {"requests": n_requests, "gpu_busy": warm.get("gpu_busy"), "p99_ms": warm.get("p99_ms"),
                       "host": warm.get("host")},
            "note": "16 2-D scenes (64 star polygons) + 8 closed 3-D surfaces (20480 faces) + 8 sphere-row scenes; pairs "
                    "estimated from the mean neighbour-pair density of the 2^20-particle 2-D scene for the 2-D rows "
                    "only; rows_3d counts surface queries and sphere rows"}


# ----------------------------------------------------------------------------------------------- our arm
def radial_run(dev, stream, flush, n=1 << 21, steps=10, kernel="w4"):
    """solid spheres in 3-D: 2^21 (query, sphere) shell rows, h = 0.03, radii exp U(ln 0.2h, ln 50h), signed
    distances U(-1.2h, 1.2h) (clipped at -R), all 28 baseline channels, float64, inputs resident."""
    import ctypes

    import torch
    from warpsphboundaries_b200 import _lib
    from warpsphboundaries_b200.kernels import KERNEL_IDS
    from warpsphboundaries_b200.radial import RadialEvaluator
    rng = np.random.default_rng(11)
    h = 0.03
    R = np.exp(rng.uniform(np.log(0.2 * h), np.log(50 * h), n))
    d = np.maximum(rng.uniform(-1.2 * h, 1.2 * h, n), -R)
    nv = rng.normal(size=(n, 3))
    nv /= np.linalg.norm(nv, axis=1, keepdims=True)
    ev = RadialEvaluator("sphere", kernel=kernel)
    b = ev.prepare(d, nv, h, radii=R)
    meta = ev.metadata
    args = (_lib.RADIAL_SPHERE, KERNEL_IDS[kernel], _lib.PREC_FP64, _lib.ptr(b.distances), _lib.ptr(b.radii),
            _lib.ptr(b.normals), _lib.ptr(b.supports), n, meta.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            len(ev.requests), _lib.ptr(b.values), None, None, ctypes.c_void_p(stream.cuda_stream))
    for _ in range(3):
        _lib.check(_lib.lib.wsb_radial_channels(*args))
    tot = 0.0
    for _ in range(steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(_lib.lib.wsb_radial_channels(*args))
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    ms = tot / steps
    byts = n * (6 * 8 + 28 * 8)
    shell = float(np.mean(np.abs(d) < h))
    return {"workload": f"{n} sphere rows, h=0.03, R in [0.2h, 50h], d in [-1.2h, 1.2h], {kernel}, 28 channels, f64",
            "ms": ms, "rows_per_s": n / (ms * 1e-3), "hbm_gbs": byts / (ms * 1e-3) / 1e9,
            "bytes_per_row": 6 * 8 + 28 * 8, "shell_fraction": shell, "kernel": "k_radial"}


def detector_run(ns, pos, sup, pose, obb, ws, need, pairs, stream, flush, steps=5):
    """the delta+ detector inputs on the c2 rows (2^20 particles, h = 0.02, 64 star polygons): wsb_cone_area (half
    angle pi/3, seeded axes) and wsb_dir_extreme (the same vectors) on the workspace prepared once for the c2
    particles, float64, inputs resident; CUDA events around each call, L2 flushed before each."""
    import ctypes

    import torch
    from warpsphboundaries_b200 import _lib
    n = len(pos)
    gen = torch.Generator(device=pos.device).manual_seed(3)
    axes = torch.randn((n, 2), dtype=torch.float64, device=pos.device, generator=gen)
    area = torch.zeros(2 * n, dtype=torch.float64, device=pos.device)
    dmax = torch.zeros(n, dtype=torch.float64, device=pos.device)
    st = ctypes.c_void_p(stream.cuda_stream)
    p = _lib.ptr
    _lib.check(_lib.lib.wsb_aggregate_prepare(ns.handle, p(pos), p(sup), None, n, p(pose), obb, 0, p(ws), need, st),
               "wsb_aggregate_prepare")

    def cone():
        _lib.check(_lib.lib.wsb_cone_area(ns.handle, p(sup), n, p(pose), p(axes), math.pi / 3, p(area), p(ws), need,
                                          st), "wsb_cone_area")

    def dirx():
        _lib.check(_lib.lib.wsb_dir_extreme(ns.handle, n, p(pose), p(axes), p(dmax), p(ws), need, st),
                   "wsb_dir_extreme")

    res = {}
    for name, fn in (("cone_area", cone), ("dir_extreme", dirx)):
        for _ in range(3):
            fn()
        tot = 0.0
        for _ in range(steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize()
            tot += e0.elapsed_time(e1)
        ms = tot / steps
        res[name] = {"ms": ms, "rows_per_s": n / (ms * 1e-3), "pairs_per_s": pairs / (ms * 1e-3)}
    return {"workload": "c2 rows (2^20 particles, h=0.02, 64 star polygons), prepared once; cone_area half angle "
                        "pi/3; f64", "pairs": pairs, **res, "kernels": ["k_cone_area", "k_dir_extreme"]}


def disk_run(dev, stream, flush, steps=5, kernel="w4", n_particles=1 << 20):
    """a fibre bundle: 1024 non-overlapping solid disks, radii U(0.5h, 5h), in [0, 4]^2, h = 0.02, 2^20 particles
    uniform in [0, 4]^2, the twelve channels of every particle (wsb_disk_aggregate), float64, inputs resident; CUDA
    events around the call, L2 flushed before each."""
    import ctypes

    import torch
    from warpsphboundaries_b200 import _lib
    from warpsphboundaries_b200.scene import DiskArrayRep
    from warpsphboundaries_b200.kernels import KERNEL_IDS
    rng = np.random.default_rng(31)
    h = 0.02
    C, R = [], []
    grid = {}
    while len(C) < 1024:                               # rejection sampling on a coarse hash of the centres
        r = float(rng.uniform(0.5 * h, 5 * h))
        c = rng.uniform(r, 4.0 - r, 2)
        key = (int(c[0] / (12 * h)), int(c[1] / (12 * h)))
        near = [j for dx in (-1, 0, 1) for dy in (-1, 0, 1) for j in grid.get((key[0] + dx, key[1] + dy), ())]
        if all(math.hypot(*(c - C[j])) > r + R[j] + 0.1 * h for j in near):
            grid.setdefault(key, []).append(len(C))
            C.append(c)
            R.append(r)
    rep = DiskArrayRep(np.array(C), np.array(R)).to(dev)
    nd = rep.native(h, dev)
    n = n_particles
    X = rng.uniform(0.0, 4.0, (n, 2))
    pos = torch.tensor(X, dtype=torch.float64, device=dev)
    sup = torch.full((n,), h, dtype=torch.float64, device=dev)
    pose = torch.tensor([0.0, 0.0, 1.0, 0.0], dtype=torch.float64, device=dev)
    out = [torch.empty(n * k, dtype=torch.float64, device=dev) for k in (1, 2, 4, 2, 4)]
    st = ctypes.c_void_p(stream.cuda_stream)
    ws, need = nd.workspace(n)
    args = (nd.handle, KERNEL_IDS[kernel], _lib.ptr(pos), _lib.ptr(sup), None, n, _lib.ptr(pose),
            _lib.OUT_ALL | _lib.OUT_ASSIGN, *[_lib.ptr(o) for o in out], _lib.ptr(ws), need, st)
    for _ in range(3):
        _lib.check(_lib.lib.wsb_disk_aggregate(*args), "wsb_disk_aggregate")
    tot = 0.0
    for _ in range(steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(_lib.lib.wsb_disk_aggregate(*args), "wsb_disk_aggregate")
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    ms = tot / steps
    # (particle, disk) pairs within reach, counted once on the host from a sample
    Cn, Rn = np.array(C), np.array(R)
    samp = X[:: max(1, n // 65536)]
    pairs = 0
    for k in range(0, len(samp), 4096):
        D = np.hypot(samp[k:k + 4096, None, 0] - Cn[None, :, 0], samp[k:k + 4096, None, 1] - Cn[None, :, 1])
        pairs += int((D < Rn[None] + h).sum())
    pairs = pairs * n / len(samp)
    return {"workload": f"1024 solid disks (r U(0.5h, 5h)) in [0,4]^2, {n} particles, h=0.02, {kernel}, 12 channels, "
                        "f64", "ms": ms, "particles_per_s": n / (ms * 1e-3), "pairs_est": pairs,
            "pairs_per_s": pairs / (ms * 1e-3), "kernels": ["k_disk_rows", "k_disk_warp"]}


def mesh_run(dev, stream, flush, steps=5, kernel="w4", n_particles=1 << 21):
    """the 3-D scene: 2^21 particles uniform in [-1, 1]^3, h = 0.03, a jittered icosphere of 20480 faces (radius 0.6),
    the 28 baseline channels of every particle, float64, inputs resident; CUDA events around wsb_mesh_channels."""
    import ctypes

    import torch
    from warpsphboundaries_b200 import workloads
    from warpsphboundaries_b200.mesh3d import ClosedMesh
    V, Fc, X, h = workloads.c3(n_particles=n_particles)
    n = len(X)
    m = ClosedMesh(V, Fc, h, dev)
    pos = torch.tensor(X, dtype=torch.float64, device=dev)
    sup = torch.full((n,), h, dtype=torch.float64, device=dev)
    out = torch.empty((n, 28), dtype=torch.float64, device=dev)
    for _ in range(2):
        m.channels(pos, sup, kernel, out=out, stream=stream)
    torch.cuda.synchronize()
    nwork = int(m._ws[2 * ((4 * n + 255) // 256 * 256):][:4].view(torch.int32).item())
    tot = 0.0
    for _ in range(steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m.channels(pos, sup, kernel, out=out, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    ms = tot / steps
    inside = float(out[:, 0].mean().item())
    return {"workload": f"c3: {n} particles in [-1,1]^3, h=0.03, icosphere {len(Fc)} faces (r 0.6, 5% jitter), "
                        f"{kernel}, 28 channels, f64", "ms": ms, "particles_per_s": n / (ms * 1e-3),
            "surface_rows": nwork, "surface_rows_per_s": nwork / (ms * 1e-3), "mean_lambda": inside,
            "kernels": ["k_mesh_rowinfo", "k_mesh_rows", "k_mesh_eval"], "launches_per_step": 3}


def our_arm(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    # the CPU baseline's worker processes, spawned before the first CUDA call
    cpu_ref = CpuReference(args.particles) if rank == 0 and world == 1 and not args.no_cpu_baseline else None
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    from warpsphboundaries_b200 import _lib
    from warpsphboundaries_b200.fixedadj import fixed_topology
    from warpsphboundaries_b200.kernels import KERNEL_IDS, pair_work
    from warpsphboundaries_b200.provider import AnalyticBoundary, FusedGroup, FusedWall, WallOutput
    from warpsphboundaries_b200.scene import Body, Scene, SurfaceRep, _stream
    from warpsphboundaries_b200.shim import KernelFunctions, ParticleState

    loops, X, h = workload(args.particles, rank)
    N = len(X)
    rep = SurfaceRep.loops(loops)
    body = Body(center=(0.0, 0.0), angle=0.0, reps=[rep])
    scene = Scene([body], dev)
    pos = torch.tensor(X, dtype=torch.float64, device=dev).contiguous()
    sup = torch.full((N,), h, dtype=torch.float64, device=dev)
    ns = rep.native(h, dev)
    # neighbour pairs of the workload (kernel independent), counted once outside the timing
    ft = fixed_topology(rep, pos, sup, torch.ones(N, dtype=torch.bool, device=dev), h)
    P = int((ft.e >= 0).sum())
    del ft
    torch.cuda.empty_cache()
    ws, need = ns.workspace(N)
    pose = body.pose_tensor(dev)
    obb = (_lib.ctypes.c_double * 4)(*body.obb())
    outs = {k: [torch.zeros(N, dtype=torch.float64, device=dev), torch.zeros((N, 2), dtype=torch.float64, device=dev),
                torch.zeros((N, 4), dtype=torch.float64, device=dev), torch.zeros((N, 2), dtype=torch.float64, device=dev),
                torch.zeros((N, 4), dtype=torch.float64, device=dev)] for k in KERNELS}
    prec = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED, "fp32": _lib.PREC_FP32}
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    kids = _lib.int32s([KERNEL_IDS[k] for k in KERNELS])
    gout = [_lib.ptrs([outs[k][j] for k in KERNELS]) for j in range(5)]

    def step(precision, timers=None, grouped=True):
        """prepare, then the four kernel groups: one grouped pass (the FusedWall path), or one pass per kernel"""
        ev = []
        e0 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        _lib.check(_lib.lib.wsb_aggregate_prepare(ns.handle, _lib.ptr(pos), _lib.ptr(sup), None, N, _lib.ptr(pose),
                                                  obb, 0, _lib.ptr(ws), need, _stream()), "prepare")
        e1 = torch.cuda.Event(enable_timing=True)
        e1.record(stream)
        ev.append(("prepare", e0, e1))
        if grouped:
            # the library records p0 / p1 around the pair kernel itself (wsb_set_pair_events), so the roofline times
            # k_agg_pairs alone; a / b bracket the whole evaluation (pair pass + expansion)
            p0 = torch.cuda.Event(enable_timing=True)
            p1 = torch.cuda.Event(enable_timing=True)
            p0.record(stream)
            p1.record(stream)
            a = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _lib.check(_lib.lib.wsb_set_pair_events(_lib.ctypes.c_void_p(p0.cuda_event),
                                                    _lib.ctypes.c_void_p(p1.cuda_event)))
            try:
                _lib.check(_lib.lib.wsb_aggregate_evaluate_groups(ns.handle, len(KERNELS), kids, prec[precision],
                                                                  _lib.ptr(sup), N, _lib.ptr(pose),
                                                                  _lib.OUT_ALL | _lib.OUT_ASSIGN, *gout, _lib.ptr(ws),
                                                                  need, _stream()), "evaluate_groups")
            finally:
                _lib.check(_lib.lib.wsb_set_pair_events(None, None))
            b = torch.cuda.Event(enable_timing=True)
            b.record(stream)
            ev.append(("pairs", p0, p1))
            ev.append(("groups", a, b))                     # last: a step ends with the whole evaluation
            if timers is not None:
                timers.append(ev)
            return
        for k in KERNELS:
            o = outs[k]
            a = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            _lib.check(_lib.lib.wsb_aggregate_evaluate(ns.handle, KERNEL_IDS[k], prec[precision], _lib.ptr(sup), N,
                                                       _lib.ptr(pose), _lib.OUT_ALL | _lib.OUT_ASSIGN,
                                                       *[_lib.ptr(t) for t in o],
                                                       _lib.ptr(ws), need, _stream()), "evaluate")
            b = torch.cuda.Event(enable_timing=True)
            b.record(stream)
            ev.append((k, a, b))
        if timers is not None:
            timers.append(ev)

    def timed(precision, steps, warmup, grouped=True):
        for _ in range(warmup):
            step(precision, grouped=grouped)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        timers = []
        for _ in range(steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            step(precision, timers, grouped=grouped)
            torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        step_ms = [ev[0][1].elapsed_time(ev[-1][2]) for ev in timers]
        eval_ms = {name: statistics.mean(e[i][1].elapsed_time(e[i][2]) for e in timers)
                   for i, (name, _, _) in enumerate(timers[0]) if i > 0 and name != "pairs"}
        if any(name == "pairs" for name, _, _ in timers[0]):
            k = [name for name, _, _ in timers[0]].index("pairs")
            timed.pairs_ms = statistics.mean(e[k][1].elapsed_time(e[k][2]) for e in timers)
        prep_ms = statistics.mean(e[0][1].elapsed_time(e[0][2]) for e in timers)
        return sum(step_ms), eval_ms, prep_ms

    clocks = Clocks()
    clocks.start(local)
    total_ms, eval_ms, prep_ms = timed(args.precision, args.steps, args.warmup)
    main_pairs_ms = getattr(timed, "pairs_ms", None)
    clk = clocks.stop()
    # the same four kernels as four single-kernel passes over the prepared rows (reported beside the grouped pass)
    sep_ms = None
    if world == 1:
        ms_s, ev_s, pr_s = timed(args.precision, max(3, args.steps // 2), 1, grouped=False)
        sep_ms = {**ev_s, "prepare": pr_s, "step": ms_s / max(3, args.steps // 2)}
    from warpsphboundaries_b200 import shard
    total_ms = shard.max_over_ranks(total_ms, dev)             # the slowest rank's device time
    pairs_step = P * len(KERNELS)                              # this rank's pairs per step
    job_pairs_step = shard.sum_over_ranks(pairs_step, dev)     # all ranks' pairs per step
    value = job_pairs_step * args.steps / (total_ms * 1e-3)

    # ---- roofline of the dominant kernel (the fused evaluate pass): algorithmic float64 flops per launch
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    import ctypes
    pk = ctypes.CDLL(os.path.join(ROOT, "warpsphboundaries_b200", "_build", "libwsbpeak.so"))
    pk.wsbpeak_fp64_tflops.restype = ctypes.c_double
    pk.wsbpeak_fp32_tflops.restype = ctypes.c_double
    fp64_peak = max(pk.wsbpeak_fp64_tflops(200000) for _ in range(3))
    fp32_peak = max(pk.wsbpeak_fp32_tflops(200000) for _ in range(3))
    flops = {k: P * pair_work(k)["flops"] for k in KERNELS}
    pairs_ms = main_pairs_ms or sum(eval_ms.values())
    achieved = sum(flops.values()) / (pairs_ms * 1e-3) / 1e12
    traffic = None
    tp = os.path.join(ROOT, "profiles", "k_agg_pairs_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp)).get("bytes_per_launch")
        except Exception:
            traffic = None

    # ---- the metric's comparison on the same prepared scene: the plain float64 route (the reference's structure:
    # neighbour slots, the per-slot plan interpreter, the contraction; one aggregate per kernel), the fused float64
    # pass and the fused mixed pass (four kernels in one pass each)
    routes = None
    if world == 1 and not args.no_routes:
        nr = max(3, args.steps // 2)
        ms_f, _, _ = timed("fp64", nr, 1)
        ms_m, _, _ = timed("mixed", nr, 1)
        ms_32, _, _ = timed("fp32", nr, 1)
        ab = AnalyticBoundary(scene, route="plain")
        ps = ParticleState(pos, sup)
        kfs = (KernelFunctions.CubicSpline, KernelFunctions.Wendland2, KernelFunctions.Wendland4,
               KernelFunctions.Wendland6)
        for kf in kfs:
            ab.aggregate(ps, h, kernel=kf, lean=True)
        torch.cuda.synchronize()
        flush.fill_(1)
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        for kf in kfs:
            ab.aggregate(ps, h, kernel=kf, lean=True)
        s1.record(stream)
        torch.cuda.synchronize()
        plain = pairs_step / (s0.elapsed_time(s1) * 1e-3)
        del ab
        torch.cuda.empty_cache()
        fused64 = pairs_step * nr / (ms_f * 1e-3)
        mixed = pairs_step * nr / (ms_m * 1e-3)
        fp32 = pairs_step * nr / (ms_32 * 1e-3)
        headline = {"mixed": mixed, "fp64": fused64, "fp32": fp32}[args.precision]
        routes = {"plain_fp64_pairs_per_s": plain, "fused_fp64_pairs_per_s": fused64, "mixed_pairs_per_s": mixed,
                  "fp32_route_pairs_per_s": fp32,
                  "batched_over_plain": headline / plain, "fused_fp64_over_plain": fused64 / plain,
                  "what": "one step (prepare + the four kernels) per route on the same scene and particles; plain = "
                          "k_fixed_topology slots + k_slot_channels_plain (the reference's per-slot plan "
                          "interpreter) + k_contract, one aggregate per kernel"}

    # ---- the adjoint (d sum(lam) / dx of every particle, w4): prepare + backward per call, timed alone
    adjoint = None
    if world == 1:
        g_lam = torch.ones(N, dtype=torch.float64, device=dev)
        d_pos = torch.zeros((N, 2), dtype=torch.float64, device=dev)

        def back():
            _lib.check(_lib.lib.wsb_aggregate_backward(ns.handle, KERNEL_IDS["w4"], _lib.ptr(pos), _lib.ptr(sup), None,
                                                       N, _lib.ptr(pose), obb, 0, _lib.ptr(g_lam), None, None,
                                                       _lib.ptr(d_pos), None, _lib.ptr(ws), need, _stream()),
                       "backward")
        for _ in range(3):
            back()
        torch.cuda.synchronize()
        tb = 0.0
        for _ in range(5):
            flush.fill_(1)
            torch.cuda.synchronize()
            a0 = torch.cuda.Event(enable_timing=True)
            a1 = torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            back()
            a1.record(stream)
            torch.cuda.synchronize()
            tb += a0.elapsed_time(a1)
        adjoint = {"what": "d sum(lam)/dx of every particle, w4, prepare + k_agg_backward", "ms": tb / 5,
                   "pairs_per_s": P / (tb / 5 * 1e-3)}

    # ---- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        hpos = torch.tensor(X, dtype=torch.float64).pin_memory()
        hsup = torch.full((N,), h, dtype=torch.float64).pin_memory()
        dpos = torch.empty_like(pos)
        dsup = torch.empty_like(sup)
        names = ("lam", "G", "Cov", "m1", "m2")                  # lambda and the twelve moments, every kernel
        host_out = {k: [torch.empty((1, N), dtype=torch.float64).pin_memory(),
                        torch.empty((1, N, 2), dtype=torch.float64).pin_memory(),
                        torch.empty((1, N, 2, 2), dtype=torch.float64).pin_memory(),
                        torch.empty((1, N, 2), dtype=torch.float64).pin_memory(),
                        torch.empty((1, N, 2, 2), dtype=torch.float64).pin_memory()] for k in KERNELS}
        groups = tuple(FusedGroup(k) for k in KERNELS)

        def e2e_step():
            # inputs up, the four kernel groups of the scene in one FusedWall (fused.py:506-547), results down
            dpos.copy_(hpos, non_blocking=True)
            dsup.copy_(hsup, non_blocking=True)
            fw = FusedWall(scene, ParticleState(dpos, dsup), h, groups, precision=args.precision)
            for gi, k in enumerate(KERNELS):
                for dst, name in zip(host_out[k], names):
                    dst.copy_(fw.res[gi][name], non_blocking=True)
            return fw

        for _ in range(args.warmup):
            e2e_step()
        torch.cuda.synchronize()
        # sequential: each step alone (upload, compute, download), L2 flushed before it
        seq = 0.0
        for _ in range(args.steps):
            flush.fill_(1)
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            e2e_step()
            b.record(stream)
            torch.cuda.synchronize()
            seq += a.elapsed_time(b)
        # pipelined, as a host program runs a stream of steps: step k + 1's inputs go up (copy stream) and step k's
        # results come down (second copy stream) while the device computes; every step still moves all its bytes,
        # the inputs are double-buffered, the L2 flush precedes every step's compute, and the timed span runs from
        # the first upload to the last download
        up, down = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)
        dpos2 = [dpos, torch.empty_like(pos)]
        dsup2 = [dsup, torch.empty_like(sup)]
        freed = [None, None]                                   # compute of the step that last read each buffer
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(up)
        for k in range(args.steps):
            sl = k % 2
            if freed[sl] is not None:
                up.wait_event(freed[sl])
            with torch.cuda.stream(up):
                dpos2[sl].copy_(hpos, non_blocking=True)
                dsup2[sl].copy_(hsup, non_blocking=True)
            arrived = torch.cuda.Event()
            arrived.record(up)
            stream.wait_event(arrived)
            flush.fill_(1)
            fw = FusedWall(scene, ParticleState(dpos2[sl], dsup2[sl]), h, groups, precision=args.precision)
            done = torch.cuda.Event()
            done.record(stream)
            freed[sl] = done
            down.wait_event(done)
            with torch.cuda.stream(down):
                for gi, kn in enumerate(KERNELS):
                    for dst, name in zip(host_out[kn], names):
                        src = fw.res[gi][name]
                        src.record_stream(down)            # not reused before its download is done
                        dst.copy_(src, non_blocking=True)
        t1.record(down)
        torch.cuda.synchronize()
        tot = t0.elapsed_time(t1)
        tot = shard.max_over_ranks(tot, dev)
        seq = shard.max_over_ranks(seq, dev)
        e2e = {"value": job_pairs_step * args.steps / (tot * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": N * 3 * 8, "d2h_bytes_per_step": len(KERNELS) * N * 13 * 8,
               "downloads": "lam, G, Cov, m1, m2 of every kernel (13 float64 per particle per kernel)",
               "ms_per_step": tot / args.steps, "pipelined": True,
               # the step's bound: its download over the host link (the upload overlaps it on the other direction)
               "d2h_gbs": len(KERNELS) * N * 13 * 8 * args.steps / (tot * 1e-3) / 1e9,
               "sequential": {"value": job_pairs_step * args.steps / (seq * 1e-3), "ms_per_step": seq / args.steps}}

    def side(fn, *a, **k):
        """a side leg: its result, or its error as one line (a failing side leg never takes the headline line down)"""
        try:
            return fn(*a, **k)
        except Exception as exc:                                   # noqa: BLE001 -- reported in the JSON line
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
            return {"error": f"{type(exc).__name__}: {str(exc)[:300]}"}

    radial = side(radial_run, dev, stream, flush) if world == 1 else None
    detector = side(detector_run, ns, pos, sup, pose, obb, ws, need, P, stream, flush) if world == 1 else None
    disks = side(disk_run, dev, stream, flush) if world == 1 else None
    mesh = side(mesh_run, dev, stream, flush, n_particles=args.mesh_particles) if world == 1 and not args.no_mesh \
        else None

    serving = None
    if rank == 0 and world == 1 and args.serve_requests > 0:
        serving = side(serving_run, args.serve_requests, dev, P / N)

    cpu = None
    if cpu_ref is not None:
        cpu_ref.step()                                             # warm-up
        pr, sec = 0, 0.0
        for _ in range(2):
            p_, t_ = cpu_ref.step()
            pr += p_
            sec += t_
        cpu_ref.close()
        cpu = {"value": pr / sec, "unit": UNIT, "cores": cpu_ref.procs, "kind": "port", "sample": cpu_ref.sample,
               "ms_per_step": sec / 2 * 1e3}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": {"fp64": "f64", "mixed": "f64+f32", "fp32": "f32+f64"}[args.precision],
                "data": "synthetic (seeded)",
                "config": config(N), "pairs_per_kernel": P, "route": args.route, "precision": args.precision,
                "routes": routes,
                "roofline": {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                             "frac": achieved / fp64_peak, "traffic": traffic,
                             "kernel": "k_agg_pairs<KPack<cubic, w2, w4, w6>> (wsb_aggregate_evaluate_groups), timed "
                                       "alone by events the library records around it",
                             "flops_per_pair": {k: pair_work(k)["flops"] for k in KERNELS},
                             "peak_source": "measured: libwsbpeak FP64 FMA stream (this GPU, this run)",
                             "fp32_peak_tflops": fp32_peak, "hbm_gbs_measured_peaks": peaks.get("hbm_gbs")},
                "kernel_ms": {**{k: v for k, v in eval_ms.items()}, "prepare": prep_ms, "k_agg_pairs": pairs_ms},
                "kernel_ms_separate": sep_ms,
                "gpu_launches": args.steps * (5 + 1),   # prepare: 5 kernels; one pair kernel for the four groups
                "clocks": clk, "e2e": e2e, "cpu_baseline": cpu, "serving": serving, "radial": radial, "mesh3d": mesh, "adjoint": adjoint,
                "detector": detector, "disks": disks}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def side_leg(args):
    """one side leg alone on cuda:0 (the 3-D sphere rows or the 3-D closed surface), its JSON object printed."""
    import torch
    dev = torch.device("cuda:0")
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    if args.leg == "radial":
        res = radial_run(dev, stream, flush, steps=args.steps)
    elif args.leg == "serving":
        res = serving_run(args.serve_requests, dev, 2.09)
    elif args.leg == "disks":
        res = disk_run(dev, stream, flush, steps=args.steps)
    else:
        res = mesh_run(dev, stream, flush, steps=args.steps, n_particles=args.mesh_particles)
    print(json.dumps({"leg": args.leg, **res}), flush=True)


def main():
    args = parse()
    if args.leg != "all" and args.impl != "reference":
        side_leg(args)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        our_arm(args)


if __name__ == "__main__":
    main()
