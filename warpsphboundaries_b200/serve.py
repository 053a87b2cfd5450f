"""Continuous-batching request loop for boundary queries from many simulations.

    srv = BoundaryServer(device="cuda:0")
    srv.register("tank-3", scene, support=0.02)                 # geometry, cell grid, indicator cache resident
    rid = srv.submit("tank-3", positions, supports, "w4", grad=False)    # positions / supports: device tensors
    srv.register_mesh("hull-1", vertices, faces, support=0.03)    # 3-D: a closed triangle surface
    srv.run()                                                    # or srv.poll() from the caller's own loop
    res = srv.result(rid)        # {"lam": [B, n], "G": [B, n, 2], "Cov": [B, n, 2, 2], "m1": [B, n, 2], "m2": [B, n, 2, 2]
                                 #  (+ "d_pos": [n, 2] with grad=True: the adjoint of sum(lam))}
                                 # closed surfaces: {"channels": [n, 28]} (wsb_mesh_channels order)
                                 # sphere rows: {"channels": [n, 28]} (baseline(3) order)

Scheduling (one host thread, the caller's):
* requests queue per (scene, kernel, grad) (sphere rows: per kernel); a batch takes the oldest requests of one queue up to `max_batch_rows`
  rows and is admitted while the device memory it reserves (inputs, outputs, workspace) fits `hbm_budget`;
* a batch is ONE fused launch family over the concatenated rows of its requests.  Rows are independent (each row's
  pairs are summed in its own fixed order), so a request's result is bit-identical alone and in any mix;
* batches run on `streams` CUDA streams at once, so requests that arrive while others are on the GPU are admitted as
  stream slots and memory free up, and their work overlaps on the device; `light_streams` more streams of higher
  priority take only batches whose estimated device time (rows x a per-class cost) is below `light_cost_s`, so short
  requests are not queued behind closed-surface batches of several milliseconds and their blocks are scheduled first;
* with `use_graphs=True` (the default), batches of at most `graph_max_rows` rows replay a CUDA graph captured per
  (bucket, scene, kernel) over its own static inputs padded to a power-of-two bucket (padding rows are masked out),
  outputs and workspace; a key is captured once it has been launched `graph_after_uses` times, so one-off keys stay
  eager; the capture runs on a stream of its own that never holds work, so it waits for no batch in flight; any stream
  slot replays a key's graph once the graph's previous replay (with its output copies) has completed, and runs the
  batch eagerly otherwise; captures stop once they hold `graph_budget` bytes;
* solid spheres (`register_spheres`): a request is a set of (query, sphere) rows [n, 5] = (signed distance, outward
  normal, radius) with supports; the rows carry their own geometry and support, so the requests of every sphere
  scene with one kernel share a queue and a batch (one wsb_radial_channels launch over the concatenated rows) serves
  several scenes;
* nothing is allocated per batch: a request's outputs come from a pool of power-of-two buffers when it is submitted
  (on the caller's stream), a scalar support is a view of a resident vector, a single-request batch writes straight
  into the request's outputs, a multi-request batch into persistent per-stream buffers that are then copied into each
  request's outputs;
* admission: a batch is launched while the device memory it reserves fits `hbm_budget`, and `submit` blocks (it
  keeps polling) while the outputs of queued and in-flight requests would exceed it -- back-pressure instead of an
  unbounded queue; a completed request's outputs are the caller's until it releases them, so a caller should
  release results as it takes them;
* latency of a request = completion (its batch's end event observed) - arrival; `stats()` reports p50 / p99.
"""
import itertools
import time
from dataclasses import dataclass
from typing import Dict, List, Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr
from .kernels import KERNEL_IDS
from .provider import FusedGroup, FusedWall
from .scene import SurfaceRep
from .shim import ParticleState, kernelName

F64 = torch.float64
OUT_KEYS = ("lam", "G", "Cov", "m1", "m2")
_TAIL = {"lam": (), "G": (2,), "Cov": (2, 2), "m1": (2,), "m2": (2, 2)}


@dataclass
class Request:
    rid: int
    scene_id: str
    kernel: str
    pos: torch.Tensor
    sup: torch.Tensor
    grad: bool
    arrival: float
    result: Optional[dict] = None
    done: Optional[float] = None
    launched: Optional[float] = None        # host time its batch was issued (queue wait = launched - arrival)
    flat: Optional[torch.Tensor] = None
    nbytes: int = 0


@dataclass
class _Batch:
    reqs: List[Request]
    rows: int
    reserved: int
    event: torch.cuda.Event
    start: Optional[torch.cuda.Event] = None


class _Graph:
    """a captured batch graph: its static inputs (positions, supports, row mask), workspace and outputs, and the event
    of its last replay's end (its output copies included)."""

    def __init__(self, pos, sup, allowed, ws, out):
        self.pos, self.sup, self.allowed, self.ws, self.out = pos, sup, allowed, ws, out
        self.graph = None
        self.done = None


class _Slot:
    """one stream and its persistent batch buffers."""

    def __init__(self, device, light=False):
        self.device = device
        self.light = light            # a light-lane slot: high stream priority, batches of small estimated cost only
        self.stream = torch.cuda.Stream(device=device, priority=-1 if light else 0)
        self.busy = None
        self.cap = 0
        self.B = 0
        self.buf = None

    def workspace(self, nbytes):
        """the persistent workspace of this stream (one batch at a time uses it)."""
        if getattr(self, "ws", None) is None or self.ws.numel() < nbytes:
            with torch.cuda.stream(self.stream):
                self.ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=self.device)
        return self.ws

    def buffers3(self, rows):
        """persistent buffers of a closed-surface batch: positions [cap, 3], supports, channels [cap, 28]."""
        if getattr(self, "buf3", None) is None or rows > self.cap3:
            cap = max(rows, int(1.5 * getattr(self, "cap3", 0)), 1 << 16)
            with torch.cuda.stream(self.stream):
                self.buf3 = {"pos": torch.empty((cap, 3), dtype=F64, device=self.device),
                             "sup": torch.empty(cap, dtype=F64, device=self.device),
                             "chan": torch.empty((cap, 28), dtype=F64, device=self.device)}
            self.cap3 = cap
        return self.buf3

    def buffers_sph(self, rows):
        """persistent buffers of a sphere batch: rows [cap, 5], supports, channels [cap, 28], invariants, status."""
        if getattr(self, "bufs", None) is None or rows > self.caps:
            cap = max(rows, int(1.5 * getattr(self, "caps", 0)), 1 << 16)
            with torch.cuda.stream(self.stream):
                self.bufs = {"rows": torch.empty((cap, 5), dtype=F64, device=self.device),
                             "sup": torch.empty(cap, dtype=F64, device=self.device),
                             "chan": torch.empty((cap, 28), dtype=F64, device=self.device),
                             "work": torch.empty((cap, 9), dtype=F64, device=self.device),
                             "status": torch.empty(cap, dtype=torch.int32, device=self.device)}
            self.caps = cap
        return self.bufs

    def buffers(self, rows, B):
        """persistent batch buffers for `rows` rows of a B-body scene (grown geometrically, allocated on this stream)."""
        if self.buf is None or rows > self.cap or B > self.B:
            cap = max(rows, int(1.5 * self.cap), 1 << 16)
            self.B = max(B, self.B)
            with torch.cuda.stream(self.stream):
                self.buf = {"pos": torch.empty((cap, 2), dtype=F64, device=self.device),
                            "sup": torch.empty(cap, dtype=F64, device=self.device),
                            "one": torch.ones(cap, dtype=F64, device=self.device),
                            "d_pos": torch.empty((cap, 2), dtype=F64, device=self.device),
                            **{k: torch.empty((self.B, cap) + _TAIL[k], dtype=F64, device=self.device)
                               for k in OUT_KEYS}}
            self.cap = cap
        return self.buf


class BoundaryServer:
    def __init__(self, device="cuda:0", streams=4, max_batch_rows=1 << 20, hbm_budget=None, use_graphs=True,
                 graph_max_rows=1 << 16, precision="fp64", graph_after_uses=4, pool_limit=None,
                 graph_budget=2 << 30, light_streams=2, light_cost_s=1e-3):
        self.device = torch.device(device)
        self.scenes: Dict[str, tuple] = {}
        self.queues: Dict[tuple, List[Request]] = {}
        self.slots = [_Slot(self.device) for _ in range(streams)] + \
            [_Slot(self.device, light=True) for _ in range(light_streams)]
        self.light_cost_s = float(light_cost_s)
        self.max_batch_rows = int(max_batch_rows)
        free, total = torch.cuda.mem_get_info(self.device)
        self.hbm_budget = int(hbm_budget if hbm_budget is not None else 0.25 * free)
        self.reserved = 0
        self.use_graphs = use_graphs
        self.graph_max_rows = int(graph_max_rows)
        self.graph_after_uses = int(graph_after_uses)
        self.precision = precision
        self.graphs = {}                    # (bucket, scene, kernel) -> _Graph
        self.cap_stream = torch.cuda.Stream(self.device) if use_graphs else None    # captures only: never holds work
        self.graph_budget = int(graph_budget)  # device bytes all captured graphs may hold (their outputs, workspaces)
        self.graph_bytes = 0
        self.uses = {}
        self.requests: Dict[int, Request] = {}
        self._ids = itertools.count()
        self.completed: List[Request] = []
        self.n_queued = 0
        self.n_inflight = 0
        self.t_first = None
        self.t_last = None
        self.plans = {}
        self.ws_bytes = 0
        self.pool = {}                      # size class -> free output buffers
        self.pooled_bytes = 0
        self.pool_limit = int(pool_limit if pool_limit is not None else 0.1 * free)
        self.held_bytes = 0                 # outputs of queued and in-flight requests
        self.support_vecs = {}              # support value -> resident vector filled with it
        self.intervals = []                 # (start, end) events of retired batches (device busy time)
        self.host = {"batches": 0, "requests": 0, "launch_s": 0.0, "captures": 0, "replays": 0, "graph_busy": 0}   # host-side cost of the launches

    # ------------------------------------------------------------------ scenes
    def register(self, scene_id, scene, support):
        """keep `scene` resident: its surfaces' static structures are built now for `support`, with the launch plan
        (pose, body box, surface handles) resolved once."""
        for b in scene.bodies:
            for r in b.fused_reps(float(support), self.device):     # boxes, cavities, sampled distances: polygons
                if not isinstance(r, SurfaceRep) or r._triangle:
                    raise NotImplementedError("BoundaryServer: surface loops only (no disk sets, no conditioned "
                                              "single triangles)")
        plan = []
        for b in scene.bodies:
            reps = [r.native(float(support), self.device) for r in b.fused_reps(float(support), self.device)]
            plan.append((b.pose_tensor(self.device), (_lib.ctypes.c_double * 4)(*b.obb()), int(b.unbounded()), reps))
            for ns in reps:
                self.ws_bytes = max(self.ws_bytes, int(lib.wsb_aggregate_workspace_size(ns.handle, self.max_batch_rows)) +
                                    int(lib.wsb_aggregate_staging_size(ns.handle, self.max_batch_rows)))
        self.scenes[scene_id] = (scene, float(support))
        self.plans[scene_id] = plan

    def register_mesh(self, scene_id, vertices, faces, support):
        """keep a closed triangle surface resident (3-D): requests on it return the 28 baseline channels per row
        ("channels" [n, 28], the order of wsb_mesh_channels)."""
        from .mesh3d import ClosedMesh
        mesh = ClosedMesh(vertices, faces, float(support), self.device)
        self.scenes[scene_id] = (mesh, float(support))
        self.plans[scene_id] = None
        self.ws_bytes = max(self.ws_bytes, int(lib.wsb_mesh_workspace_size(mesh.handle, self.max_batch_rows)))

    def register_spheres(self, scene_id, support):
        """a resident solid-sphere scene (3-D): requests are (query, sphere) rows [n, 5] = (signed outward distance
        |x - c| - R, unit outward normal, radius R) and return the 28 baseline channels per row
        (fluxbridge RadialEvaluator("sphere"), float64)."""
        self.scenes[scene_id] = ("spheres", float(support))
        self.plans[scene_id] = "spheres"

    def _is_mesh(self, scene_id):
        return self.plans.get(scene_id, ()) is None

    def _is_spheres(self, scene_id):
        return self.plans.get(scene_id, ()) == "spheres"

    def _qkey(self, r):
        """the queue of a request: requests of one queue run in one launch family.  Sphere rows carry their own
        geometry and support, so the requests of every sphere scene with one kernel share a queue (one launch serves
        several scenes); other requests queue per (scene, kernel, adjoint)."""
        if self._is_spheres(r.scene_id):
            return ("<spheres>", r.kernel, False)
        return (r.scene_id, r.kernel, r.grad)

    def _cls(self, r):
        """the request class of the per-class latency report."""
        if self._is_mesh(r.scene_id):
            return "3d_surface"
        if self._is_spheres(r.scene_id):
            return "3d_spheres"
        return "2d_grad" if r.grad else "2d"

    # ------------------------------------------------------------------ requests
    def submit(self, scene_id, positions, supports, kernel, grad=False, arrival=None):
        """queue a request; its outputs are allocated here, on the caller's stream."""
        if scene_id not in self.scenes:
            raise KeyError(f"unknown scene {scene_id!r}")
        kname = kernelName(kernel)
        pos = positions.to(self.device, F64).contiguous()
        if torch.is_tensor(supports):
            sup = supports.to(self.device, F64).contiguous()
        else:
            sup = self._support_vec(float(supports), len(pos))
        r = Request(next(self._ids), scene_id, kname, pos, sup, bool(grad),
                    time.perf_counter() if arrival is None else arrival)
        if self._is_mesh(scene_id) or self._is_spheres(scene_id):
            return self._submit_mesh(r)
        B, n = len(self.scenes[scene_id][0].bodies), len(pos)
        r.nbytes = self._admit(13 * B * n + (2 * n if r.grad else 0))
        flat = self._take(13 * B * n + (2 * n if r.grad else 0))          # one buffer, from the pool when possible
        r.flat = flat
        r.result, off = {}, 0
        for k in OUT_KEYS:
            size = B * n * int(np.prod(_TAIL[k], dtype=np.int64))
            r.result[k] = flat[off:off + size].view((B, n) + _TAIL[k])
            off += size
        if r.grad:
            r.result["d_pos"] = flat[off:off + 2 * n].view(n, 2)
            r.result["d_pos"].zero_()
        self.requests[r.rid] = r
        self.queues.setdefault(self._qkey(r), []).append(r)
        self.n_queued += 1
        return r.rid

    def _submit_mesh(self, r):
        if r.grad:
            raise NotImplementedError("BoundaryServer: 3-D scenes serve the channels, not the adjoint")
        width = 5 if self._is_spheres(r.scene_id) else 3
        if r.pos.dim() != 2 or r.pos.shape[1] != width:
            raise ValueError(f"BoundaryServer: this scene's requests take rows [n, {width}]")
        n = len(r.pos)
        r.nbytes = self._admit(28 * n)
        r.flat = self._take(28 * n)
        r.result = {"channels": r.flat[:28 * n].view(n, 28)}
        self.requests[r.rid] = r
        self.queues.setdefault(self._qkey(r), []).append(r)
        self.n_queued += 1
        return r.rid

    def result(self, rid):
        """the outputs of a request (owned by the request; complete once `poll` has retired its batch)."""
        return self.requests[rid].result

    def release(self, rid):
        """hand a finished request's output buffer back to the pool (its result tensors must not be used after)."""
        r = self.requests.pop(rid)
        if r.done is None:
            raise ValueError("release: the request has not completed")
        flat = getattr(r, "flat", None)
        if flat is not None and self.pooled_bytes + 8 * flat.numel() <= self.pool_limit:
            self.pool.setdefault(flat.numel(), []).append(flat)
            self.pooled_bytes += 8 * flat.numel()
        r.result = None
        r.flat = None

    @staticmethod
    def _size_class(n):
        """the float64 elements of the pooled buffer that holds n (a power of two, at least 4096)."""
        return max(1 << 12, 1 << (int(n) - 1).bit_length())

    def _admit(self, n):
        """back-pressure for a request of n float64 outputs: the outputs of queued and in-flight requests count against
        hbm_budget; while they would exceed it the caller waits (polling).  A completed request's outputs are the
        caller's until it releases them (a caller that holds many unreleased results holds that memory).  Returns the
        bytes counted (the pooled size class)."""
        nbytes = 8 * self._size_class(n)
        while self.held_bytes + nbytes > self.hbm_budget and (self.n_queued or self.n_inflight):
            self.poll()
        self.held_bytes += nbytes
        return nbytes

    def _support_vec(self, value, n):
        """a view of n copies of `value` from a resident vector (grown geometrically; no allocation per request)."""
        v = self.support_vecs.get(value)
        if v is None or v.numel() < n:
            v = torch.full((max(n, self.max_batch_rows, 2 * (0 if v is None else v.numel())),), value, dtype=F64,
                           device=self.device)
            self.support_vecs[value] = v
        return v[:n]

    def _take(self, n):
        """a float64 buffer of at least n elements: pooled size classes (powers of two) avoid allocator calls in the
        steady state."""
        cls = self._size_class(n)
        lst = self.pool.get(cls)
        if lst:
            self.pooled_bytes -= 8 * cls
            return lst.pop()
        return torch.empty(cls, dtype=F64, device=self.device)

    # ------------------------------------------------------------------ bytes a batch holds on the device
    def _bytes(self, scene, support, rows, grad):
        if isinstance(scene, str):                                    # sphere rows
            return (8 * 28 + 8 * 6 + 8 * 9 + 4) * rows
        if not hasattr(scene, "bodies"):                              # a closed surface
            return (8 * 28 + 32) * rows + int(lib.wsb_mesh_workspace_size(scene.handle, rows))
        B = len(scene.bodies)
        ws = 0
        for b in scene.bodies:
            for r in b.fused_reps(support, self.device):
                h_ = r.native(support, self.device).handle
                ws = max(ws, int(lib.wsb_aggregate_workspace_size(h_, rows)) + int(lib.wsb_aggregate_staging_size(h_, rows)))
        return (8 * 13 * B + 24 + (16 if grad else 0)) * rows + ws

    # ------------------------------------------------------------------ the loop
    # device seconds a row, by request class (measured on B200 at large batches: 2-D one kernel with prepare, the
    # adjoint about as much again; closed surfaces of the 3-D configuration; sphere rows), for the lane choice only
    _ROW_COST = {"2d": 2.5e-10, "2d_grad": 5e-10, "3d_surface": 6.5e-9, "3d_spheres": 2.5e-10}

    def _cost(self, r):
        """the estimated device time of a request (seconds): what sends a batch to the light lanes."""
        return 2e-5 + len(r.pos) * self._ROW_COST[self._cls(r)]

    def _next_batch(self, light_only=False):
        """the queue whose oldest request arrived first; its oldest requests up to max_batch_rows rows.  light_only:
        among the queues whose head is light (estimated cost below light_cost_s), up to that cost."""
        best = None
        for key, q in self.queues.items():
            if not q or (light_only and self._cost(q[0]) >= self.light_cost_s):
                continue
            if best is None or q[0].arrival < self.queues[best][0].arrival:
                best = key
        if best is None:
            return None
        q = self.queues[best]
        take, rows, cost = [], 0, 0.0
        while q and (not take or (rows + len(q[0].pos) <= self.max_batch_rows and
                                  (not light_only or cost + self._cost(q[0]) < self.light_cost_s))):
            r = q.pop(0)
            take.append(r)
            rows += len(r.pos)
            cost += self._cost(r)
        self.n_queued -= len(take)
        return take, rows

    def poll(self):
        """retire finished batches, then launch queued work while stream slots and memory allow.  Returns the number
        of requests still queued plus batches in flight."""
        for s in self.slots:
            b = s.busy
            if b is not None and b.event.query():
                # the caller's stream owns the requests' tensors: order it after this batch so their memory is only
                # reused once the batch is done (the event has completed: this wait costs nothing)
                torch.cuda.current_stream(self.device).wait_event(b.event)
                t = time.perf_counter()
                for r in b.reqs:
                    r.done = t
                    self.completed.append(r)
                    self.held_bytes -= r.nbytes
                self.reserved -= b.reserved
                self.intervals.append((b.start, b.event))
                s.busy = None
                self.n_inflight -= 1
                self.t_last = t
        while self.n_queued:
            # a free standard slot takes the oldest queue's batch; with only light slots free, the oldest light batch
            # (so short requests do not wait behind batches of several milliseconds)
            free = [i for i, s in enumerate(self.slots) if s.busy is None]
            if not free:
                break
            std = [i for i in free if not self.slots[i].light]
            picked = self._next_batch(light_only=not std)
            if picked is None:
                break
            reqs, rows = picked
            light = [i for i in free if self.slots[i].light]
            si = light[0] if light and sum(self._cost(r) for r in reqs) < self.light_cost_s else std[0] if std else \
                light[0]
            scene, support = self.scenes[reqs[0].scene_id]
            need = self._bytes(scene, support, rows, reqs[0].grad)
            if self.reserved and self.reserved + need > self.hbm_budget:
                q = self.queues[self._qkey(reqs[0])]
                q[:0] = reqs                        # not admitted yet: back to the head of its queue
                self.n_queued += len(reqs)
                break
            self.reserved += need
            t0 = time.perf_counter()
            for r in reqs:
                r.launched = t0
            self._launch(si, reqs, rows, scene, support, need)
            self.host["launch_s"] += time.perf_counter() - t0
            self.host["batches"] += 1
            self.host["requests"] += len(reqs)
            self.n_inflight += 1
        return self.n_queued + self.n_inflight

    def run(self):
        while self.poll():
            time.sleep(0)

    # ------------------------------------------------------------------ launches
    def _launch_mesh(self, si, reqs, rows, mesh, need):
        slot = self.slots[si]
        if self.t_first is None:
            self.t_first = time.perf_counter()
        slot.stream.wait_stream(torch.cuda.current_stream(self.device))
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(slot.stream)
        with torch.cuda.stream(slot.stream):
            if len(reqs) == 1:
                pos, sup, out = reqs[0].pos, reqs[0].sup, reqs[0].result["channels"]
            else:
                buf = slot.buffers3(rows)
                pos, sup, out = buf["pos"][:rows], buf["sup"][:rows], buf["chan"][:rows]
                off = 0
                for r in reqs:
                    n = len(r.pos)
                    pos[off:off + n].copy_(r.pos)
                    sup[off:off + n].copy_(r.sup)
                    off += n
            ws = slot.workspace(self.ws_bytes)
            check(lib.wsb_mesh_channels(mesh.handle, KERNEL_IDS[reqs[0].kernel], ptr(pos), ptr(sup), rows, ptr(out),
                                        None, ptr(ws), ws.numel(), _lib.ctypes.c_void_p(slot.stream.cuda_stream)),
                  "wsb_mesh_channels")
            if len(reqs) > 1:
                off = 0
                for r in reqs:
                    n = len(r.pos)
                    r.result["channels"].copy_(out[off:off + n])
                    off += n
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(slot.stream)
        slot.busy = _Batch(reqs, rows, need, ev, ev0)

    def _launch_spheres(self, si, reqs, rows, support, need):
        """one wsb_radial_channels launch over the concatenated sphere rows of the batch."""
        slot = self.slots[si]
        if self.t_first is None:
            self.t_first = time.perf_counter()
        slot.stream.wait_stream(torch.cuda.current_stream(self.device))
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(slot.stream)
        with torch.cuda.stream(slot.stream):
            buf = slot.buffers_sph(rows)
            off = 0
            for r in reqs:
                n = len(r.pos)
                buf["rows"][off:off + n].copy_(r.pos)
                buf["sup"][off:off + n].copy_(r.sup)
                off += n
            rw = buf["rows"][:rows]
            d = rw[:, 0].contiguous()
            nrm = rw[:, 1:4].contiguous()
            rad = rw[:, 4].contiguous()
            out = buf["chan"][:rows]
            check(lib.wsb_radial_channels(_lib.RADIAL_SPHERE, KERNEL_IDS[reqs[0].kernel], _lib.PREC_FP64, ptr(d),
                                          ptr(rad), ptr(nrm), ptr(buf["sup"]), rows, self._radial_meta(),
                                          28, ptr(out), ptr(buf["work"]), ptr(buf["status"]),
                                          _lib.ctypes.c_void_p(slot.stream.cuda_stream)), "wsb_radial_channels")
            off = 0
            for r in reqs:
                n = len(r.pos)
                r.result["channels"].copy_(out[off:off + n])
                off += n
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(slot.stream)
        slot.busy = _Batch(reqs, rows, need, ev, ev0)

    def _radial_meta(self):
        if getattr(self, "_meta", None) is None:
            from .radial import RadialEvaluator
            self._meta_ev = RadialEvaluator("sphere", kernel="w2", device=self.device)
            self._meta = self._meta_ev.metadata.ctypes.data_as(_lib.ctypes.POINTER(_lib.ctypes.c_int32))
        return self._meta

    def _launch(self, si, reqs, rows, scene, support, need):
        if self._is_mesh(reqs[0].scene_id):
            return self._launch_mesh(si, reqs, rows, scene, need)
        if self._is_spheres(reqs[0].scene_id):
            return self._launch_spheres(si, reqs, rows, support, need)
        slot = self.slots[si]
        kname, grad = reqs[0].kernel, reqs[0].grad
        B = len(scene.bodies)
        plan = self.plans[reqs[0].scene_id]
        if self.t_first is None:
            self.t_first = time.perf_counter()
        slot.stream.wait_stream(torch.cuda.current_stream(self.device))   # inputs and outputs come from the caller
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record(slot.stream)
        with torch.cuda.stream(slot.stream):
            single = len(reqs) == 1
            if single:
                pos, sup, outs = reqs[0].pos, reqs[0].sup, reqs[0].result
            else:
                buf = slot.buffers(rows, B)
                pos, sup = buf["pos"][:rows], buf["sup"][:rows]
                off = 0
                for r in reqs:
                    n = len(r.pos)
                    pos[off:off + n].copy_(r.pos)
                    sup[off:off + n].copy_(r.sup)
                    off += n
                outs = {k: buf[k][:B, :rows] for k in OUT_KEYS}
            gkey = None
            if self.use_graphs and not grad and rows <= self.graph_max_rows:
                gkey = (self._bucket(rows), reqs[0].scene_id, kname)
                self.uses[gkey] = self.uses.get(gkey, 0) + 1
                if gkey not in self.graphs and self.uses[gkey] < self.graph_after_uses:
                    gkey = None
            if gkey is not None and self._graph_run(slot, gkey, plan, support, kname, pos, sup, rows, outs):
                pass
            else:
                self._aggregate(plan, kname, pos, sup, None, rows, outs, slot.workspace(self.ws_bytes),
                                slot.stream)
            if grad:
                if single:
                    d_pos = reqs[0].result["d_pos"]
                else:
                    d_pos = slot.buffers(rows, B)["d_pos"][:rows]
                    d_pos.zero_()
                self._adjoint(plan, support, kname, pos, sup, d_pos, slot)
            if not single:
                off = 0
                for r in reqs:
                    n = len(r.pos)
                    for k in OUT_KEYS:
                        r.result[k].copy_(outs[k][:, off:off + n])
                    if grad:
                        r.result["d_pos"].copy_(d_pos[off:off + n])
                    off += n
            ev = torch.cuda.Event(enable_timing=True)
            ev.record(slot.stream)
        slot.busy = _Batch(reqs, rows, need, ev, ev0)

    def _aggregate(self, plan, kname, pos, sup, allowed, n, outs, ws, stream):
        """the fused aggregate of every body and surface of a resolved scene into `outs` (the first surface of a body
        assigns its rows, the others add)."""
        kid = KERNEL_IDS[kname]
        prec = _lib.PREC_MIXED if self.precision == "mixed" else _lib.PREC_FP64
        st = _lib.ctypes.c_void_p(stream.cuda_stream)
        for bi, (pose, obb, unbounded, reps) in enumerate(plan):
            o = [ptr(outs[k][bi]) for k in OUT_KEYS]
            for ri, ns in enumerate(reps):
                mode = _lib.OUT_ALL | (_lib.OUT_ASSIGN if ri == 0 else 0)
                check(lib.wsb_aggregate(ns.handle, kid, prec, ptr(pos), ptr(sup), ptr(allowed), n, ptr(pose), obb,
                                        unbounded, mode, *o, ptr(ws), ws.numel(), None, st), "wsb_aggregate")

    def _adjoint(self, plan, support, kname, pos, sup, d_pos, slot):
        """adds d(sum lam)/dpos of every body and surface into d_pos (the gradient-flagged requests)."""
        N = len(pos)
        g_lam = slot.buffers(N, len(plan))["one"][:N]
        ws = slot.workspace(self.ws_bytes)
        kid = KERNEL_IDS[kname]
        for pose, obb, unbounded, reps in plan:
            for ns in reps:
                check(lib.wsb_aggregate_backward(ns.handle, kid, ptr(pos), ptr(sup), None, N, ptr(pose), obb,
                                                 unbounded, ptr(g_lam), None, None, ptr(d_pos), None, ptr(ws),
                                                 ws.numel(), _lib.ctypes.c_void_p(slot.stream.cuda_stream)),
                      "wsb_aggregate_backward")

    @staticmethod
    def _bucket(rows):
        return max(1024, 1 << (int(rows) - 1).bit_length())

    def _graph_run(self, slot, key, plan, support, kname, pos, sup, rows, outs):
        """replay the key's graph for this batch on the slot's stream (capturing it first if the budget allows).
        False: the batch runs eagerly (over budget, or the graph's previous replay has not completed)."""
        bucket = key[0]
        B = len(plan)
        g = self.graphs.get(key)
        if g is None:
            # graph-owned static inputs, workspace and outputs: a captured graph keeps its pointers, so they are never
            # freed; a capture that would take the graphs past `graph_budget` is not made
            need = max(int(lib.wsb_aggregate_workspace_size(ns.handle, bucket)) +
                       int(lib.wsb_aggregate_staging_size(ns.handle, bucket))
                       for _, _, _, reps in plan for ns in reps)
            gbytes = need + 8 * 13 * B * bucket + 28 * bucket
            if self.graph_bytes + gbytes > self.graph_budget:
                return False
            self.graph_bytes += gbytes
            with torch.cuda.stream(slot.stream):
                g = _Graph(torch.zeros((bucket, 2), dtype=F64, device=self.device),
                           torch.full((bucket,), support, dtype=F64, device=self.device),
                           torch.ones(bucket, dtype=torch.int32, device=self.device),
                           torch.empty(need, dtype=torch.uint8, device=self.device),
                           {k: torch.empty((B, bucket) + _TAIL[k], dtype=F64, device=self.device) for k in OUT_KEYS})
                # eager run on the slot's stream (one-time library setup happens outside the capture; the replay
                # below is ordered after it on the same stream)
                self._aggregate(plan, kname, g.pos, g.sup, g.allowed, bucket, g.out, g.ws, slot.stream)
            # captured on the capture stream, which holds no work: recording launches waits for nothing in flight
            # (torch.cuda.graph() would also synchronise and empty the allocator's cache)
            graph = torch.cuda.CUDAGraph()
            with torch.cuda.stream(self.cap_stream):
                graph.capture_begin(capture_error_mode="thread_local")
                try:
                    self._aggregate(plan, kname, g.pos, g.sup, g.allowed, bucket, g.out, g.ws, self.cap_stream)
                finally:
                    graph.capture_end()
            g.graph = graph
            self.graphs[key] = g
            self.host["captures"] += 1
        elif g.done is not None and not g.done.query():
            self.host["graph_busy"] += 1
            return False                                        # replaying on another slot: this batch runs eagerly
        g.pos[:rows].copy_(pos)
        g.sup[:rows].copy_(sup)
        g.allowed[:rows].fill_(1)
        g.allowed[rows:].fill_(0)
        g.graph.replay()
        for k in OUT_KEYS:
            outs[k].copy_(g.out[k][:, :rows])
        g.done = torch.cuda.Event()
        g.done.record(slot.stream)
        self.host["replays"] += 1
        return True

    # ------------------------------------------------------------------ statistics
    def stats(self):
        lat = np.array([(r.done - r.arrival) * 1e3 for r in self.completed])
        out = {"requests": len(self.completed)}
        if len(lat):
            out.update(p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                       mean_ms=float(lat.mean()), max_ms=float(lat.max()))
        classes = {}
        for r in self.completed:
            classes.setdefault(self._cls(r), []).append(((r.done - r.arrival) * 1e3, (r.launched - r.arrival) * 1e3))
        # per class: latency p50 / p99, and the p99 of the queue wait (arrival to the batch's issue) beside it
        out["classes"] = {c: {"requests": len(v), "p50_ms": float(np.percentile([x for x, _ in v], 50)),
                              "p99_ms": float(np.percentile([x for x, _ in v], 99)),
                              "wait_p99_ms": float(np.percentile([w for _, w in v], 99))}
                          for c, v in sorted(classes.items())}
        if self.t_first is not None and self.t_last is not None:
            out["wall_s"] = self.t_last - self.t_first
        if self.intervals:
            # device busy fraction: the union of the batches' [start, end] intervals over the span they cover
            ref = self.intervals[0][0]
            iv = sorted((ref.elapsed_time(a), ref.elapsed_time(b)) for a, b in self.intervals)
            busy, cur0, cur1 = 0.0, iv[0][0], iv[0][1]
            for a, b in iv[1:]:
                if a > cur1:
                    busy += cur1 - cur0
                    cur0, cur1 = a, b
                else:
                    cur1 = max(cur1, b)
            busy += cur1 - cur0
            span = max(b for _, b in iv) - min(a for a, _ in iv)
            out["gpu_busy"] = busy / span if span > 0 else None
        hb = self.host
        if hb["batches"]:
            # host time spent issuing batches (argument setup, copies into batch buffers, launches, graph replays)
            out["host"] = {"batches": hb["batches"], "requests_per_batch": hb["requests"] / hb["batches"],
                           "launch_ms_per_batch": 1e3 * hb["launch_s"] / hb["batches"], "captures": hb["captures"],
                           "graph_replays": hb["replays"], "graph_busy_fallbacks": hb["graph_busy"]}
            if out.get("wall_s"):
                out["host"]["launch_fraction"] = hb["launch_s"] / out["wall_s"]
        return out

    def reset_stats(self):
        """forget completed requests' latencies and the busy intervals (e.g. after a warm-up)."""
        self.completed.clear()
        self.intervals.clear()
        self.t_first = self.t_last = None
        self.host = {"batches": 0, "requests": 0, "launch_s": 0.0, "captures": 0, "replays": 0, "graph_busy": 0}
