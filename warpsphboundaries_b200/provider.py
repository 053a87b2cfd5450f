"""The analytic boundary as a provider for an SPH scheme: the drop-in for `AnalyticBoundary` /
`BoundaryProvider` (src/warpSPHBoundaries/scene/provider.py:38-113) and `FusedWall`
(src/warpSPHBoundaries/scene/fused.py:500-725).

    ab = AnalyticBoundary(scene)                      # route="fused" (default) or "plain"; precision "fp64" | "mixed"
    fw = ab.aggregate(ps, support, kernel=KernelFunctions.Wendland4, lean=True)
    fw.out["lam"] [B, N], fw.out["G"] [B, N, 2], fw.out["Cov"] [B, N, 2, 2]      # float64, world frame
    fw.evaluate((WallOutput("m1", 0, "m1"), WallOutput("m2", 0, "m2"), WallOutput("A", 0, "a1g1")), a1=a1)

Routes:
  fused  wsb_aggregate: body frame, broadphase, cell-sorted rows, float64 neighbour predicate and the closed-form
         channels of each neighbour pair accumulated in registers, indicator, scaling, rotation -- one pass per
         (body, surface), no per-pair storage.
  plain  the reference's structure on the GPU: fixed-capacity slots (wsb_fixed_topology), the per-slot plan
         interpreter (wsb_slot_channels_plain) writing c[N*K, 12], and the per-row contraction (wsb_contract).

Kernel groups: the smoothing kernels (cubic, w2, w4, w6, quartic, quintic, poly6) and the wall-operator kernels of the
delta+ layout: `cone` (its G is the free-surface cover vector), `lw2` / `lw4` (W'/r; the `lap` output kind is
2 lam - tr Cov, the wall Laplacian before the scheme's factor) and the tensile `w2p5` / `w4p5` (W^5, degree 25 / 40,
by chord quadrature on the fused route; their groups serve G only).  `cone_area` (the wedge and full-disk areas of
the solid in the support) and `dir_extreme` (the largest direction cosine towards the solid) run on the prepared rows of
every (body, surface): wsb_cone_area / wsb_dir_extreme.
"""
import math
from dataclasses import dataclass
from typing import Optional, Protocol, runtime_checkable

import torch

from . import _lib
from ._lib import check, lib, ptr
from .fixedadj import body_candidates, fixed_adjacency
from .kernels import KERNEL_IDS, QUAD_KERNEL_IDS

_GROUP_IDS = {**KERNEL_IDS, **QUAD_KERNEL_IDS}     # every kernel a FusedWall group may name
from .scene import DiskArrayRep, Scene, SurfaceRep, _stream
from .shim import (GradientScheme, KernelFunctions, OperationDirection, OperationProperties, WarpOperation, kernelName,
                   queryAllowed)

F64 = torch.float64
KINDS = {"lam": (0, 1), "g0": (1, 2), "cov": (2, 4), "a1g1": (3, 2), "lap": (4, 1), "m1": (5, 2), "m2": (6, 4)}
_PREC = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED, "fp32": _lib.PREC_FP32}


@runtime_checkable
class BoundaryProvider(Protocol):
    """what a scheme needs from a boundary representation (provider.py:38-45)."""
    bodies: list

    def aggregate(self, ps, support, **kwargs): ...

    def signed_distance(self, x, body=None, supportMax=None, want_body=False): ...


@dataclass(frozen=True)
class WallOutput:
    name: str
    group: int
    kind: str


@dataclass(frozen=True)
class FusedGroup:
    """one kernel of the fused evaluation (warpfused.py:31-55): `kernel` (registered name), `channels` (None = all)."""
    kernel: str
    channels: Optional[tuple] = None
    route: Optional[str] = None
    nodes: Optional[int] = None
    panels: Optional[int] = None


class WallAggregate:
    """marker base of the wall aggregates a scheme consumes (fused.py:497-499)."""


class FusedWall(WallAggregate):
    """all twelve channels of every (body, surface) at one position set, per kernel group, world frame, float64:
    lam [B, N], G [B, N, 2], Cov [B, N, 2, 2], m1 [B, N, 2], m2 [B, N, 2, 2]."""

    def __init__(self, scene, ps, support, groups, route="fused", precision="fp64", allowed=None, workspaces=None,
                 outs=None):
        self.scene = scene
        self.groups = tuple(groups)
        self.dev = scene.device
        self.route = route
        self.precision = precision
        self.support = float(support)
        self.workspaces = workspaces           # optional {id(rep): uint8 tensor}: caller-owned workspaces (graphs)
        pos = ps.positions.to(self.dev, F64).contiguous()
        sup = ps.supports.to(self.dev, F64).contiguous()
        self.N = N = len(pos)
        self._pos, self._sup = pos, sup         # the position set cone_area / dir_extreme prepare again
        self._allowed = None if allowed is None else allowed.to(self.dev, torch.int32).contiguous()
        B = len(scene.bodies)
        for g in self.groups:
            if g.kernel not in _GROUP_IDS:
                raise NotImplementedError(f"FusedWall: kernel group {g.kernel!r} is not built")
            if g.kernel in QUAD_KERNEL_IDS and route == "plain":
                raise NotImplementedError(f"FusedWall: the tensile group {g.kernel!r} has no plain route")
        sig = (route, self.support) + tuple(id(r) for b in scene.bodies for r in b.reps)
        if getattr(scene, "_wsb_checked", None) != sig:
            for b in scene.bodies:
                for r in b.fused_reps(self.support, self.dev):
                    if isinstance(r, DiskArrayRep):
                        if route != "fused":
                            raise NotImplementedError("FusedWall: disk sets take the fused route")
                    elif r._triangle is not None and route == "plain":
                        raise NotImplementedError("FusedWall: conditioned single triangles have no plain route")
            scene._wsb_checked = sig
        if any(g.kernel in QUAD_KERNEL_IDS for g in self.groups) and any(
                isinstance(r, DiskArrayRep) for b in scene.bodies for r in b.fused_reps(self.support, self.dev)):
            raise NotImplementedError("FusedWall: the tensile groups have no disk element")
        self.res = []
        self.qstatus = {}                      # (group, body, rep) -> [N] int32 of conditioned triangles
        self.estimates = {}                    # (group, body, rep) -> [N, 12] quadrature estimates
        alloc = torch.empty if route == "fused" else torch.zeros     # the fused route assigns every row of a body
        if outs is not None and (route != "fused" or len(self.groups) != 1):
            raise ValueError("FusedWall: caller-owned outputs serve the fused route with one kernel group")
        for g in self.groups:
            if outs is not None:
                out = outs                                             # caller-owned [B, N, ...] float64 buffers
            else:
                out = {"lam": alloc((B, N), dtype=F64, device=self.dev),
                       "G": alloc((B, N, 2), dtype=F64, device=self.dev),
                       "Cov": alloc((B, N, 2, 2), dtype=F64, device=self.dev),
                       "m1": alloc((B, N, 2), dtype=F64, device=self.dev),
                       "m2": alloc((B, N, 2, 2), dtype=F64, device=self.dev)}
            self.res.append(out)
        kids = [_GROUP_IDS[g.kernel] for g in self.groups]
        if route == "fused":
            self._fused(pos, sup, allowed, kids, self.res)
        elif route == "plain":
            for gi, kid in enumerate(kids):
                self._plain(ps, kid, self.res[gi])
        elif route == "scene":
            self._scene_route(ps, self.res)
        else:
            raise ValueError(f"unknown route {route!r}")
        self.out = {}

    def _fused(self, pos, sup, allowed, kids, outs):
        """every group of every (body, surface) at once: one wsb_aggregate_groups call per surface (the groups share
        the prepared rows and, for the kernel sets the library packs, the pass over the neighbour pairs:
        fused.py:506-547); a conditioned single triangle runs per group, its quadrature rows combined in."""
        N = self.N
        al = None if allowed is None else allowed.to(torch.int32).contiguous()
        names = ("lam", "G", "Cov", "m1", "m2")
        for bi, body in enumerate(self.scene.bodies):
            if not body.reps:
                for out in outs:
                    for t in out.values():
                        t[bi].zero_()
                continue
            pose = body.pose_tensor(self.dev)
            obb = (_lib.ctypes.c_double * 4)(*body.obb())
            for ri, rep in enumerate(body.fused_reps(self.support, self.dev)):
                mode = _lib.OUT_ALL | (_lib.OUT_ASSIGN if ri == 0 else 0)     # the first representation assigns
                if isinstance(rep, DiskArrayRep):
                    nd = rep.native(self.support, self.dev)
                    dws, dneed = nd.workspace(N)
                    for gi, kid in enumerate(kids):
                        o = outs[gi]
                        check(lib.wsb_disk_aggregate(nd.handle, kid, ptr(pos), ptr(sup), ptr(al), N, ptr(pose), mode,
                                                     ptr(o["lam"][bi]), ptr(o["G"][bi]), ptr(o["Cov"][bi]),
                                                     ptr(o["m1"][bi]), ptr(o["m2"][bi]), ptr(dws), dneed, _stream()),
                              "wsb_disk_aggregate")
                    continue
                ns = rep.native(self.support, self.dev)
                if self.workspaces is not None:
                    ws = self.workspaces[id(rep)]
                    need = ws.numel()
                else:
                    ws, need = ns.workspace(N)
                if rep._triangle is None:
                    tgt = {k: _lib.ptrs([out[k][bi] for out in outs]) for k in names}
                    check(lib.wsb_aggregate_groups(ns.handle, len(kids), _lib.int32s(kids), _PREC[self.precision],
                                                   ptr(pos), ptr(sup), ptr(al), N, ptr(pose), obb,
                                                   int(body.unbounded()), mode, tgt["lam"], tgt["G"], tgt["Cov"],
                                                   tgt["m1"], tgt["m2"], ptr(ws), need, _stream()),
                          "wsb_aggregate_groups")
                    continue
                for gi, kid in enumerate(kids):
                    # closed form into scratch, then the rows the quadrature takes are overridden while combining
                    self._group = gi
                    tgt = {k: torch.empty_like(outs[gi][k][bi]) for k in names}
                    check(lib.wsb_aggregate(ns.handle, kid, _PREC[self.precision], ptr(pos), ptr(sup), ptr(al), N,
                                            ptr(pose), obb, int(body.unbounded()), _lib.OUT_ALL | _lib.OUT_ASSIGN,
                                            ptr(tgt["lam"]), ptr(tgt["G"]), ptr(tgt["Cov"]), ptr(tgt["m1"]),
                                            ptr(tgt["m2"]), ptr(ws), need, None, _stream()), "wsb_aggregate")
                    self._conditioned(body, bi, ri, rep, pos, sup, al, kid, pose, tgt, outs[gi])

    def _conditioned(self, body, bi, ri, rep, pos, sup, al, kid, pose, closed, out, tolerance=2e-12,
                     max_panels=4096):
        """the conditioned area quadrature of a single-triangle rep on its small / sliver rows, combined with the
        closed form of the other rows (warptriangle.py:126-201, fused.py:556-564)."""
        N = self.N
        tri, area2, sign = rep._triangle
        state = torch.tensor([body.state_row()], dtype=F64, device=self.dev)
        local = torch.empty((N, 2), dtype=F64, device=self.dev)
        check(lib.wsb_kinematics(ptr(state), 1, ptr(pos), N, None, ptr(local), None, None, _stream()),
              "wsb_kinematics")
        vals = torch.empty((N, 12), dtype=F64, device=self.dev)
        est = torch.empty((N, 12), dtype=F64, device=self.dev)
        st = torch.empty(N, dtype=torch.int32, device=self.dev)
        check(lib.wsb_triangle_channels(_lib.dptr(tri), area2, sign, rep.background, kid, ptr(local), ptr(sup),
                                        ptr(al), N, tolerance, max_panels, ptr(vals), ptr(est), ptr(st), _stream()),
              "wsb_triangle_channels")
        check(lib.wsb_triangle_combine(ptr(vals), ptr(st), ptr(sup), ptr(pose), N, int(ri > 0), ptr(closed["lam"]),
                                       ptr(closed["G"]), ptr(closed["Cov"]), ptr(closed["m1"]), ptr(closed["m2"]),
                                       ptr(out["lam"][bi]), ptr(out["G"][bi]), ptr(out["Cov"][bi]),
                                       ptr(out["m1"][bi]), ptr(out["m2"][bi]), _stream()), "wsb_triangle_combine")
        key = (self._group, bi, ri)
        self.qstatus[key] = st
        self.estimates[key] = est

    def _scene_route(self, ps, outs):
        """the Scene route (provider.py:89-92 with fixedAdjacency=False): one `Scene.adjacency` (candidates and the
        pair list of every surface), then per group `Scene.precompute` (per-pair channels, per-query sums, indicator,
        conditioned triangles) and the world-frame moments added into the [B, N] outputs of the candidate rows."""
        props = OperationProperties(operationMode=OperationDirection.BoundaryToFluid)
        adj = self.scene.adjacency(ps, props)
        for g, out in zip(self.groups, outs):
            pm = self.scene.precompute(adj, OperationProperties(kernel=g.kernel), precision=self.precision)
            for bi, ent in enumerate(pm.entries):
                for m in ent["surface"] + ent["implicit"]:
                    q = m.q.long()
                    out["lam"][bi].index_add_(0, q, m.lam)
                    out["G"][bi].index_add_(0, q, m.g0)
                    out["Cov"][bi].index_add_(0, q, m.g1)
                    out["m1"][bi].index_add_(0, q, m.m1)
                    out["m2"][bi].index_add_(0, q, m.m2)

    def _plain(self, ps, kid, out):
        props = OperationProperties(operationMode=OperationDirection.BoundaryToFluid)
        adj = fixed_adjacency(self.scene, ps, props, self.support)
        for bi, ba in enumerate(adj.bodies):
            R = ba.body.pose.Rflat().contiguous()
            lp, ls = ba.lpos.contiguous(), ba.lsup.contiguous()
            for rep, topo in zip(ba.repList, ba.reps):
                ns = rep.native(self.support, self.dev)
                c = torch.empty(self.N * topo.K * 12, dtype=F64, device=self.dev)
                check(lib.wsb_slot_channels_plain(ns.handle, kid, ptr(lp), ptr(ls), ptr(topo.e), self.N, ptr(c),
                                                  _stream()), "wsb_slot_channels_plain")
                check(lib.wsb_contract(ns.handle, kid, ptr(topo.e), ptr(c), ptr(topo.ind), ptr(ls), self.N, ptr(R),
                                       ptr(out["lam"][bi]), ptr(out["G"][bi]), ptr(out["Cov"][bi]), ptr(out["m1"][bi]),
                                       ptr(out["m2"][bi]), _stream()), "wsb_contract")

    @staticmethod
    def supported(scene, lowering=True):
        return all(b.fusable() for b in scene.bodies) if lowering else \
            all(isinstance(r, SurfaceRep) for b in scene.bodies for r in b.reps)

    def evaluate(self, outputs, a1=None):
        """{name: tensor [B, N, ...]} float64, world frame (fused.py:612-659).  `a1` [B, N, 2]: world vectors of the
        'a1g1' outputs (sum_d a1_d g1_dj)."""
        res = {}
        for o in outputs:
            if o.kind not in KINDS:
                raise ValueError(f"unknown output kind {o.kind!r}")
            r = self.res[o.group]
            if self.groups[o.group].kernel in QUAD_KERNEL_IDS and o.kind != "g0":
                raise ValueError(f"FusedWall.evaluate: the tensile group {self.groups[o.group].kernel!r} serves 'g0' "
                                 f"only")
            if o.kind == "lam":
                res[o.name] = r["lam"]
            elif o.kind == "g0":
                res[o.name] = r["G"]
            elif o.kind == "cov":
                res[o.name] = r["Cov"]
            elif o.kind == "m1":
                res[o.name] = r["m1"]
            elif o.kind == "m2":
                res[o.name] = r["m2"]
            elif o.kind == "a1g1":
                if a1 is None:
                    raise ValueError("FusedWall.evaluate: a1 [B, N, 2] is required for 'a1g1' outputs")
                res[o.name] = torch.einsum("bnd,bndj->bnj", a1.to(self.dev, F64), r["Cov"])
            elif o.kind == "lap":
                # the wall Laplacian of the registered W'/r kernel (lw2 / lw4): 2 lam - tr g1, the indicator cancels
                # (fused.py:11); the trace is the same in the body and the world frame
                if self.groups[o.group].kernel not in ("lw2", "lw4"):
                    raise ValueError("FusedWall.evaluate: 'lap' outputs come from an lw2 / lw4 group")
                res[o.name] = 2.0 * r["lam"] - (r["Cov"][..., 0, 0] + r["Cov"][..., 1, 1])
            else:
                raise ValueError(f"FusedWall.evaluate: unknown output kind {o.kind!r}")
        return res

    def _tensors(self):
        out = []
        for k, r in enumerate(self.res):
            for name in sorted(r):
                out.append((name, k, r[name]))
        return out

    def copy_from(self, other):
        """overwrite this aggregate's buffers in place with `other`'s (same scene, groups and N), so kernels and CUDA
        graphs that read these buffers see the new position set (fused.py:707-719)."""
        a, b = self._tensors(), other._tensors()
        if [(n, k, t.shape) for n, k, t in a] != [(n, k, t.shape) for n, k, t in b]:
            raise ValueError("FusedWall.copy_from: different structure")
        for (_, _, ta), (_, _, tb) in zip(a, b):
            ta.copy_(tb)
        for name in self.out:
            if name in other.out:
                self.out[name].copy_(other.out[name])

    def reset_derived(self):
        """no lazily derived buffers exist in this implementation (fused.py:721-725)."""

    def _surfaces(self):
        """(body index, native surface or disk set, workspace, bytes, pose) of every (body, representation); a
        surface's workspace is prepared for this position set (wsb_aggregate_prepare: body frame, broadphase,
        neighbour masks, indicator), a disk set needs none (None, 0)."""
        N = self.N
        for bi, body in enumerate(self.scene.bodies):
            if not body.reps:
                continue
            pose = body.pose_tensor(self.dev)
            obb = (_lib.ctypes.c_double * 4)(*body.obb())
            for rep in body.fused_reps(self.support, self.dev):
                if isinstance(rep, DiskArrayRep):
                    yield bi, rep.native(self.support, self.dev), None, 0, pose
                    continue
                ns = rep.native(self.support, self.dev)
                if self.workspaces is not None:
                    ws = self.workspaces[id(rep)]
                    need = ws.numel()
                else:
                    ws, need = ns.workspace(N)
                check(lib.wsb_aggregate_prepare(ns.handle, ptr(self._pos), ptr(self._sup), ptr(self._allowed), N,
                                                ptr(pose), obb, int(body.unbounded()), ptr(ws), need, _stream()),
                      "wsb_aggregate_prepare")
                yield bi, ns, ws, need, pose

    def cone_area(self, axes, half_angle):
        """[2, N] float64 (fused.py:788-835): row 0 the area of solid cap disk(x, H) cap wedge(x, axis, half_angle)
        (units length^2; half_angle >= pi is the full disk), row 1 the full-disk area of the solid, summed over the
        bodies; H is each query's support and `axes` [N, 2] are world vectors (only the direction matters).  A query
        outside the broadphase of a surface whose solid is the outside lies deep in it: the whole sector.  One
        wsb_aggregate_prepare + wsb_cone_area per (body, surface), float64 whatever the precision of the groups."""
        ha = float(half_angle)
        if not math.isfinite(ha) or ha < 0.0:
            raise ValueError("FusedWall.cone_area: the half angle must be finite and >= 0")
        N = self.N
        ax = axes.to(self.dev, F64).contiguous()
        if tuple(ax.shape) != (N, 2):
            raise ValueError(f"FusedWall.cone_area: axes of shape {tuple(ax.shape)}, expected ({N}, 2)")
        out = torch.zeros(2 * N, dtype=F64, device=self.dev)
        for _, ns, ws, need, pose in self._surfaces():
            if ws is None:
                check(lib.wsb_disk_cone_area(ns.handle, ptr(self._pos), ptr(self._sup), ptr(self._allowed), N,
                                             ptr(pose), ptr(ax), ha, ptr(out), _stream()), "wsb_disk_cone_area")
                continue
            check(lib.wsb_cone_area(ns.handle, ptr(self._sup), N, ptr(pose), ptr(ax), ha, ptr(out), ptr(ws), need,
                                    _stream()), "wsb_cone_area")
        return out.reshape(2, N)

    def dir_extreme(self, vecs):
        """[B, N] float64 (fused.py:741-786): for the world vectors `vecs` [B, N, 2] (one per body and query) the
        largest |cos| between the vector and a direction from the query to a solid point of that body within one
        support -- 1 where the line of the vector meets the solid there, 0 for a zero vector or no solid in support;
        the maximum over the body's surfaces.  One wsb_aggregate_prepare + wsb_dir_extreme per (body, surface)."""
        N, B = self.N, len(self.scene.bodies)
        v = vecs.to(self.dev, F64).contiguous()
        if tuple(v.shape) != (B, N, 2):
            raise ValueError(f"FusedWall.dir_extreme: vecs of shape {tuple(v.shape)}, expected ({B}, {N}, 2)")
        out = torch.zeros((B, N), dtype=F64, device=self.dev)
        for bi, ns, ws, need, pose in self._surfaces():
            if ws is None:
                check(lib.wsb_disk_dir_extreme(ns.handle, ptr(self._pos), ptr(self._sup), ptr(self._allowed), N,
                                               ptr(pose), ptr(v[bi]), ptr(out[bi]), _stream()), "wsb_disk_dir_extreme")
                continue
            check(lib.wsb_dir_extreme(ns.handle, N, ptr(pose), ptr(v[bi]), ptr(out[bi]), ptr(ws), need, _stream()),
                  "wsb_dir_extreme")
        return out


_FAMILY = {"Wendland2": "w2", "Wendland4": "w4"}


class AnalyticBoundary:
    """the analytic bodies of a `Scene` as a boundary provider (provider.py:48-113)."""

    def __init__(self, scene: Scene, route: str = "fused", precision: str = "fp64"):
        if precision not in _PREC:
            raise ValueError(f"precision must be one of {sorted(_PREC)}")
        self.scene = scene
        self.route = route
        self.precision = precision
        self._layouts = {}

    @property
    def bodies(self):
        return self.scene.bodies

    def family(self, kernel):
        fam = _FAMILY.get(getattr(kernel, "name", None))
        if fam is None:
            raise NotImplementedError("exact wall operations: Wendland C2 and C4 only")
        return fam

    def supported(self, fixedAdjacency=True):
        return FusedWall.supported(self.scene, fixedAdjacency)

    def properties(self, kernel, operation=WarpOperation.Density):
        return OperationProperties(kernel=kernel, operation=operation, gradientMode=GradientScheme.Naive,
                                   operationMode=OperationDirection.BoundaryToFluid)

    def layout(self, kernel, laplacian, fixedAdjacency=True):
        """(groups, roles) of the delta+ layout (provider.py:73-87): the scheme kernel ('w'), the cover vector's cone
        kernel ('cone', G only), the wall Laplacian's W'/r kernel ('lap', when `laplacian`) and the tensile W^5 kernel
        ('tens', G only); built once per configuration."""
        key = (kernel, bool(laplacian), bool(fixedAdjacency))
        if key not in self._layouts:
            fam = self.family(kernel)
            groups, idx = [FusedGroup(kernelName(kernel)), FusedGroup("cone", (3, 4))], {"w": 0, "cone": 1}
            if laplacian:
                idx["lap"] = len(groups)
                groups.append(FusedGroup("l" + fam))
            idx["tens"] = len(groups)
            groups.append(FusedGroup(fam + "p5", (3, 4)))
            self._layouts[key] = (tuple(groups), idx)
        return self._layouts[key]

    def aggregate(self, ps, support, kernel=KernelFunctions.Wendland2, laplacian=False, fixedAdjacency=True,
                  lean=False):
        """the wall evaluation at the positions of `ps` (provider.py:89-110): `.out` holds lam, G, Cov per body;
        `evaluate` serves m1, m2 and a1g1 as well; without `lean` the delta+ layout adds cover, lap (when `laplacian`)
        and tens, raw (the scheme applies its factors).  `support`: host float >= every support of `ps`.
        `fixedAdjacency=False` takes the Scene route (Scene.adjacency + Scene.precompute: pair lists, per-pair
        channels, per-query sums) instead of the fused pass; the same values within rounding."""
        if lean:
            groups, idx = (FusedGroup(kernelName(kernel)),), {"w": 0}
        else:
            groups, idx = self.layout(kernel, laplacian, fixedAdjacency)
        allowed = None
        if getattr(ps, "kinds", None) is not None:      # without kinds every query is served: no mask, no host read
            allowed = queryAllowed(ps, self.properties(kernel).operationMode, self.scene.device)
        route = self.route if fixedAdjacency else "scene"          # Scene.adjacency + precompute (the oracle path)
        fw = FusedWall(self.scene, ps, support, groups, route=route, precision=self.precision, allowed=allowed)
        outs = [WallOutput("lam", 0, "lam"), WallOutput("G", 0, "g0"), WallOutput("Cov", 0, "cov")]
        if not lean:
            outs.append(WallOutput("cover", idx["cone"], "g0"))
            if "lap" in idx:
                outs.append(WallOutput("lap", idx["lap"], "lap"))
            outs.append(WallOutput("tens", idx["tens"], "g0"))
        fw.out = fw.evaluate(outs)
        return fw

    def signed_distance(self, x, body=None, supportMax=None, want_body=False):
        return self.scene.signed_distance(x, body=body, supportMax=supportMax, want_body=want_body)
