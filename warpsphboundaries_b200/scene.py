"""Scene layer (2-D): rigid bodies with a pose, closed polygonal surfaces, kinematics and signed distance.

The types and method names follow the reference's scene layer
(src/warpSPHBoundaries/scene/scene.py): `Pose` (:64-97), `SurfaceRep` (:213-428),
`Body` (:905-1067), `BodyKinematics` (:1155-1225), `Scene` (:1228-1372).  Every
per-particle computation runs in libwsb.so on the GPU; this module holds the
geometry, caches the device-resident static structures of each surface per
(support, device) and marshals tensors.
"""
import ctypes
from dataclasses import dataclass, field
from fractions import Fraction
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr

F64 = torch.float64


# ----------------------------------------------------------------------------------------------------------- frames
@dataclass
class Pose:
    center: torch.Tensor
    angle: float = 0.0

    def _cs(self):
        a = float(self.angle)
        return float(np.cos(a)), float(np.sin(a))

    @property
    def R(self):
        c, s = self._cs()
        return torch.tensor([[c, -s], [s, c]], dtype=F64, device=self.center.device)

    def Rflat(self):
        return self.R.reshape(-1)

    def toLocal(self, p):
        """(p - center) R with the rotation written out (scene.py:75-79)."""
        c, s = self._cs()
        d = p - self.center
        return torch.stack([d[:, 0] * c + d[:, 1] * s, d[:, 1] * c - d[:, 0] * s], 1)

    def toWorld(self, p):
        c, s = self._cs()
        return torch.stack([p[:, 0] * c - p[:, 1] * s + self.center[0], p[:, 0] * s + p[:, 1] * c + self.center[1]], 1)

    def vecToWorld(self, v):
        c, s = self._cs()
        return torch.stack([v[:, 0] * c - v[:, 1] * s, v[:, 0] * s + v[:, 1] * c], 1)


# ----------------------------------------------------------------------------------------------------------- native surface
class NativeSurface:
    """the device-resident static structures of one closed surface for supports <= support_max (wsb_surface)."""

    def __init__(self, vertices, edges, background, support_max, device):
        v = np.ascontiguousarray(vertices.detach().cpu().numpy(), dtype=np.float64).reshape(-1)
        e = np.ascontiguousarray(edges.detach().cpu().numpy(), dtype=np.int32).reshape(-1)
        self.device = torch.device(device)
        idx = self.device.index if self.device.index is not None else torch.cuda.current_device()
        h = ctypes.c_void_p()
        check(lib.wsb_surface_create(v.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(v) // 2,
                                     e.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(e) // 2, int(background),
                                     float(support_max), idx, ctypes.byref(h)), "wsb_surface_create")
        self.handle = h
        info = _lib.SurfaceInfo()
        check(lib.wsb_surface_info_get(h, ctypes.byref(info)), "wsb_surface_info_get")
        self.info = info
        self.K = int(info.K)
        self.support_max = float(support_max)
        self._ws = {}

    def workspace(self, n):
        """the workspace for n rows on the current stream: one buffer per stream, grown geometrically and reused for
        any smaller row count (the library carves it per call and allocates nothing itself)."""
        # with the staging region: the evaluations store every row's outputs in one coalesced pass
        need = int(lib.wsb_aggregate_workspace_size(self.handle, int(n)) +
                   lib.wsb_aggregate_staging_size(self.handle, int(n)))
        key = torch.cuda.current_stream(self.device).cuda_stream
        ws = self._ws.get(key)
        if ws is None or ws.numel() < need:
            ws = torch.empty(max(need, int(1.5 * ws.numel()) if ws is not None else need, 1), dtype=torch.uint8,
                             device=self.device)
            self._ws[key] = ws
        return ws, need

    def cells(self):
        """(start [nx*ny+1], items [n_items]) host copies of the edge cell list."""
        start = np.zeros(self.info.nx * self.info.ny + 1, dtype=np.int32)
        items = np.zeros(max(int(self.info.n_items), 1), dtype=np.int32)
        check(lib.wsb_surface_cells(self.handle, start.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                    items.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))), "wsb_surface_cells")
        return start, items[: int(self.info.n_items)]

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and lib is not None:
            lib.wsb_surface_destroy(h)
            self.handle = None


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


# ----------------------------------------------------------------------------------------------------------- representations
class SurfaceRep:
    """closed polylines in the body frame, counter-clockwise around the SOLID (solid on the left of every edge);
    `background = 1` when the solid is the unbounded outside (scene.py:213-233)."""
    kind = "surface"

    def __init__(self, vertices, edges, background: int = 0, conditioned: bool = True):
        self.vertices = torch.as_tensor(vertices, dtype=F64)
        self.edges = torch.as_tensor(edges, dtype=torch.int32)
        self.background = int(background)
        # a single triangle takes the conditioned area quadrature on its small / sliver rows (warptriangle.py:126-201)
        self._triangle = self._triangle_meta() if conditioned else None
        self._native = {}

    def _triangle_meta(self):
        """(ordered vertices [6], 2 area, sign) of a single-triangle loop, or None (warptriangle.py:290-310): the
        vertices in the loop's order, the exact signed area, the rule's order with the shortest edge last."""
        if len(self.vertices) != 3 or len(self.edges) != 3:
            return None
        v = self.vertices.detach().cpu().numpy()
        e = {tuple(int(x) for x in pair) for pair in self.edges.detach().cpu().tolist()}
        if e == {(0, 1), (1, 2), (2, 0)}:
            loop = [0, 1, 2]
        elif e == {(0, 2), (2, 1), (1, 0)}:
            loop = [0, 2, 1]
        else:
            return None
        a, b, c = [[Fraction(float(x)) for x in v[i]] for i in loop]
        signed = (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0])
        if not signed:
            return None
        short = int(np.argmin([float(((v[(i + 1) % 3] - v[i]) ** 2).sum()) for i in range(3)]))
        order = [short, (short + 2) % 3, (short + 1) % 3]
        return (np.ascontiguousarray(v[order].reshape(-1), dtype=np.float64), float(abs(signed)),
                1.0 if signed > 0 else -1.0)

    @staticmethod
    def _orient(P, solid):
        local = P.astype(np.longdouble) - P[0].astype(np.longdouble)
        terms = local[:, 0] * np.roll(local[:, 1], -1) - np.roll(local[:, 0], -1) * local[:, 1]
        a = np.sum(terms)
        if len(P) == 3 or abs(a) <= 64 * np.finfo(np.longdouble).eps * np.sum(abs(terms)):
            v = [[Fraction(float(c)) for c in p] for p in P]
            a = sum((v[i][0] - v[0][0]) * (v[(i + 1) % len(v)][1] - v[0][1]) -
                    (v[(i + 1) % len(v)][0] - v[0][0]) * (v[i][1] - v[0][1]) for i in range(len(v)))
        if (a > 0) != (solid == "inside"):
            P = P[::-1].copy()
        return P

    @staticmethod
    def polygon(points, solid: str = "inside", conditioned: bool = True):
        """one closed loop through `points` [n, 2]; 'inside': the polygon is the solid (made counter-clockwise),
        'outside': a hole in an infinite solid (clockwise, background 1) (scene.py:235-256)."""
        P = SurfaceRep._orient(np.asarray(points, dtype=float), solid)
        n = len(P)
        E = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1)
        return SurfaceRep(np.ascontiguousarray(P), E, background=0 if solid == "inside" else 1, conditioned=conditioned)

    @staticmethod
    def loops(loops, solid: str = "inside"):
        """several closed loops in one representation (solids that overlap add through the winding number)."""
        V, E, off = [], [], 0
        for pts in loops:
            P = SurfaceRep._orient(np.asarray(pts, dtype=float), solid)
            n = len(P)
            V.append(P)
            E.append(np.stack([off + np.arange(n), off + (np.arange(n) + 1) % n], 1))
            off += n
        return SurfaceRep(np.concatenate(V), np.concatenate(E), background=0 if solid == "inside" else 1,
                          conditioned=False)

    @staticmethod
    def box(lo, hi, solid: str = "inside"):
        (x0, y0), (x1, y1) = lo, hi
        return SurfaceRep.polygon([(x0, y0), (x1, y0), (x1, y1), (x0, y1)], solid)

    @staticmethod
    def regularPolygon(center, radius, n, solid="inside", areaPreserving=True):
        r = radius * np.sqrt(2 * np.pi / (n * np.sin(2 * np.pi / n))) if areaPreserving else radius
        t = 2 * np.pi * np.arange(n) / n
        return SurfaceRep.polygon(np.stack([center[0] + r * np.cos(t), center[1] + r * np.sin(t)], 1), solid)

    def to(self, device):
        self.vertices = self.vertices.to(device)
        self.edges = self.edges.to(device)
        return self

    def bounds(self):
        return self.vertices.amin(0), self.vertices.amax(0)

    def native(self, supportMax, device) -> NativeSurface:
        """the static device structures for supports <= supportMax on `device` (built once, cached)."""
        dev = torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("SurfaceRep: the boundary integrals run on CUDA devices only (no CPU fallback)")
        key = (float(supportMax), str(dev))
        ns = self._native.get(key)
        if ns is None:
            ns = NativeSurface(self.vertices, self.edges, self.background, float(supportMax), dev)
            self._native[key] = ns
        return ns

    def _default_native(self, device):
        if self._native:
            for (sm, d), ns in self._native.items():
                if d == str(torch.device(device)):
                    return ns
        lo, hi = self.bounds()
        ext = float((hi - lo).max())
        return self.native(max(ext / 64.0, 1e-9), device)

    def indicator(self, p, supports=None):
        """winding number of the loops around each point (+ background); on the boundary the angle fraction
        (scene.py:350-396), evaluated on the device."""
        ns = self._default_native(p.device)
        p = p.to(F64).contiguous()
        n = len(p)
        sup = (supports.to(F64) if supports is not None else torch.ones(n, dtype=F64, device=p.device)).contiguous()
        slots = torch.empty(n * ns.K, dtype=torch.int32, device=p.device)
        ind = torch.empty(n, dtype=F64, device=p.device)
        check(lib.wsb_fixed_topology(ns.handle, ptr(p), ptr(sup), None, n, ptr(slots), ptr(ind), _stream()),
              "wsb_fixed_topology")
        return ind

    def topology(self, lpos, lsup):
        """(query row, edge) pairs with segment distance < support (scene.py:374-382): a compacted fixed topology."""
        from .fixedadj import fixed_topology
        if len(lpos) == 0:
            return None
        supmax = float(lsup.max())
        ft = fixed_topology(self, lpos, lsup, torch.ones(len(lpos), dtype=torch.bool, device=lpos.device), supmax)
        keep = ft.e >= 0
        return SurfaceTopology(ft.qi[keep], ft.e[keep], supmax, ft.ind)

    def moments(self, topo, lpos, lsup, qglobal, kernel, device, channels=None, precision="fp64"):
        """complete polygon moments of the queries lpos [C, 2] (body frame, supports lsup [C]) from the pair list
        `topo` (scene.py:384-416): the twelve channels of every pair on the device (wsb_pair_channels), summed per
        query, plus the indicator times the whole-plane constants; a conditioned single triangle overrides the rows its
        area quadrature takes; physical units.  Channels 0..8 are the legacy nine, 9..11 m20, m11, m02; None asks for
        all twelve and an explicit subset zeroes the others.  A tensile kernel (w2p5 / w4p5) defines g0 only.  Returns
        `RepMoments` in the body frame, q = `qglobal`."""
        from .kernels import KERNEL_IDS, QUAD_KERNEL_IDS, plane_channels
        from .shim import kernelName
        name = kernel if isinstance(kernel, str) and kernel in QUAD_KERNEL_IDS else kernelName(kernel)
        requested = set(range(12)) if channels is None else {int(k) for k in channels}
        if not requested <= set(range(12)):
            raise ValueError("Surface moment channels must be in 0..11")
        quad = name in QUAD_KERNEL_IDS
        if name not in KERNEL_IDS and not quad:
            raise NotImplementedError(f"SurfaceRep.moments: kernel {name!r} is not built")
        if precision == "fp32":
            raise NotImplementedError("SurfaceRep.moments: the float route runs on the fused pass (FusedWall)")
        if precision not in ("fp64", "mixed"):
            raise ValueError("precision must be 'fp64', 'mixed' or 'fp32'")
        if quad and self._triangle is not None:
            raise NotImplementedError("SurfaceRep.moments: the tensile kernels have no conditioned-triangle route")
        dev = torch.device(device)
        lp = lpos.to(dev, F64).contiguous()
        ls = lsup.to(dev, F64).contiguous()
        C = len(lp)
        kid = QUAD_KERNEL_IDS[name] if quad else KERNEL_IDS[name]
        out = torch.zeros((C, 12), dtype=F64, device=dev)
        if topo is not None and len(topo.qi):
            ns = self.native(topo.supMax, dev)
            P = len(topo.qi)
            qi = topo.qi.to(dev, torch.int32).contiguous()
            e = topo.e.to(dev, torch.int32).contiguous()
            c = torch.empty((P, 12), dtype=F64, device=dev)
            st = torch.zeros(1, dtype=torch.int32, device=dev)
            check(lib.wsb_pair_channels(ns.handle, kid, _lib.PREC_MIXED if precision == "mixed" else _lib.PREC_FP64,
                                        ptr(qi), ptr(e), P, ptr(lp), ptr(ls), C, ptr(c), ptr(st), _stream()),
                  "wsb_pair_channels")
            # per-query sums in pair order (deterministic, unlike an atomic index_add): the pairs of a query are
            # contiguous (rows ascending), laid out [query, rank, 12] and reduced over the rank
            q = qi.long()
            cnt = torch.bincount(q, minlength=C)
            start = torch.cumsum(cnt, 0) - cnt
            rank = torch.arange(P, device=dev) - start[q]
            pad = torch.zeros((C, int(cnt.max()), 12), dtype=F64, device=dev)
            pad[q, rank] = c
            out = pad.sum(1)
        estimate = torch.zeros((C, 12), dtype=F64, device=dev)
        status = torch.zeros(C, dtype=torch.int32, device=dev)
        if quad:
            keep = torch.zeros(12, dtype=torch.bool, device=dev)
            keep[3:5] = True
            out = torch.where(keep, out, torch.full_like(out, float("nan")))
        else:
            ind = topo.indicator(self, lp, ls) if topo is not None else self.indicator(lp, ls)
            out += ind[:, None] * torch.tensor(plane_channels(name), dtype=F64, device=dev)
            if self._triangle is not None and C:
                tri, area2, sign = self._triangle
                vals = torch.empty((C, 12), dtype=F64, device=dev)
                check(lib.wsb_triangle_channels(_lib.dptr(tri), area2, sign, self.background, kid, ptr(lp), ptr(ls),
                                                None, C, 2e-12, 4096, ptr(vals), ptr(estimate), ptr(status), _stream()),
                      "wsb_triangle_channels")
                out = torch.where((status != 0)[:, None], vals, out)
        mask = torch.tensor([float(k in requested) for k in range(12)], dtype=F64, device=dev)
        one = torch.ones_like(ls)
        physical = torch.stack([one, ls, ls, 1 / ls, 1 / ls, one, one, one, one, ls * ls, ls * ls, ls * ls], 1)
        out = out * mask * physical
        estimate = estimate * mask * physical
        m2 = (torch.stack([out[:, 9], out[:, 10], out[:, 10], out[:, 11]], 1).reshape(-1, 2, 2)
              if requested & {9, 10, 11} else None)
        return RepMoments(qglobal, out[:, 0], out[:, 3:5], out[:, 1:3], out[:, 5:9].reshape(-1, 2, 2), m2, estimate,
                          status)

    def pairs(self, lpos, lsup, qglobal, kernel, device, channels=None, precision="fp64"):
        """topology + moments in one call (scene.py:418-422; the fallback surfaces of implicit representations)."""
        return self.moments(self.topology(lpos, lsup), lpos, lsup, qglobal, kernel, device, channels, precision)



class BoxRep(SurfaceRep):
    """an axis-aligned rectangle [lo, hi] in the body frame (scene.py:459-510): the solid (`solid='inside'`: an
    obstacle, a baffle, a floor slab) or the fluid domain (`solid='outside'`: a tank, a channel).  The reference
    evaluates a box from Chebyshev corner tables (scene/box.py; table error up to 1e-7 on the gradient channels of w2
    and 1e-6 for lw2) and its exact polygon for the kinked kernels; here every kernel runs the exact closed form of
    that polygon -- four edges, at most four neighbour pairs a row -- so a box is the SurfaceRep of its outline (a
    tank: the clockwise outline with background 1), and `surface()` is the box itself."""
    kind = "box"

    def __init__(self, lo, hi, solid: str = "inside"):
        if solid not in ("inside", "outside"):
            raise ValueError("solid must be 'inside' or 'outside'")
        lo_h = tuple(float(v) for v in torch.as_tensor(lo, dtype=F64).reshape(2))
        hi_h = tuple(float(v) for v in torch.as_tensor(hi, dtype=F64).reshape(2))
        if not (hi_h[0] > lo_h[0] and hi_h[1] > lo_h[1]):
            raise ValueError(f"BoxRep: hi {hi_h} must exceed lo {lo_h} in both coordinates")
        (x0, y0), (x1, y1) = lo_h, hi_h
        P = SurfaceRep._orient(np.array([(x0, y0), (x1, y0), (x1, y1), (x0, y1)], dtype=float), solid)
        super().__init__(np.ascontiguousarray(P), np.array([[0, 1], [1, 2], [2, 3], [3, 0]]),
                         background=0 if solid == "inside" else 1, conditioned=False)
        self.solid = solid
        self.lo_h, self.hi_h = lo_h, hi_h      # host copies: reading a device tensor would synchronise
        self.lo = torch.tensor(lo_h, dtype=F64)
        self.hi = torch.tensor(hi_h, dtype=F64)

    def to(self, device):
        super().to(device)
        self.lo, self.hi = self.lo.to(device), self.hi.to(device)
        return self

    def surface(self):
        return self

    def signed(self, lpos):
        """(d, n) of body-frame points (scene.py:490-506): the signed distance, positive in the fluid, and the unit
        normal from the wall into the fluid -- from the closest point of the box outside it, else the normal of the
        nearest face plane."""
        lo, hi = self.lo.to(lpos.device), self.hi.to(lpos.device)
        c, hw = 0.5 * (lo + hi), 0.5 * (hi - lo)
        r = lpos - c
        q = r.abs() - hw
        sd = q.clamp(min=0).norm(dim=1) + q.max(dim=1).values.clamp(max=0)
        ax = (q[:, 1] > q[:, 0]).long()
        sgn = torch.where(r.gather(1, ax[:, None])[:, 0] >= 0, 1.0, -1.0).to(F64)
        face = torch.zeros_like(lpos).scatter_(1, ax[:, None], sgn[:, None])
        dirv = lpos - torch.minimum(torch.maximum(lpos, lo), hi)
        dn = dirv.norm(dim=1, keepdim=True)
        outward = torch.where(dn > 1e-12, dirv / dn.clamp(min=1e-300), face)
        if self.solid == "inside":
            return sd, outward
        return -sd, -face


class NativeDisks:
    """the device-resident cell grid of a disk set for supports <= support_max (wsb_disks)."""

    def __init__(self, centres, radii, support_max, device):
        c = np.ascontiguousarray(centres.detach().cpu().numpy(), dtype=np.float64).reshape(-1)
        r = np.ascontiguousarray(radii.detach().cpu().numpy(), dtype=np.float64).reshape(-1)
        self.device = torch.device(device)
        idx = self.device.index if self.device.index is not None else torch.cuda.current_device()
        h = ctypes.c_void_p()
        check(lib.wsb_disks_create(c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                   r.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(r), float(support_max), idx,
                                   ctypes.byref(h)), "wsb_disks_create")
        self.handle = h
        self._ws = {}

    def workspace(self, n):
        """the work-list buffer for n rows on the current stream (one per stream, grown geometrically)."""
        need = int(lib.wsb_disk_workspace_size(self.handle, int(n)))
        key = torch.cuda.current_stream(self.device).cuda_stream
        ws = self._ws.get(key)
        if ws is None or ws.numel() < need:
            ws = torch.empty(max(need, int(1.5 * ws.numel()) if ws is not None else need, 1), dtype=torch.uint8,
                             device=self.device)
            self._ws[key] = ws
        return ws, need

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and lib is not None:
            lib.wsb_disks_destroy(h)
            self.handle = None


class DiskArrayRep:
    """solid disks in the body frame, centres [M, 2] and radii [M] (scene.py:808-905): a fibre bundle moving as one
    body; the disks must not overlap (their integrals add).  Every (particle, disk) pair within reach is integrated
    exactly by the disk element (wsb_disk_aggregate) -- no polygon, any radius."""
    kind = "disks"

    def __init__(self, centres, radii):
        self.centres = torch.as_tensor(centres, dtype=F64).reshape(-1, 2)
        self.radii = torch.as_tensor(radii, dtype=F64).reshape(-1)
        if len(self.centres) != len(self.radii):
            raise ValueError("DiskArrayRep: centres and radii differ in length")
        if len(self.radii) and not bool((self.radii > 0).all()):
            raise ValueError("DiskArrayRep: every radius must be positive")
        self._native = {}

    def to(self, device):
        self.centres, self.radii = self.centres.to(device), self.radii.to(device)
        return self

    def bounds(self):
        c, r = self.centres.cpu(), self.radii.cpu()[:, None]
        return (c - r).amin(0), (c + r).amax(0)

    def native(self, supportMax, device) -> NativeDisks:
        dev = torch.device(device)
        if dev.type != "cuda":
            raise RuntimeError("DiskArrayRep: the boundary integrals run on CUDA devices only (no CPU fallback)")
        key = (float(supportMax), str(dev))
        nd = self._native.get(key)
        if nd is None:
            nd = NativeDisks(self.centres, self.radii, float(supportMax), dev)
            self._native[key] = nd
        return nd

    def signed(self, lpos, chunk=1 << 16):
        """(d, n) of body-frame points: the distance to the nearest circle, negative inside a disk, and the unit
        normal into the fluid (radially outward from that disk's centre)."""
        c, r = self.centres.to(lpos.device), self.radii.to(lpos.device)
        d = torch.empty(len(lpos), dtype=F64, device=lpos.device)
        n = torch.empty((len(lpos), 2), dtype=F64, device=lpos.device)
        for k in range(0, len(lpos), chunk):
            v = lpos[k:k + chunk, None, :] - c[None]
            dist = v.norm(dim=2)
            j = (dist - r[None]).argmin(1)
            rows = torch.arange(len(j), device=lpos.device)
            d[k:k + chunk] = dist[rows, j] - r[j]
            n[k:k + chunk] = v[rows, j] / dist[rows, j].clamp(min=1e-300)[:, None]
        return d, n

class ImplicitRep:
    """an analytic primitive in the body frame (scene.py:558-596).  The fused wall path integrates its exact form: a
    solid disk is a one-disk DiskArrayRep (the disk element), a cavity disk (fluid inside the circle) its
    area-preserving regular polygon with edges <= the policy's bound times the support (at least 24 edges), integrated
    exactly like any surface.  A half plane has no such form: NotImplementedError on the fused path."""
    kind = "implicit"

    def __init__(self, shape, policy=None):
        from .implicit import TierPolicy
        self.shape = shape
        self.policy = policy or TierPolicy()
        self._fallback = {}

    def to(self, device):
        for s in self._fallback.values():
            s.to(device)
        return self

    def bounds(self):
        from .implicit import DiskBody
        s = self.shape
        if isinstance(s, DiskBody):
            c = torch.as_tensor(s.center, dtype=F64)
            return c - s.radius, c + s.radius
        big = 1e8
        return torch.full((2,), -big, dtype=F64), torch.full((2,), big, dtype=F64)

    def unbounded(self):
        """the solid reaches infinity: a half plane or a cavity (scene.py:1036-1046)."""
        from .implicit import HalfPlaneBody
        return isinstance(self.shape, HalfPlaneBody) or getattr(self.shape, "solid", None) == "outside"

    def lowered(self, hmin, device):
        """the exact-integral form for the fused wall evaluation (scene.py:582-588)."""
        from .implicit import DiskBody
        if not isinstance(self.shape, DiskBody):
            raise NotImplementedError("FusedWall: a half plane has no polygon form (the reference serves it by its "
                                      "per-operation path, not the fused wall)")
        if self.shape.solid == "inside":
            return self.disks().to(device)
        return self.fallbackSurface(hmin, device)

    def disks(self):
        """a solid disk as a one-disk DiskArrayRep, cached (scene.py:576-580)."""
        if getattr(self, "_disks", None) is None:
            self._disks = DiskArrayRep([self.shape.center], [self.shape.radius])
        return self._disks

    def fallbackSurface(self, hmin, device):
        """the area-preserving regular polygon with n = max(24, ceil(2 pi R / (edge bound * hmin))) edges, cached per
        n (scene.py:590-596)."""
        s = self.shape
        n = max(24, int(np.ceil(2 * np.pi * s.radius / (self.policy.maxPolygonEdgeOverH * float(hmin)))))
        if n not in self._fallback:
            self._fallback[n] = SurfaceRep.regularPolygon(s.center, s.radius, n, solid=s.solid)
        return self._fallback[n].to(device)

    def signed(self, lpos):
        d, n, _ = self.shape.signed(lpos)
        return d, n


def _marching_squares(d, origin, spacing):
    """the zero level set of node values d [nx, ny] (d < 0 solid) as a SurfaceRep with the solid on the left of every
    edge (scene.py:762-805).  Per cell the sign changes along its counter-clockwise boundary are exits (solid ->
    fluid) and entries; each exit links to the next entry along the boundary, or -- in a saddle cell whose mean
    value is solid (the solid connects across the cell) -- to the previous one.  A crossing's vertex interpolates d
    linearly from the first end of the cell side as the cell walks it.  The border nodes must all be fluid (an
    obstacle, background 0) or all solid (a tank, background 1)."""
    d = np.asarray(d, dtype=float)
    nx, ny = d.shape
    solid = d < 0
    border = np.concatenate([solid[0], solid[-1], solid[1:-1, 0], solid[1:-1, -1]])
    if border.any() and not border.all():
        raise ValueError("SdfRep.contour: the sampled grid must cover the body with a margin (all border nodes "
                         "fluid, or all solid)")
    background = 1 if border.all() else 0
    ox, oy = float(origin[0]), float(origin[1])
    verts, vid, edges = [], {}, []

    def crossing(a, b):
        key = (a, b)
        if key not in vid:
            t = d[a] / (d[a] - d[b])
            vid[key] = len(verts)
            verts.append((ox + spacing * (a[0] + t * (b[0] - a[0])), oy + spacing * (a[1] + t * (b[1] - a[1]))))
        return vid[key]

    corners = solid[:-1, :-1].astype(np.int8) + solid[1:, :-1] + solid[1:, 1:] + solid[:-1, 1:]
    for i, j in zip(*np.nonzero((corners > 0) & (corners < 4))):
        i, j = int(i), int(j)
        ring = ((i, j), (i + 1, j), (i + 1, j + 1), (i, j + 1))
        seq = []                                       # (is_exit, vertex) in boundary order
        for k in range(4):
            a, b = ring[k], ring[(k + 1) % 4]
            if solid[a] != solid[b]:
                seq.append((bool(solid[a]), crossing(a, b)))
        m = len(seq)
        step = -1 if (m == 4 and d[i:i + 2, j:j + 2].mean() < 0) else 1
        for k in range(m):
            if seq[k][0]:
                q = (k + step) % m
                while seq[q][0]:
                    q = (q + step) % m
                edges.append((seq[k][1], seq[q][1]))
    if not edges:
        raise ValueError("SdfRep.contour: no zero level set in the sampled grid")
    return SurfaceRep(np.asarray(verts, dtype=float), np.asarray(edges, dtype=np.int32), background=background,
                      conditioned=False)


class SdfRep:
    """a sampled signed distance in the body frame, positive in the fluid, on a regular grid (scene.py:599-705).
    The fused wall path integrates its exact polygon form: the given `fallback` surface, else the marching-squares
    contour of the samples.  The reference's sampled-field tier-3 model belongs to its per-operation path and is
    not built; the signed distance of the representation is the exact distance to that polygon."""
    kind = "sdf"

    def __init__(self, values, origin, spacing, fallback: Optional[SurfaceRep] = None, **guards):
        self.d = torch.as_tensor(values, dtype=F64)
        self.origin = torch.as_tensor(origin, dtype=F64)
        self.spacing = float(spacing)
        if not self.spacing > 0:
            raise ValueError("SdfRep: the grid spacing must be positive")
        self.fallback = fallback
        self.guards = guards           # the reference's tier-3 guard settings, kept for its signature
        self._contour = None

    @staticmethod
    def fromFunction(fn, lo, hi, spacing, **kw):
        """sample fn(points [M, 2]) -> d on the regular grid covering [lo, hi] (scene.py:640-647)."""
        nx = int(np.ceil((hi[0] - lo[0]) / spacing)) + 1
        ny = int(np.ceil((hi[1] - lo[1]) / spacing)) + 1
        X, Y = np.meshgrid(lo[0] + spacing * np.arange(nx), lo[1] + spacing * np.arange(ny), indexing="ij")
        pts = torch.as_tensor(np.stack([X.ravel(), Y.ravel()], 1), dtype=F64)
        return SdfRep(fn(pts).reshape(nx, ny), lo, spacing, **kw)

    def to(self, device):
        self.d, self.origin = self.d.to(device), self.origin.to(device)
        if self.fallback is not None:
            self.fallback.to(device)
        if self._contour is not None:
            self._contour.to(device)
        return self

    def contour(self):
        if self._contour is None:
            self._contour = _marching_squares(self.d.cpu().numpy(), self.origin.cpu().numpy(),
                                              self.spacing).to(self.d.device)
        return self._contour

    def lowered(self, hmin, device):
        """the given fallback surface, else the contour (scene.py:663-666)."""
        fb = self.fallback if self.fallback is not None else self.contour()
        return fb.to(device)

    def unbounded(self):
        return bool(self.lowered(0.0, self.d.device).background)

    def bounds(self):
        ext = torch.as_tensor(self.d.shape, dtype=F64) - 1
        o = self.origin.cpu()
        return o, o + ext * self.spacing

@dataclass
class SurfaceTopology:
    """the pair list of one SurfaceRep against a set of queries (scene.py:145-178): (query row, edge) pairs with the
    segment closer than the support, rows ascending, a row's edges in cell-list order; the rows' indicator."""
    qi: torch.Tensor
    e: torch.Tensor
    supMax: float
    _ind: Optional[torch.Tensor] = None

    def indicator(self, rep, lpos, lsup=None):
        if self._ind is None:
            self._ind = rep.indicator(lpos, lsup)
        return self._ind

    def restrict(self, rowmap, rows):
        """the pairs of the rows `rows` only, renumbered by `rowmap` (old row -> new row or -1; scene.py:160-178)."""
        new = rowmap[self.qi.long()]
        sel = new >= 0
        return SurfaceTopology(new[sel].to(torch.int32), self.e[sel], self.supMax,
                               None if self._ind is None else self._ind[rows])


@dataclass
class RepMoments:
    """per-query moments of one representation in physical units (scene.py:181-210): lam [P], g0 [P, 2] =
    int grad_x W, m1 [P, 2] = int y W, g1 [P, 2, 2] = int y_d d_j W, m2 [P, 2, 2] = int y_d y_e W (y = x' - x_i);
    the conditioned quadrature's estimate [P, 12] and status [P] (0 closed form, 1 refined area, -1 failed)."""
    q: torch.Tensor
    lam: torch.Tensor
    g0: torch.Tensor
    m1: Optional[torch.Tensor] = None
    g1: Optional[torch.Tensor] = None
    m2: Optional[torch.Tensor] = None
    quadrature_estimate: Optional[torch.Tensor] = None
    quadrature_status: Optional[torch.Tensor] = None

    def toWorld(self, pose: Pose):
        """the moments rotated to the world frame; error estimates rotated by |R| (bounds stay bounds)."""
        R = pose.R.to(self.lam.device)
        est = self.quadrature_estimate
        if est is not None:
            A = R.abs()
            est = est.clone()
            est[:, 1:3] = est[:, 1:3] @ A.T
            est[:, 3:5] = est[:, 3:5] @ A.T
            est[:, 5:9] = (A @ est[:, 5:9].reshape(-1, 2, 2) @ A.T).flatten(1)
            E = A @ torch.stack([est[:, 9], est[:, 10], est[:, 10], est[:, 11]], 1).reshape(-1, 2, 2) @ A.T
            est[:, 9], est[:, 10], est[:, 11] = E[:, 0, 0], E[:, 0, 1], E[:, 1, 1]
        return RepMoments(self.q, self.lam, self.g0 @ R.T, None if self.m1 is None else self.m1 @ R.T,
                          None if self.g1 is None else R @ self.g1 @ R.T, None if self.m2 is None else R @ self.m2 @ R.T,
                          est, self.quadrature_status)


@dataclass
class PairMoments:
    """the per-pair integrals of ONE kernel (and channel set) over an adjacency (scene.py:1111-1120): per body
    dict(body, cand, surface=[RepMoments world], implicit=[RepMoments world], volume=[]); `channels` None = all
    twelve."""
    numQueries: int
    kernel: str
    entries: list
    stats: dict
    channels: Optional[frozenset] = None


# ----------------------------------------------------------------------------------------------------------- bodies
@dataclass
class Body:
    bodyId: int = 0
    center: tuple = (0.0, 0.0)
    angle: float = 0.0
    linearVelocity: tuple = (0.0, 0.0)
    angularVelocity: float = 0.0
    reps: list = field(default_factory=list)
    linearAcceleration: tuple = (0.0, 0.0)
    angularAcceleration: float = 0.0
    bc: str = "noSlip"
    bcValue: tuple = (0.0, 0.0)

    def __post_init__(self):
        self.center = torch.as_tensor(self.center, dtype=F64)
        self.linearVelocity = torch.as_tensor(self.linearVelocity, dtype=F64)
        self.linearAcceleration = torch.as_tensor(self.linearAcceleration, dtype=F64)
        self.bcValue = torch.as_tensor(self.bcValue, dtype=F64)

    @property
    def pose(self):
        return Pose(self.center, float(self.angle))

    def relative(self, world):
        return world - self.center

    def toLocal(self, world):
        return self.pose.toLocal(world)

    def velocityAt(self, world):
        """v + omega J (x - c) (scene.py:1063-1067)."""
        w = float(self.angularVelocity)
        r = self.relative(world)
        return self.linearVelocity.to(world.device) + w * torch.stack([-r[:, 1], r[:, 0]], 1)

    def accelerationAt(self, world):
        """a + alpha J s - omega^2 s (scene.py:934-939)."""
        s = self.relative(world)
        w, al = float(self.angularVelocity), float(self.angularAcceleration)
        return self.linearAcceleration.to(world.device) + al * torch.stack([-s[:, 1], s[:, 0]], 1) - w * w * s

    def move(self, dt: float):
        """explicit Euler pose update (scene.py:968-973)."""
        self.center = self.center + dt * self.linearVelocity
        self.angle = float(self.angle) + dt * float(self.angularVelocity)
        self.linearVelocity = self.linearVelocity + dt * self.linearAcceleration.to(self.linearVelocity.device)
        self.angularVelocity = float(self.angularVelocity) + dt * float(self.angularAcceleration)

    def obb(self):
        """the bounding box of the representations in the body frame (host floats, cached)."""
        key = tuple(id(r) for r in self.reps)
        c = self.__dict__.get("_obbCache")
        if c is None or c[0] != key:
            # a sampled distance is integrated as its polygon, which a fallback surface may extend past the grid
            los, his = zip(*[(r.lowered(0.0, r.d.device) if isinstance(r, SdfRep) else r).bounds() for r in self.reps])
            lo = torch.stack([a.cpu() for a in los]).amin(0)
            hi = torch.stack([a.cpu() for a in his]).amax(0)
            c = (key, (float(lo[0]), float(lo[1]), float(hi[0]), float(hi[1])))
            self._obbCache = c
        return c[1]

    def unbounded(self):
        """the static exterior-solid broadphase convention (scene.py:1036-1046): a surface with background 1 (a tank
        outline), a cavity disk or a half plane, a sampled distance whose contour is a tank."""
        return any((isinstance(r, SurfaceRep) and r.background) or
                   (isinstance(r, (ImplicitRep, SdfRep)) and r.unbounded()) for r in self.reps)

    def fusable(self):
        from .implicit import DiskBody
        return all(isinstance(r, (SurfaceRep, SdfRep, DiskArrayRep)) or
                   (isinstance(r, ImplicitRep) and isinstance(r.shape, DiskBody)) for r in self.reps)

    def fused_reps(self, hmin, device):
        """the representations as the fused wall evaluation integrates them exactly (scene.py:970-997): SurfaceRep,
        BoxRep and DiskArrayRep as they are, ImplicitRep and SdfRep lowered (a solid disk to a disk set, a cavity or
        a sampled distance to a polygon); cached per (hmin, device).  NotImplementedError for a representation
        without such a form."""
        cache = self.__dict__.setdefault("_fusedCache", {})
        key = (float(hmin), str(device), tuple(id(r) for r in self.reps))
        if key not in cache:
            out = []
            for r in self.reps:
                if isinstance(r, (SurfaceRep, DiskArrayRep)):
                    out.append(r)
                elif isinstance(r, (ImplicitRep, SdfRep)):
                    out.append(r.lowered(hmin, device))
                else:
                    raise NotImplementedError(f"FusedWall: {type(r).__name__} is not built")
            cache[key] = out
        return cache[key]

    def pose_tensor(self, device):
        """(cx, cy, cos, sin) on the device, cached while the pose is unchanged."""
        c, s = self.pose._cs()
        key = (self.center.data_ptr(), self.center._version, c, s, str(device))
        hit = self.__dict__.get("_poseCache")
        if hit is None or hit[0] != key:
            t = torch.cat([self.center.to(device, F64).reshape(2), torch.tensor([c, s], dtype=F64, device=device)])
            hit = (key, t)
            self._poseCache = hit
        return hit[1]

    def state_row(self):
        """(cx, cy, cos, sin, vx, vy, omega, ax, ay, alpha) of the kinematics kernel."""
        c, s = self.pose._cs()
        return [float(self.center[0]), float(self.center[1]), c, s, float(self.linearVelocity[0]),
                float(self.linearVelocity[1]), float(self.angularVelocity), float(self.linearAcceleration[0]),
                float(self.linearAcceleration[1]), float(self.angularAcceleration)]


class BodyKinematics:
    """rigid-body fields of all bodies at the positions x, [B, N, 2] each, from one kernel launch (scene.py:1155-1225):
    rel = x - c, local = Pose.toLocal(x), velocity = v + omega J rel, acceleration = a + alpha J rel - omega^2 rel."""

    def __init__(self, bodies, x):
        self.x = x.to(F64).contiguous()
        self._bodies = bodies
        B, N, dev = len(bodies), len(x), x.device
        state = torch.tensor([b.state_row() for b in bodies], dtype=F64, device=dev).reshape(-1)
        self.rel = torch.empty((B, N, 2), dtype=F64, device=dev)
        self._loc = torch.empty_like(self.rel)
        self._vel = torch.empty_like(self.rel)
        self._acc = torch.empty_like(self.rel)
        check(lib.wsb_kinematics(ptr(state), B, ptr(self.x), N, ptr(self.rel), ptr(self._loc), ptr(self._vel),
                                 ptr(self._acc), _stream()), "wsb_kinematics")

    @property
    def local(self):
        return self._loc

    @property
    def velocity(self):
        return self._vel

    @property
    def acceleration(self):
        return self._acc


class Scene:
    def __init__(self, bodies: List[Body], device="cuda"):
        self.bodies = bodies
        self.device = torch.device(device)
        for b in bodies:
            b.center = b.center.to(self.device)
            b.linearVelocity = b.linearVelocity.to(self.device)
            b.linearAcceleration = b.linearAcceleration.to(self.device)
            b.bcValue = b.bcValue.to(self.device)
            for r in b.reps:
                r.to(self.device)

    def kinematics(self, x):
        return BodyKinematics(self.bodies, x) if self.bodies else None

    # ---- the Scene route to the twelve moments: adjacency (integers, kernel independent) then precompute (per kernel)
    def adjacency(self, queryParticles, operationProperties):
        """`SceneAdjacency` (scene.py:1400-1416): per body the candidate queries (support circle against the body box;
        every allowed query of an unbounded body), their body-frame positions and supports, and the pair topology of
        every SurfaceRep (None for the other representations, whose pairs `precompute` makes).  Only
        `operationProperties.operationMode` is read; one adjacency serves every kernel and channel set."""
        from .fixedadj import BodyAdjacency, SceneAdjacency, body_candidates
        from .shim import queryAllowed
        dev = self.device
        pos = queryParticles.positions.to(dev, F64).contiguous()
        sup = queryParticles.supports.to(dev, F64).contiguous()
        if pos.shape[1] != 2:
            raise NotImplementedError("2D only")
        allowed = queryAllowed(queryParticles, operationProperties.operationMode, dev)
        kin = self.kinematics(pos)
        bodies, stats = [], {"candidates": []}
        for bi, body in enumerate(self.bodies):
            valid = body_candidates(body, kin.local[bi], sup, allowed)
            cand = torch.nonzero(valid).flatten()
            lpos, lsup = kin.local[bi][cand].contiguous(), sup[cand].contiguous()
            stats["candidates"].append(int(len(cand)))
            reps = [(r.topology(lpos, lsup) if isinstance(r, SurfaceRep) and len(cand) else None) for r in body.reps]
            bodies.append(BodyAdjacency(body, cand, lpos, lsup, reps))
        return SceneAdjacency(len(pos), bodies, stats, queryParticles)

    def precompute(self, adjacency, operationProperties, channels=None, precision="fp64"):
        """`PairMoments` of one kernel over an adjacency (scene.py:1418-1433): per body the world-frame `RepMoments` of
        every SurfaceRep on its pair list ('surface'), of implicit and sampled shapes through their exact polygon
        ('implicit'); channels as in `SurfaceRep.moments`.  Disk sets have no pair-list form here (the fused route
        integrates them)."""
        from .shim import kernelName
        from .kernels import QUAD_KERNEL_IDS
        k = operationProperties.kernel
        name = k if isinstance(k, str) and k in QUAD_KERNEL_IDS else kernelName(k)
        entries, stats = [], {"candidates": list(adjacency.stats.get("candidates") or []), "pairs": 0}
        for ba in adjacency.bodies:
            ent = {"body": ba.body, "cand": ba.cand, "surface": [], "implicit": [], "volume": []}
            if len(ba.cand):
                pose = ba.body.pose
                for rep, topo in zip(ba.body.reps, ba.reps):
                    if isinstance(rep, SurfaceRep):
                        m = rep.moments(topo, ba.lpos, ba.lsup, ba.cand, name, self.device, channels, precision)
                        ent["surface"].append(m.toWorld(pose))
                    elif isinstance(rep, (ImplicitRep, SdfRep)):
                        surf = rep.lowered(float(ba.lsup.max()), self.device)
                        if not isinstance(surf, SurfaceRep):
                            raise NotImplementedError("Scene.precompute: a solid disk has no pair-list form here "
                                                      "(the fused route integrates it)")
                        m = surf.pairs(ba.lpos, ba.lsup, ba.cand, name, self.device, channels, precision)
                        ent["implicit"].append(m.toWorld(pose))
                    else:
                        raise NotImplementedError(f"Scene.precompute: {type(rep).__name__} has no pair-list form here "
                                                  f"(the fused route integrates it)")
            stats["pairs"] += sum(len(m.q) for m in ent["surface"] + ent["implicit"])
            entries.append(ent)
        return PairMoments(adjacency.numQueries, name, entries, stats,
                           None if channels is None else frozenset(int(c) for c in channels))

    def pairMoments(self, queryParticles, operationProperties, channels=None, precision="fp64"):
        """adjacency + precompute in one call (scene.py:1435-1437)."""
        return self.precompute(self.adjacency(queryParticles, operationProperties), operationProperties, channels,
                               precision)

    def moments(self, source, queryParticles, operationProperties, channels=None, precision="fp64"):
        """`source` as PairMoments: None builds adjacency + precompute, a SceneAdjacency is precomputed, a PairMoments
        is returned as it is (scene.py:1439-1446)."""
        from .fixedadj import SceneAdjacency
        if source is None:
            return self.pairMoments(queryParticles, operationProperties, channels, precision)
        if isinstance(source, SceneAdjacency):
            return self.precompute(source, operationProperties, channels, precision)
        if isinstance(source, PairMoments):
            return source
        raise TypeError(f"Scene.moments: unsupported source {type(source).__name__}")

    def signed_distance(self, points, body=None, supportMax=None, want_body=False):
        """(d [M], n [M, 2], hit [M][, body [M]]) of world points to the nearest body: d > 0 in the fluid, n the unit
        normal from the wall into the fluid (scene.py:1312-1372)."""
        pts = points.to(self.device, F64).contiguous()
        M = len(pts)
        bidx = torch.full((M,), -1, dtype=torch.long, device=self.device)
        best = torch.full((M,), float("inf"), dtype=F64, device=self.device)
        normal = torch.zeros((M, 2), dtype=F64, device=self.device)
        hit = torch.zeros(M, dtype=torch.bool, device=self.device)
        for bi, bd in enumerate(self.bodies):
            if body is not None and bi != body:
                continue
            lp = bd.toLocal(pts).contiguous()
            for rep in bd.reps:
                if isinstance(rep, SdfRep):
                    rep = rep.lowered(0.0, self.device)        # the exact distance to its polygon form
                if isinstance(rep, (BoxRep, ImplicitRep, DiskArrayRep)):
                    # the shape's own closed form and normals (scene.py:1351-1353, 1360-1362)
                    d, nl = rep.signed(lp)
                    n = bd.pose.vecToWorld(nl)
                    better = d < best
                    best = torch.where(better, d, best)
                    normal = torch.where(better[:, None], n, normal)
                    bidx = torch.where(better, torch.full_like(bidx, bi), bidx)
                    hit |= True
                    continue
                if not isinstance(rep, SurfaceRep):
                    continue
                ns = rep.native(supportMax, self.device) if supportMax is not None else rep._default_native(self.device)
                d = torch.empty(M, dtype=F64, device=self.device)
                cp = torch.empty((M, 2), dtype=F64, device=self.device)
                nl = torch.empty((M, 2), dtype=F64, device=self.device)
                ed = torch.empty(M, dtype=torch.int32, device=self.device)
                check(lib.wsb_signed_distance(ns.handle, ptr(lp), M, float(supportMax) if supportMax else 0.0, ptr(d),
                                              ptr(cp), ptr(nl), ptr(ed), _stream()), "wsb_signed_distance")
                n = bd.pose.vecToWorld(nl)
                better = d < best
                best = torch.where(better, d, best)
                normal = torch.where(better[:, None], n, normal)
                bidx = torch.where(better, torch.full_like(bidx, bi), bidx)
                hit |= True
        if want_body:
            return best, normal, hit, bidx
        return best, normal, hit

    def inside(self, points, body=None):
        pts = points.to(self.device, F64)
        out = torch.zeros(len(pts), dtype=torch.bool, device=self.device)
        for bi, bd in enumerate(self.bodies):
            if body is not None and bi != body:
                continue
            lp = bd.toLocal(pts)
            for rep in bd.reps:
                if isinstance(rep, SdfRep):
                    rep = rep.lowered(0.0, self.device)
                if isinstance(rep, (ImplicitRep, DiskArrayRep)):
                    out |= rep.signed(lp)[0] < 0
                elif isinstance(rep, SurfaceRep):
                    out |= rep.indicator(lp) > 0.5
        return out
