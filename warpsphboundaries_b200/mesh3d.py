"""Closed triangle surfaces in 3-D: the degree-two kernel-integral contract over the solid they bound.

Mirrors fluxbridge's closed-surface entry (src/warpSPHBoundaries/fluxbridge/geometry.py:75-84 Geometry.closed_surface,
src/warpSPHBoundaries/fluxbridge/evaluate.py:11-187 Evaluator / Batch): `Geometry.closed_surface(vertices, faces)`,
`Evaluator(geometry, requests, kernel=, precision=, device=).prepare(queries, supports)` -> `Batch.launch()`.
All per-query work (face search, inside test, face -> edge reductions, per-query sums) is `wsb_mesh_channels` of
libwsb.so.  Requests are the 28 baseline requests of the 3-D contract (value moments |alpha| <= 2, kernel-gradient
moments |alpha| <= 1, the kernel Hessian) or any subset of them.

Precision names follow the reference: "float64" and "float32_compensated" run the float64 kernels ("float32" is not
offered: the float64 path is the accurate one and is not slower than a paired-float emulation on this hardware).
"""
import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr
from .kernels import KERNEL_IDS
from .radial import KERNELS, Request, baseline

F64 = torch.float64
_BASE = baseline(3)
_COLUMN = {(r.alpha, r.derivative): k for k, r in enumerate(_BASE)}


def _column(req):
    """column of a request in the native 28-channel row (Hessian entries are symmetric: (j, i) reads (i, j))."""
    d = tuple(req.derivative)
    if len(d) == 2 and d[0] > d[1]:
        d = (d[1], d[0])
    return _COLUMN.get((tuple(req.alpha), d))


class ClosedMesh:
    """a closed surface resident on one device with its face grid for supports up to `support_max`."""

    def __init__(self, vertices, faces, support_max, device="cuda"):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("ClosedMesh lives on a CUDA device (libwsb.so has no CPU path)")
        V = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).reshape(-1, 3))
        Fc = np.ascontiguousarray(np.asarray(faces, dtype=np.int32).reshape(-1, 3))
        self.support_max = float(support_max)
        self.n_faces = len(Fc)
        h = ctypes.c_void_p()
        check(lib.wsb_mesh_create(V.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), len(V),
                                  Fc.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(Fc), self.support_max,
                                  self.device.index if self.device.index is not None else torch.cuda.current_device(),
                                  ctypes.byref(h)), "wsb_mesh_create")
        self.handle = h
        self._ws = None

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            lib.wsb_mesh_destroy(h)
            self.handle = None

    def workspace(self, n):
        need = int(lib.wsb_mesh_workspace_size(self.handle, n))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(max(need, 1), dtype=torch.uint8, device=self.device)
        return self._ws

    def channels(self, pos, sup, kernel="w4", out=None, inside=None, stream=None):
        """[n, 28] float64 baseline channels of the queries pos [n, 3] with supports sup [n] (device tensors)."""
        n = len(pos)
        if out is None:
            out = torch.empty((n, 28), dtype=F64, device=self.device)
        if n == 0:
            return out
        ws = self.workspace(n)
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        check(lib.wsb_mesh_channels(self.handle, KERNEL_IDS[kernel], ptr(pos), ptr(sup), n, ptr(out), ptr(inside),
                                    ptr(ws), ws.numel(), ctypes.c_void_p(st.cuda_stream)), "wsb_mesh_channels")
        return out

    def inside(self, pos, stream=None):
        n = len(pos)
        out = torch.empty(n, dtype=torch.int32, device=self.device)
        if n:
            st = stream if stream is not None else torch.cuda.current_stream(self.device)
            check(lib.wsb_mesh_inside(self.handle, ptr(pos), n, ptr(out), ctypes.c_void_p(st.cuda_stream)),
                  "wsb_mesh_inside")
        return out


class Geometry:
    """a closed, outward-oriented triangle surface (fluxbridge geometry.py:75-84); the surface checks (watertight,
    consistently oriented, positive volume, no zero-area face) run when the first device copy is made."""

    def __init__(self, vertices, faces):
        self.dimension = 3
        self.measure = "volume"
        self.vertices = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).reshape(-1, 3))
        self.faces = np.ascontiguousarray(np.asarray(faces, dtype=np.int64).reshape(-1, 3))
        if not np.isfinite(self.vertices).all():
            raise ValueError("vertices must be finite")
        self.from_tets = False
        self._meshes = {}

    @classmethod
    def closed_surface(cls, vertices, faces):
        return cls(vertices, faces)

    @classmethod
    def from_elements(cls, elements, dimension=3, measure="volume"):
        """the solid of a conforming tetrahedral mesh (fluxbridge geometry.py:20-63: `Geometry(elements, 3,
        'volume')`, each element a [4, 3] array).  The requests are integrals over the solid, and over a conforming
        mesh the elements' integrals add up to those of the union, whose boundary the closed-surface path
        integrates exactly: every face is oriented outward from its tetrahedron (the reference's rule), vertices are
        welded by exact coordinates, and the faces that two tetrahedra share with opposite orientations cancel.
        ValueError for a degenerate tetrahedron or a face shared with the same orientation (overlapping elements);
        NotImplementedError for 2-D elements and surface measure."""
        if dimension != 3 or measure != "volume":
            raise NotImplementedError("fluxbridge elements: 3-D volume tetrahedra only (closed_surface for a skin)")
        index, verts, count = {}, [], {}
        for el in elements:
            v = np.asarray(el, dtype=np.float64)
            if v.shape != (4, 3) or not np.isfinite(v).all():
                raise ValueError("volume elements must be tetrahedra with finite vertices")
            ids = []
            for p in v:
                key = tuple(float(x) for x in p)
                if key not in index:
                    index[key] = len(verts)
                    verts.append(key)
                ids.append(index[key])
            for i in range(4):
                f = [j for j in range(4) if j != i]
                p, q, r = v[f]
                side = float(np.dot(np.cross(q - p, r - p), v[i] - p))
                if side == 0.0:
                    raise ValueError("degenerate tetrahedron")
                if side > 0:                          # the opposite vertex lies on the normal's side: flip outward
                    f[1], f[2] = f[2], f[1]
                tri = tuple(ids[j] for j in f)
                k = min(range(3), key=lambda s: tri[s])
                tri = tri[k:] + tri[:k]               # rotation with the smallest id first keeps the orientation
                if tri in count:
                    raise ValueError("two tetrahedra share a face with the same orientation (overlapping elements)")
                count[tri] = 1
        faces = [tri for tri in count if (tri[0], tri[2], tri[1]) not in count]
        if not faces:
            raise ValueError("no boundary faces")
        g = cls(np.array(verts), np.array(faces, dtype=np.int64))
        g.from_tets = True
        return g

    def native(self, support_max, device):
        """the device copy whose grid serves supports up to `support_max` (rebuilt when a larger one is asked)."""
        device = torch.device(device)
        key = str(device)
        m = self._meshes.get(key)
        if m is None or m.support_max < support_max:
            m = ClosedMesh(self.vertices, self.faces, support_max, device)
            self._meshes[key] = m
        return m


_PRECISIONS = ("float64", "float32_compensated")


class Evaluator:
    """the baseline kernel integrals of a closed surface at queries (fluxbridge evaluate.py:11-187)."""

    def __init__(self, geometry, requests=None, *, kernel="w2", precision="float64", device="cuda", compact=False,
                 method="analytic", search="device", nodes=16, preparation="host"):
        if not isinstance(geometry, Geometry):
            raise ValueError("geometry must come from Geometry.closed_surface or Geometry.from_elements")
        if method in ("conditioned_boundary", "tet_quadrature") and geometry.from_tets:
            method = "analytic"      # the same integrals over the solid, here by the exact boundary reduction
        if kernel not in KERNELS:
            raise ValueError("kernel must be one of " + ", ".join(KERNELS))
        if precision == "float32":
            raise NotImplementedError("closed surfaces run in float64 (precision='float64' or 'float32_compensated')")
        if precision not in _PRECISIONS:
            raise ValueError("unknown precision")
        if method != "analytic":
            raise NotImplementedError("closed surfaces: only the analytic method")
        self.geometry = geometry
        self.kernel = kernel
        self.precision = precision
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("Evaluator runs on a CUDA device (libwsb.so has no CPU path)")
        self.requests = _BASE if requests is None else tuple(requests)
        cols = []
        for r in self.requests:
            if not isinstance(r, Request) or len(r.alpha) != 3:
                raise ValueError("requests must be 3-D Request objects")
            c = _column(r)
            if c is None:
                raise NotImplementedError("closed surfaces serve the 3-D baseline requests (|alpha| <= 2, kernel "
                                          "derivatives with |alpha| + order <= 2) and subsets")
            cols.append(c)
        self.columns = cols
        self.full = cols == list(range(28))
        self.accuracy_status = "reference mpmath closed-surface fixtures pass on the GPU (float64)"

    def prepare(self, queries, supports):
        q = torch.as_tensor(queries, dtype=F64).reshape(-1, 3)
        h = torch.as_tensor(supports, dtype=F64)
        h = torch.broadcast_to(h, (len(q),)).contiguous()
        if not torch.isfinite(q).all() or not torch.isfinite(h).all() or bool((h <= 0).any()):
            raise ValueError("queries and supports must be finite with positive supports")
        # the reference's conservative domain (evaluate.py:96-114): an element spanning less than 1e-4 of a support
        span = float(np.ptp(self.geometry.vertices, axis=0).max())
        if len(h) and span / float(h.max()) < 1e-4:
            raise ValueError("tiny element relative to support: use the arbitrary-precision reference")
        return Batch(self, q.to(self.device).contiguous(), h.to(self.device))

    def evaluate(self, queries, supports):
        b = self.prepare(queries, supports)
        b.launch()
        return b.numpy()


class Batch:
    """frozen device queries and outputs; `launch` reuses them (fluxbridge evaluate.py:145-187)."""

    def __init__(self, evaluator, q, h):
        self.evaluator = evaluator
        self.count = len(q)
        self.queries = q
        self.supports = h
        smax = float(h.max()) if self.count else 1.0
        self.mesh = evaluator.geometry.native(smax, evaluator.device)
        self.raw = torch.empty((self.count, 28), dtype=F64, device=evaluator.device)
        self.inside = torch.empty(self.count, dtype=torch.int32, device=evaluator.device)
        self.values = self.raw if evaluator.full else torch.empty((self.count, len(evaluator.requests)), dtype=F64,
                                                                   device=evaluator.device)
        self.columns = torch.tensor(evaluator.columns, dtype=torch.long, device=evaluator.device)

    def launch(self):
        ev = self.evaluator
        if self.count:
            self.mesh.channels(self.queries, self.supports, ev.kernel, out=self.raw, inside=self.inside)
            if not ev.full:
                torch.index_select(self.raw, 1, self.columns, out=self.values)
        return self.values

    def numpy(self):
        return self.values.cpu().numpy()
