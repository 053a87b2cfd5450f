"""Solid half-spaces and solid spheres in 3-D: the degree-two Cartesian kernel-integral contract.

Mirrors fluxbridge's request contract and radial family (src/warpSPHBoundaries/fluxbridge/contract.py:10-46,
src/warpSPHBoundaries/fluxbridge/radial.py:108-215): `Request`, `monomials`, `baseline`, `RadialEvaluator(kind,
requests, kernel=, precision=, device=).prepare(distances, normals, supports, radii=)` -> `RadialBatch.launch()`.
The per-query work (nine axial invariants by Gauss-Legendre over the radial shells, rotation into the requested
channels) is `wsb_radial_channels` of libwsb.so; nothing here computes a channel.

Precision names follow the reference: "float64" and "float32" run those arithmetics on the GPU.
"float32_compensated" (the reference's paired-float route for GPUs with slow float64) runs the float64 kernel: on
this hardware float64 throughput is half of float32's, a paired-float operation costs several float32 operations,
and float64 is the more accurate of the two.  Its input domain checks stay those of the reference's float32 routes.
"""
from dataclasses import dataclass
from numbers import Integral

import numpy as np
import torch

from . import _lib
from ._lib import check, lib, ptr
from .kernels import KERNEL_IDS

CONTRACT_VERSION = 1
KERNELS = ("w2", "w4", "w6", "cubic")
MAX_DEGREE = 9


@dataclass(frozen=True)
class Request:
    """one Cartesian kernel integral: the monomial x^alpha times the kernel's partial derivatives `derivative`
    (contract.py:10-28)."""
    alpha: tuple
    derivative: tuple = ()

    def __post_init__(self):
        object.__setattr__(self, "alpha", tuple(self.alpha))
        object.__setattr__(self, "derivative", tuple(self.derivative))
        d = len(self.alpha)
        if d not in (2, 3) or any(not isinstance(a, Integral) or a < 0 for a in self.alpha):
            raise ValueError("alpha must contain two or three nonnegative integers")
        if sum(self.alpha) > MAX_DEGREE:
            raise ValueError("polynomial degree exceeds nine")
        if len(self.derivative) > 2 or any(not isinstance(j, Integral) or j not in range(d) for j in self.derivative):
            raise ValueError("kernel derivatives must have order 0..2 and valid axes")

    @property
    def scale(self):
        return sum(self.alpha) - len(self.derivative)


def monomials(dimension, degree):
    """exponent tuples of total degree 0..degree, graded, each degree in descending lexicographic order
    (contract.py:31-38)."""
    if dimension not in (2, 3) or not isinstance(degree, Integral) or degree not in range(10):
        raise ValueError("dimension must be 2 or 3 and degree 0..9")

    def lattice(d, n):
        if d == 1:
            return [(n,)]
        return [(i,) + rest for i in range(n, -1, -1) for rest in lattice(d - 1, n - i)]
    return tuple(a for n in range(degree + 1) for a in lattice(dimension, n))


def baseline(dimension):
    """value moments |alpha| <= 2, first kernel-derivative moments |alpha| <= 1 per axis, the symmetric kernel
    Hessian (contract.py:41-46): 28 requests in 3-D."""
    z = (0,) * dimension
    return (tuple(Request(a) for a in monomials(dimension, 2)) +
            tuple(Request(a, (j,)) for a in monomials(dimension, 1) for j in range(dimension)) +
            tuple(Request(z, (i, j)) for i in range(dimension) for j in range(i, dimension)))


_PRECISIONS = {"float64": _lib.PREC_FP64, "float32": _lib.PREC_FP32, "float32_compensated": _lib.PREC_FP64}


class RadialEvaluator:
    """Analytic solid half-space ("plane") or solid sphere, outward normals, support radius h (radial.py:108-149).

    `prepare(distances, normals, supports, radii=...)` takes per-query signed outward distances: for a sphere
    distance = |query - centre| - radius and the normal points from the centre to the query.
    """

    def __init__(self, kind, requests=None, *, kernel="w2", precision="float64", device="cuda"):
        if kind not in ("plane", "sphere") or kernel not in KERNELS:
            raise ValueError("kind must be plane or sphere and kernel must be supported")
        if precision not in _PRECISIONS:
            raise ValueError("unknown precision")
        self.kind = kind
        self.kernel = kernel
        self.precision = precision
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise RuntimeError("RadialEvaluator runs on a CUDA device (libwsb.so has no CPU path)")
        self.requests = baseline(3) if requests is None else tuple(requests)
        meta = []
        for r in self.requests:
            if not isinstance(r, Request) or len(r.alpha) != 3 or sum(r.alpha) + len(r.derivative) > 2:
                raise ValueError("radial family supports the complete 3D baseline and subsets only")
            ids = [i for i, a in enumerate(r.alpha) for _ in range(a)] + list(r.derivative)
            meta.append([sum(r.alpha), *(ids + [0, 0])[:2], len(r.derivative)])
        self.metadata = np.ascontiguousarray(np.array(meta, dtype=np.int32).reshape(-1, 4))
        self._kind_id = _lib.RADIAL_SPHERE if kind == "sphere" else _lib.RADIAL_PLANE
        self._kernel_id = KERNEL_IDS[kernel]
        self._prec_id = _PRECISIONS[precision]
        self.accuracy_status = "reference 70-digit radial and sphere fixtures pass on the GPU (float64)"

    def prepare(self, distances, normals, supports, *, radii=None):
        """validated, frozen device arrays of one batch (radial.py:151-185)."""
        d = np.atleast_1d(_host(distances))
        if d.ndim != 1:
            raise ValueError("distances must be a scalar or vector")
        count = len(d)
        try:
            h = np.broadcast_to(_host(supports), (count,)).copy()
            n = np.broadcast_to(_host(normals), (count, 3)).copy()
            r = np.zeros(count) if radii is None else np.broadcast_to(_host(radii), (count,)).copy()
        except ValueError as exc:
            raise ValueError("incompatible radial batch shapes") from exc
        if not all(np.isfinite(a).all() for a in (d, n, h, r)) or np.any(h <= 0):
            raise ValueError("radial inputs must be finite with positive support")
        if not np.allclose(np.linalg.norm(n, axis=1), 1., rtol=0., atol=1e-12):
            raise ValueError("normals must be unit outward vectors")
        if self.kind == "sphere":
            if radii is None or np.any(r <= 0) or np.any(d < -r):
                raise ValueError("sphere needs positive radii and distance >= -radius")
            lower = 1e-2 if self.precision.startswith("float32") else 1e-4
            if np.any(r / h < lower) or np.any(r / h > 1e4):
                raise ValueError("radius/support outside the tested radial conditioning domain")
        elif radii is not None:
            raise ValueError("plane does not accept sphere radii")
        dtype = np.float32 if self.precision == "float32" else np.float64
        with np.errstate(over="ignore", under="ignore", divide="ignore", invalid="ignore"):
            dd, nn, hh, rr = [a.astype(dtype) for a in (d, n, h, r)]
            square = hh * hh
            representable = (all(np.isfinite(a).all() for a in (dd, nn, hh, rr, dd / hh, rr / hh, square, 1 / square))
                             and np.all(square > 0))
        if not representable:
            name = "fp32" if dtype == np.float32 else "fp64"
            raise ValueError(f"radial inputs or support scaling exceed finite {name} storage")
        return RadialBatch(self, d, n, h, r)

    def evaluate(self, distances, normals, supports, **kwargs):
        batch = self.prepare(distances, normals, supports, **kwargs)
        batch.launch()
        return batch.numpy()


class RadialBatch:
    """Frozen prepared device arrays; `launch` reuses them and allocates nothing (radial.py:188-215)."""

    def __init__(self, evaluator, d, n, h, r):
        self.evaluator = evaluator
        self.count = len(d)
        dev = evaluator.device
        as_dev = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
        self.distances = as_dev(d)
        self.normals = as_dev(n).reshape(self.count, 3)
        self.supports = as_dev(h)
        self.radii = as_dev(r)
        self.work = torch.empty((self.count, 9), dtype=torch.float64, device=dev)
        self.values = torch.empty((self.count, len(evaluator.requests)), dtype=torch.float64, device=dev)
        self.status = torch.empty(self.count, dtype=torch.int32, device=dev)

    @property
    def bytes(self):
        return sum(t.numel() * t.element_size() for t in (self.distances, self.normals, self.supports, self.radii,
                                                           self.work, self.values, self.status))

    def launch(self, stream=None):
        ev = self.evaluator
        if self.count and len(ev.requests):
            st = stream if stream is not None else torch.cuda.current_stream(ev.device)
            meta = ev.metadata
            with torch.cuda.device(ev.device):
                check(lib.wsb_radial_channels(ev._kind_id, ev._kernel_id, ev._prec_id, ptr(self.distances),
                                              ptr(self.radii) if ev.kind == "sphere" else None, ptr(self.normals),
                                              ptr(self.supports), self.count,
                                              meta.ctypes.data_as(_lib.POINTER(_lib.c_int32)), len(ev.requests),
                                              ptr(self.values), ptr(self.work), ptr(self.status),
                                              _lib.c_void_p(st.cuda_stream)), "wsb_radial_channels")
        return self.values

    def numpy(self):
        return self.values.cpu().numpy()


def _host(a):
    if isinstance(a, torch.Tensor):
        return a.detach().to("cpu", torch.float64).numpy()
    return np.asarray(a, dtype=float)
