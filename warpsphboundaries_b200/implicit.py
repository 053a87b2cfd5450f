"""Analytic primitives of the scene layer (src/warpSPHBoundaries/scene/implicitBodies.py:292-352): `DiskBody`,
`HalfPlaneBody` and the `TierPolicy` whose polygon edge bound sets how finely the fused wall path lowers a cavity
disk to a polygon.  The tier-3 / tier-4 curvature models of the reference's per-operation path are not part of the
fused boundary integral and are not built here."""
from dataclasses import dataclass
from typing import Tuple

import torch

F64 = torch.float64


@dataclass
class TierPolicy:
    """thresholds in units of the particle's support (implicitBodies.py:292-297); the fused path uses only
    `maxPolygonEdgeOverH`, the edge bound of the tier-2 polygon."""
    tier4MaxRadius: float = 0.2
    tier3MinRadius: float = 2.0
    maxPolygonEdgeOverH: float = 1.0 / 16.0


def _const(obj, name, device):
    """`obj.<name>` as a float64 tensor on `device`, converted once per (value, device) so that no call copies a host
    tensor (a synchronisation) after the first."""
    cache = obj.__dict__.setdefault("_dev", {})
    val = getattr(obj, name)
    key = (name, str(device), tuple(val))
    if key not in cache:
        cache[key] = torch.as_tensor(val, dtype=F64, device=device)
    return cache[key]


@dataclass
class DiskBody:
    """a disk in the body frame: `solid='inside'` a solid disk (an obstacle), 'outside' a cavity (fluid inside the
    circle) (implicitBodies.py:310-338)."""
    center: Tuple[float, float]
    radius: float
    solid: str = "inside"
    bodyId: int = 0

    def signed(self, pos):
        """(d, n, kappa): the signed distance (positive in the fluid), the unit normal into the fluid, the
        curvature of the wall."""
        v = pos - _const(self, "center", pos.device)
        r = v.norm(dim=1).clamp(min=1e-300)
        e = v / r[:, None]
        if self.solid == "inside":
            return r - self.radius, e, 1.0 / self.radius
        return self.radius - r, -e, -1.0 / self.radius


@dataclass
class HalfPlaneBody:
    """the half plane behind a wall line through `point` with the unit `normal` pointing into the fluid
    (implicitBodies.py:341-351)."""
    point: Tuple[float, float]
    normal: Tuple[float, float]
    bodyId: int = 0

    def signed(self, pos):
        n = _const(self, "normal", pos.device)
        d = ((pos - _const(self, "point", pos.device)) * n).sum(1)
        return d, n.expand_as(pos), 0.0
