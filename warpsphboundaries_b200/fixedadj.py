"""Fixed-capacity, sync-free wall adjacency (src/warpSPHBoundaries/scene/fixedadj.py).

Every query is a row; a surface gets K slots per row (K = the largest number of
edges stored in one cell of its static cell list), filled with the edges whose
segment lies closer than the row's support, in cell-list order, and the row's
winding indicator.  One launch of `wsb_fixed_topology` per (body, surface); the
static cell list is built once per (surface, supportMax) by integer counting
sort inside `wsb_surface_create`.
"""
from dataclasses import dataclass, field
from typing import Optional

import torch

from ._lib import check, lib, ptr
from .scene import SurfaceRep, _stream
from .shim import queryAllowed

F64 = torch.float64
_ROWS = {}


def _slot_rows(N, K, device):
    key = (N, K, str(device))
    t = _ROWS.get(key)
    if t is None:
        t = torch.arange(N * K, device=device, dtype=torch.int32) // K
        _ROWS[key] = t
    return t


@dataclass
class FixedTopology:
    """slots instead of a pair list: e [N*K] int32 (-1 empty), qi [N*K] the row of a slot, ind [N] float64."""
    e: torch.Tensor
    qi: torch.Tensor
    K: int
    ind: torch.Tensor

    def indicator(self, rep=None, lpos=None, lsup=None):
        return self.ind

    def csr(self, rows):
        dev = self.e.device
        return (torch.arange(rows * self.K, dtype=torch.int32, device=dev),
                torch.arange(rows + 1, dtype=torch.int32, device=dev) * self.K)


def fixed_topology(rep: SurfaceRep, lpos, lsup, valid, supportMax):
    """`FixedTopology` of rows lpos [N, 2] (body frame), supports lsup [N], candidates valid [N] against `rep`
    (fixedadj.py:168-182)."""
    ns = rep.native(supportMax, lpos.device)
    N, K = len(lpos), ns.K
    lp = lpos.to(F64).contiguous()
    ls = lsup.to(F64).contiguous()
    vi = None if valid is None else valid.to(torch.int32).contiguous()
    e = torch.empty(N * K, dtype=torch.int32, device=lpos.device)
    ind = torch.empty(N, dtype=F64, device=lpos.device)
    check(lib.wsb_fixed_topology(ns.handle, ptr(lp), ptr(ls), ptr(vi), N, ptr(e), ptr(ind), _stream()),
          "wsb_fixed_topology")
    return FixedTopology(e, _slot_rows(N, K, lpos.device), K, ind)


@dataclass
class BodyAdjacency:
    body: object
    cand: torch.Tensor
    lpos: torch.Tensor
    lsup: torch.Tensor
    reps: list
    valid: Optional[torch.Tensor] = None
    repList: Optional[list] = None


@dataclass
class SceneAdjacency:
    """who interacts with whom (scene.py:1083-1108): per body a BodyAdjacency; integers and kernel-independent
    geometry only, so one adjacency serves every kernel and channel set at these positions."""
    numQueries: int
    bodies: list
    stats: dict = field(default_factory=dict)
    queryParticles: object = None
    supportMax: float = 0.0

    def restrict(self, index):
        """the adjacency of the global rows `index` (ascending, distinct) alone, renumbered 0 .. len(index) - 1
        (scene.py:1090-1108); no search."""
        dev = index.device
        newid = torch.full((self.numQueries,), -1, dtype=torch.long, device=dev)
        newid[index] = torch.arange(len(index), device=dev)
        out = []
        for ba in self.bodies:
            rows = torch.nonzero(newid[ba.cand] >= 0).flatten()
            rowmap = torch.full((len(ba.cand),), -1, dtype=torch.long, device=dev)
            rowmap[rows] = torch.arange(len(rows), device=dev)
            out.append(BodyAdjacency(ba.body, newid[ba.cand[rows]], ba.lpos[rows], ba.lsup[rows],
                                     [None if t is None else t.restrict(rowmap, rows) for t in ba.reps]))
        return SceneAdjacency(len(index), out, {"candidates": [len(b.cand) for b in out]}, None, self.supportMax)


def body_candidates(body, lpos, sup, allowed):
    """the broadphase of fixedadj.py:261-264: support circle against the body box (every row of an unbounded body)."""
    if body.unbounded():
        return allowed
    x0, y0, x1, y1 = body.obb()
    lo = torch.tensor([x0, y0], dtype=F64, device=lpos.device)
    hi = torch.tensor([x1, y1], dtype=F64, device=lpos.device)
    d = (lo - lpos).clamp(min=0) + (lpos - hi).clamp(min=0)
    return (d.norm(dim=1) < sup) & allowed


def fixed_adjacency(scene, queryParticles, operationProperties, supportMax):
    """`SceneAdjacency` of every query against every body with fixed shapes (fixedadj.py:249-270)."""
    dev = scene.device
    pos, sup = queryParticles.positions.to(dev, F64), queryParticles.supports.to(dev, F64)
    if pos.shape[1] != 2:
        raise NotImplementedError("2D only")
    allowed = queryAllowed(queryParticles, operationProperties.operationMode, dev)
    N = len(pos)
    cand = torch.arange(N, device=dev)
    kin = scene.kinematics(pos)
    bodies = []
    for bi, body in enumerate(scene.bodies):
        lpos = kin.local[bi]
        valid = body_candidates(body, lpos, sup, allowed)
        surfaces = body.fused_reps(supportMax, dev)                  # implicit / sampled shapes as their polygon
        reps = [fixed_topology(rep, lpos, sup, valid, supportMax) for rep in surfaces]
        bodies.append(BodyAdjacency(body, cand, lpos, sup, reps, valid, list(surfaces)))
    return SceneAdjacency(N, bodies, {"candidates": None}, queryParticles, float(supportMax))


def indicator_device(rep, lpos, supportMax):
    """winding number + background of body-frame points against `rep`, sync-free (fixedadj.py:273-276)."""
    n = len(lpos)
    return fixed_topology(rep, lpos, torch.full((n,), float(supportMax), dtype=F64, device=lpos.device),
                          torch.ones(n, dtype=torch.bool, device=lpos.device), supportMax).ind
