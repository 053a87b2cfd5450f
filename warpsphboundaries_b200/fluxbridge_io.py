"""The fluxbridge fixture file (schema 1) as an interchange format of element scenes and request sets.

A file holds `{"schema": 1, "dps": digits, "cases": [...]}`; a case is one element seen from one query:
`dimension` (2 or 3), `vertices` (a triangle [3, d] or a tetrahedron [4, 3]; numbers or decimal strings), `query`,
`kernel` (w2, w4, w6, cubic), `measure` ("volume", or "surface" for a 3-D triangle), `h`, `requests` (monomial
`alpha` and kernel `derivative` axes, the 3-D / 2-D contract) and `values` (decimal strings in request order).  This
is the layout the reference writes its independent 70-digit fixtures in (scripts/make_fluxbridge_fixtures.py,
tests/fixtures/fluxbridge-v1.json); `load` / `dump` keep every field as written, so a file round-trips unchanged.

`evaluate(case)` computes a case's requests on the device:
* a 3-D tetrahedron (volume) through `mesh3d.Geometry.from_elements` and the closed-surface kernels (the 28 baseline
  requests: value moments |alpha| <= 2, kernel-gradient moments |alpha| <= 1, the kernel Hessian);
* a 2-D triangle (volume) through `FusedWall` on the triangle as a polygon (value moments |alpha| <= 2 and the
  kernel-gradient moments |alpha| <= 1: lam, m1, m2, G, Cov);
and gives NaN for requests outside those sets (higher degrees, the 2-D Hessian) and for a tetrahedron whose query lies
on its boundary (the closed-surface route takes such a query as inside or outside by a ray-parity rule; the reference
uses the solid-angle fraction); 3-D surface triangles raise NotImplementedError (no surface-measure route).
"""
import json
from dataclasses import dataclass, field
from pathlib import Path
from typing import List, Tuple

import numpy as np

from .radial import Request

SCHEMA = 1


@dataclass
class Case:
    dimension: int
    vertices: list
    query: list
    kernel: str
    measure: str
    h: object
    requests: Tuple[Request, ...]
    values: List[str] = field(default_factory=list)

    @property
    def points(self):
        """the vertices as float64 [k, d]."""
        return np.array([[float(x) for x in v] for v in self.vertices], dtype=np.float64)

    @property
    def x(self):
        return np.array([float(v) for v in self.query], dtype=np.float64)

    @property
    def support(self):
        return float(self.h)

    def reference(self):
        """the stored values as float64 (NaN where none is stored)."""
        return np.array([float(v) for v in self.values], dtype=np.float64) if self.values else \
            np.full(len(self.requests), np.nan)


@dataclass
class FixtureFile:
    dps: int
    cases: List[Case]
    schema: int = SCHEMA


def _case(d):
    reqs = tuple(Request(tuple(r["alpha"]), tuple(r.get("derivative", ()))) for r in d["requests"])
    if d["dimension"] not in (2, 3) or any(len(r.alpha) != d["dimension"] for r in reqs):
        raise ValueError("fluxbridge case: dimension and request lengths disagree")
    if d["measure"] not in ("volume", "surface"):
        raise ValueError(f"fluxbridge case: unknown measure {d['measure']!r}")
    vals = list(d.get("values", []))
    if vals and len(vals) != len(reqs):
        raise ValueError("fluxbridge case: one value per request expected")
    return Case(int(d["dimension"]), d["vertices"], d["query"], d["kernel"], d["measure"], d["h"], reqs, vals)


def load(src) -> FixtureFile:
    """a fixture file from a path, a JSON string or an already parsed dict."""
    if isinstance(src, (str, Path)) and Path(src).exists():
        data = json.loads(Path(src).read_text())
    elif isinstance(src, str):
        data = json.loads(src)
    else:
        data = src
    if data.get("schema") != SCHEMA:
        raise ValueError(f"fluxbridge fixture schema {data.get('schema')!r}, expected {SCHEMA}")
    return FixtureFile(int(data["dps"]), [_case(c) for c in data["cases"]], SCHEMA)


def to_dict(f: FixtureFile) -> dict:
    cases = []
    for c in f.cases:
        d = {"dimension": c.dimension, "vertices": c.vertices, "query": c.query, "kernel": c.kernel,
             "measure": c.measure, "h": c.h,
             "requests": [{"alpha": list(r.alpha), "derivative": list(r.derivative)} for r in c.requests]}
        if c.values:
            d["values"] = list(c.values)
        cases.append(d)
    return {"schema": f.schema, "dps": f.dps, "cases": cases}


def dump(f: FixtureFile, path=None) -> str:
    """the file as JSON text in the writer's layout (two-space indent, trailing newline); written to `path` if given."""
    text = json.dumps(to_dict(f), indent=2) + "\n"
    if path is not None:
        Path(path).write_text(text)
    return text


# ------------------------------------------------------------------------------------------------ device evaluation
def _tet_columns(requests):
    from .mesh3d import _column
    return [_column(r) for r in requests]


_TWO_D = {((0, 0), ()): ("lam", ()), ((1, 0), ()): ("m1", (0,)), ((0, 1), ()): ("m1", (1,)),
          ((2, 0), ()): ("m2", (0, 0)), ((1, 1), ()): ("m2", (0, 1)), ((0, 2), ()): ("m2", (1, 1)),
          ((0, 0), (0,)): ("G", (0,)), ((0, 0), (1,)): ("G", (1,)),
          ((1, 0), (0,)): ("Cov", (0, 0)), ((1, 0), (1,)): ("Cov", (0, 1)),
          ((0, 1), (0,)): ("Cov", (1, 0)), ((0, 1), (1,)): ("Cov", (1, 1))}


def _on_tet_boundary(case: Case):
    """the query lies on the tetrahedron's boundary (a face, an edge or a vertex), decided exactly from the file's
    decimal strings: there the closed-surface route takes the query as inside or outside by its ray-parity rule, where
    the reference's solid angle gives the fraction of the surrounding sphere inside the solid."""
    from fractions import Fraction
    P = [[Fraction(str(x)) for x in v] for v in case.vertices]
    q = [Fraction(str(x)) for x in case.query]

    def vol(a, b, c, d):
        u = [b[i] - a[i] for i in range(3)]
        v = [c[i] - a[i] for i in range(3)]
        w = [d[i] - a[i] for i in range(3)]
        return (u[0] * (v[1] * w[2] - v[2] * w[1]) - u[1] * (v[0] * w[2] - v[2] * w[0]) +
                u[2] * (v[0] * w[1] - v[1] * w[0]))
    s = []
    for i in range(4):
        f = [P[j] for j in range(4) if j != i]
        ref = vol(*f, P[i])
        s.append(vol(*f, q) * (1 if ref > 0 else -1))      # >= 0: on the tetrahedron's side of face i
    return all(x >= 0 for x in s) and any(x == 0 for x in s)


def served(case: Case):
    """which of the case's requests the device routes compute (bool per request)."""
    if case.measure != "volume":
        return [False] * len(case.requests)
    if case.dimension == 3:
        if _on_tet_boundary(case):
            return [False] * len(case.requests)
        return [c is not None for c in _tet_columns(case.requests)]
    return [(r.alpha, r.derivative) in _TWO_D for r in case.requests]


def evaluate(case: Case, device="cuda"):
    """float64 values of the case's requests (NaN where not served)."""
    import torch
    out = np.full(len(case.requests), np.nan)
    if case.measure != "volume":
        raise NotImplementedError("fluxbridge surface-measure elements have no device route here")
    P, x, h = case.points, case.x, case.support
    if case.dimension == 3:
        from .mesh3d import Evaluator, Geometry
        cols = _tet_columns(case.requests) if not _on_tet_boundary(case) else [None] * len(case.requests)
        g = Geometry.from_elements([P])
        vals = Evaluator(g, None, kernel=case.kernel, device=device).evaluate(x[None], h)[0]
        for i, c in enumerate(cols):
            if c is not None:
                out[i] = vals[c]
        return out
    from .provider import FusedGroup, FusedWall
    from .scene import Body, Scene, SurfaceRep
    from .shim import ParticleState
    scene = Scene([Body(reps=[SurfaceRep.polygon(P)])], device)
    ps = ParticleState(torch.tensor(x[None], dtype=torch.float64, device=device),
                       torch.tensor([h], dtype=torch.float64, device=device))
    res = FusedWall(scene, ps, h, (FusedGroup(case.kernel),)).res[0]
    host = {k: v[0, 0].cpu().numpy() for k, v in res.items()}
    for i, r in enumerate(case.requests):
        hit = _TWO_D.get((r.alpha, r.derivative))
        if hit is not None:
            name, idx = hit
            out[i] = float(host[name][idx]) if idx else float(host[name])
    return out
