"""Generate the golden fixtures of tests/golden/ from the reference implementation.

Run in a container where the reference source tree is available (it is read,
never modified):

    python tests/golden/make_golden.py /path/to/warpSPHBoundaries-checkout

Writes
  edge2d_golden_subset.json   the reference's 40-digit golden vectors (tests/fixtures/edge2d_golden.json):
                              element cases with value, grad, moments |alpha| <= 2 and moment_grad |alpha| <= 2
  np2d_c1.npz                 the regular 256-gon scene (radius 0.45, centre (0.5, 0.5), w4, h = 0.05): a seeded
                              subset of particles with the twelve channels from the reference's numpy path
                              (edge/np2d.py, whole polygon) for cubic, w2, w4, w6
  torch2d_grad.npz            gradients of lam and the moments with respect to particle positions and polygon
                              vertices from torch autograd through the reference's edge/torch2d.py (star polygon, w4)
  radial_golden.json          solid half-spaces and spheres, 3-D: the nine radial invariants and the 28 baseline
                              channels of the reference's 70-digit fixtures (tests/fixtures/fluxbridge-radial-v1.json,
                              and the baseline requests of tests/fixtures/fluxbridge-sphere-v1.json)
  triangle_golden.json        conditioned single triangles (2-D): the reference's adversarial triangle cases (tiny, needle
                              angles, slivers; validation/adversarial.py polygon_cases) at its deterministic probes, with
                              the twelve channels (w4) of its 70-digit analytic reference (precision_polygon_reference)
  cone_area_golden.json       the area of solid cap disk(x, H) cap wedge from the reference's vectorised per-edge closed form
                              (scene/cone_area.py): an L-shape, a thin bar and a tank (background), H 0.5 and 0.23,
                              half angles pi/6, pi/3, 2 and pi
  sdf_contour_golden.json     the zero contours of sampled distances from the reference's marching squares (scene.py):
                              a disk, a tank, two merging disks (saddles), a ring
  mesh3d_golden.json          closed triangle surfaces, 3-D: the 28 baseline channels (value moments |alpha| <= 2,
                              kernel-gradient moments |alpha| <= 1, kernel Hessian) from the reference's exact
                              face-to-edge reductions in mpmath (mesh3d/reference.py ClosedSurface), 40 digits, for an
                              icosahedron, a jittered once-subdivided icosphere, a box and a notched (non-convex) block

The reference package is imported with a stub parent package because its
`__init__` needs the GPU stack (warp, warpSPHCore), which the CPU modules used
here do not.
"""
import importlib
import math
import json
import sys
import types
from fractions import Fraction as F
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
KERNELS = ["cubic", "w2", "w4", "w6"]


def load_reference(root):
    pkg = types.ModuleType("warpSPHBoundaries")
    pkg.__path__ = [str(Path(root) / "src" / "warpSPHBoundaries")]
    sys.modules["warpSPHBoundaries"] = pkg
    np2d = importlib.import_module("warpSPHBoundaries.edge.np2d")
    torch2d = importlib.import_module("warpSPHBoundaries.edge.torch2d")
    return np2d, torch2d


def c1_scene(n_particles=4096, seed=0):
    """regular 256-gon of radius 0.45 around (0.5, 0.5) (vertices at angles 2 pi k / 256) and particles uniform in
    [0.05, 0.95]^2 rejected outside the polygon (seeded)."""
    k = np.arange(256)
    P = np.stack([0.5 + 0.45 * np.cos(2 * np.pi * k / 256), 0.5 + 0.45 * np.sin(2 * np.pi * k / 256)], 1)
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < n_particles:
        c = rng.uniform(0.05, 0.95, size=(4 * n_particles, 2))
        r2 = ((c - 0.5) ** 2).sum(1)
        # inside the polygon: the inscribed-circle test is not enough near edges; use the exact crossing rule
        inside = _inside_polygon(c, P)
        pts.extend(c[inside][: n_particles - len(pts)])
    return P, np.asarray(pts[:n_particles])


def _inside_polygon(x, P):
    a = P
    b = np.roll(P, -1, 0)
    cnt = np.zeros(len(x), dtype=np.int64)
    for i in range(len(P)):
        ay, by = a[i, 1], b[i, 1]
        straddle = (ay > x[:, 1]) != (by > x[:, 1])
        xc = a[i, 0] + (x[:, 1] - ay) * (b[i, 0] - a[i, 0]) / np.where(by == ay, 1, by - ay)
        cnt += straddle & (x[:, 0] < xc)
    return cnt % 2 == 1


def golden_subset(root):
    d = json.loads((Path(root) / "tests" / "fixtures" / "edge2d_golden.json").read_text())
    out = {"meta": {"source": "tests/fixtures/edge2d_golden.json of the reference", "format": d["meta"]["format"],
                    "digits": d["meta"]["digits"], "conventions": d["meta"]["conventions"]}, "cases": []}
    moms = ["1,0", "0,1", "2,0", "1,1", "0,2"]
    grads = ["0,0", "1,0", "0,1", "2,0", "1,1", "0,2"]
    for c in d["cases"]:
        if c["kind"] != "element":
            continue
        rec = {"id": c["id"], "tags": c["tags"], "polygon": c["polygon"], "x": c["x"], "h": c["h"], "where": c["where"], "kernels": {}}
        for k, e in c["kernels"].items():
            rec["kernels"][k] = {"value": e["value"], "grad": e["grad"], "moments": {m: e["moments"][m] for m in moms},
                                 "moment_grad": {g: e["moment_grad"][g] for g in grads}}
        out["cases"].append(rec)
    (HERE / "edge2d_golden_subset.json").write_text(json.dumps(out, indent=1))
    print("edge2d_golden_subset.json:", len(out["cases"]), "cases")


def np2d_c1(np2d, n_sub=384, seed=0):
    P, X = c1_scene()
    h = 0.05
    rng = np.random.default_rng(seed + 1)
    # the subset mixes near-wall particles (the interesting ones) and interior ones
    d_wall = 0.45 * np.cos(np.pi / 256) - np.sqrt(((X - 0.5) ** 2).sum(1))
    near = np.flatnonzero(d_wall < h)
    far = np.flatnonzero(d_wall >= h)
    sub = np.sort(np.concatenate([rng.choice(near, n_sub * 3 // 4, replace=False), rng.choice(far, n_sub // 4, replace=False)]))
    xs = X[sub]
    K = len(P)
    out = {}
    for k in KERNELS:
        V = (P[None, :, :] - xs[:, None, :]) / h          # normalised coordinates: the reference functions at h = 1
        Z = np.zeros((len(xs), 2))
        ch = np.zeros((len(xs), 12))
        ch[:, 0] = np2d.moment(V, Z, k, (0, 0), 1.0)
        ch[:, 1] = np2d.moment(V, Z, k, (1, 0), 1.0) * h
        ch[:, 2] = np2d.moment(V, Z, k, (0, 1), 1.0) * h
        g0 = np2d.grad_moment(V, Z, k, (0, 0), 1.0)
        g10 = np2d.grad_moment(V, Z, k, (1, 0), 1.0)
        g01 = np2d.grad_moment(V, Z, k, (0, 1), 1.0)
        ch[:, 3:5] = g0 / h
        ch[:, 5:7] = g10
        ch[:, 7:9] = g01
        ch[:, 9] = np2d.moment(V, Z, k, (2, 0), 1.0) * h * h
        ch[:, 10] = np2d.moment(V, Z, k, (1, 1), 1.0) * h * h
        ch[:, 11] = np2d.moment(V, Z, k, (0, 2), 1.0) * h * h
        out[k] = ch
        print("np2d", k, "done")
    np.savez_compressed(HERE / "np2d_c1.npz", polygon=P, particles=X, subset=sub, h=h, **{f"ch_{k}": v for k, v in out.items()})


def star(n, rbar, center, jitter, rng):
    t = 2 * np.pi * np.arange(n) / n
    r = rbar * (1 + rng.uniform(-jitter, jitter, n))
    return np.stack([center[0] + r * np.cos(t), center[1] + r * np.sin(t)], 1)


def torch2d_grads(torch2d, seed=0, n_pts=96):
    import torch
    rng = np.random.default_rng(seed + 7)
    P = star(128, 0.1, (0.5, 0.5), 0.15, rng)                    # ccw star polygon, 128 vertices
    h = 0.02
    r = np.sqrt(((P - 0.5) ** 2).sum(1))
    ang = rng.uniform(0, 2 * np.pi, n_pts)
    rad = np.interp(ang, 2 * np.pi * np.arange(129) / 128, np.concatenate([r, r[:1]])) + rng.uniform(-0.8 * h, 0.8 * h, n_pts)
    X = np.stack([0.5 + rad * np.cos(ang), 0.5 + rad * np.sin(ang)], 1)
    res = {}
    for al in [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]:
        Vt = torch.tensor(np.broadcast_to(P, (n_pts, 128, 2)).copy(), dtype=torch.float64, requires_grad=True)
        Xt = torch.tensor(X, dtype=torch.float64, requires_grad=True)
        m = torch2d.moment(Vt, Xt, "w4", al, h)
        m.sum().backward()
        key = f"{al[0]}{al[1]}"
        res[f"m_{key}"] = m.detach().numpy()
        res[f"dx_{key}"] = Xt.grad.numpy()
        res[f"dv_{key}"] = Vt.grad.numpy()
        print("torch2d", al, "done")
    np.savez_compressed(HERE / "torch2d_grad.npz", polygon=P, particles=X, h=h, **res)


def torch2d_c4(torch2d, n_pts=256):
    """the gradient scene at its full size (workloads.c4: 2^18 particles in [0, 4]^2, 16 star polygons of 128
    vertices, h = 0.02, w4): for 256 seeded particles within 0.95 h of an edge, each moment m_alpha (|alpha| <= 2)
    summed over the 16 polygons by the reference's torch2d.moment (whole polygons), its autograd gradient per particle
    and the vertex gradient of sum_i m_alpha(x_i) per polygon."""
    import torch
    sys.path.insert(0, str(HERE.parent.parent))
    from warpsphboundaries_b200 import workloads
    loops, X, h = workloads.c4()
    V, E = workloads.edges_of(loops)
    A, B = V[E[:, 0]], V[E[:, 1]]
    rng = np.random.default_rng(404)
    rows = []
    for i in rng.permutation(len(X)):
        d = B - A
        t = np.clip(((X[i] - A) * d).sum(1) / (d * d).sum(1), 0.0, 1.0)
        if np.linalg.norm(X[i] - (A + t[:, None] * d), axis=1).min() < 0.95 * h:
            rows.append(int(i))
            if len(rows) == n_pts:
                break
    rows = np.array(rows)
    P = np.stack(loops)                                                    # [16, 128, 2]
    res = {}
    for al in [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]:
        Xt = torch.tensor(X[rows], dtype=torch.float64, requires_grad=True)
        Vts = [torch.tensor(np.broadcast_to(L, (len(rows), 128, 2)).copy(), dtype=torch.float64, requires_grad=True)
               for L in P]
        m = sum(torch2d.moment(Vt, Xt, "w4", al, h) for Vt in Vts)
        m.sum().backward()
        key = f"{al[0]}{al[1]}"
        res[f"m_{key}"] = m.detach().numpy()
        res[f"dx_{key}"] = Xt.grad.numpy()
        res[f"dv_{key}"] = np.stack([Vt.grad.numpy().sum(0) for Vt in Vts])
        print("torch2d c4", al, "done")
    np.savez_compressed(HERE / "torch2d_c4.npz", rows=rows, particles=X[rows], h=h, **res)


def fluxbridge_subset(root):
    """the single-element cases of the reference's fluxbridge-v1.json (schema 1) -- 2-D triangles and 3-D tetrahedra
    at five queries, four kernels, with the baseline requests plus two high-degree ones, and the surface triangles --
    in the same schema, for the interchange-format tests (the full-degree coverage cases are left out for size)."""
    src = json.loads((Path(root) / "tests" / "fixtures" / "fluxbridge-v1.json").read_text())
    cases = [c for c in src["cases"] if len(c["requests"]) <= 32]
    out = {"schema": src["schema"], "dps": src["dps"], "cases": cases}
    (HERE / "fluxbridge_v1_subset.json").write_text(json.dumps(out, indent=2) + "\n")
    print("fluxbridge_v1_subset.json:", len(cases), "of", len(src["cases"]), "cases")


def radial_golden(root):
    fx = Path(root) / "tests" / "fixtures"
    rad = json.loads((fx / "fluxbridge-radial-v1.json").read_text())
    out = {"meta": {"source": "tests/fixtures/fluxbridge-radial-v1.json and fluxbridge-sphere-v1.json of the reference",
                    "dps": rad["dps"], "support": "1 (distances and radii in units of the support)",
                    "invariants": "lam, m1_axial, m2_tangent, m2_axial, G_axial, g1_tangent, g1_axial, H_tangent, "
                                  "H_axial", "values": "the 28 baseline channels in request order"},
           "radial": [], "sphere": []}
    for c in rad["cases"]:
        out["radial"].append({k: c[k] for k in ("kind", "kernel", "distance", "radius", "normal", "invariants",
                                                "values")})
    sph = json.loads((fx / "fluxbridge-sphere-v1.json").read_text())
    for c in sph["cases"]:
        vals = {}
        for req, v in zip(c["requests"], c["values"]):
            if sum(req["alpha"]) + len(req["derivative"]) <= 2 and (len(req["derivative"]) == 0 or
                                                                   sum(req["alpha"]) + len(req["derivative"]) <= 2):
                vals[json.dumps([req["alpha"], req["derivative"]])] = v
        out["sphere"].append({"label": c["label"], "kernel": c["kernel"], "distance": c["distance"],
                              "radius": c["radius"], "normal": c["normal"], "values": vals})
    (HERE / "radial_golden.json").write_text(json.dumps(out, indent=1))
    print("radial_golden.json:", len(out["radial"]), "radial cases,", len(out["sphere"]), "sphere cases")


def _icosahedron(radius):
    t = (1 + 5 ** 0.5) / 2
    V = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
                  [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], float)
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]
    return V / np.linalg.norm(V[0]) * radius, F


def _subdivide(V, F):
    V = [tuple(v) for v in V]
    mid = {}

    def m(a, b):
        key = (min(a, b), max(a, b))
        if key not in mid:
            mid[key] = len(V)
            V.append(tuple((np.array(V[a]) + np.array(V[b])) / 2))
        return mid[key]
    out = []
    for a, b, c in F:
        ab, bc, ca = m(a, b), m(b, c), m(c, a)
        out += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
    return np.array(V), out


def _box_faces(lo, hi):
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    V = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0], [x0, y0, z1], [x1, y0, z1], [x1, y1, z1],
                  [x0, y1, z1]], float)
    F = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (1, 2, 6), (1, 6, 5), (2, 3, 7), (2, 7, 6),
         (3, 0, 4), (3, 4, 7)]
    return V, F


def _notched_block():
    """an L-shaped prism (non-convex): the square [0,0.8]^2 minus [0.4,0.8]x[0.4,0.8], extruded over z in [0, 0.5]."""
    P = [(0, 0), (0.8, 0), (0.8, 0.4), (0.4, 0.4), (0.4, 0.8), (0, 0.8)]
    n = len(P)
    V = [(x, y, 0.0) for x, y in P] + [(x, y, 0.5) for x, y in P]
    F = [(0, 3, 1), (1, 3, 2), (0, 5, 3), (3, 5, 4)]                 # bottom (outward -z), fan of the L
    F += [(n + a, n + c, n + b) for a, b, c in F]                      # top, reversed
    for i in range(n):
        j = (i + 1) % n
        F += [(i, j, n + j), (i, n + j, n + i)]
    return np.array(V), F


def mesh3d_golden(root, dps=40):
    ref = importlib.import_module("warpSPHBoundaries.mesh3d.reference")
    import mpmath as mp
    rng = np.random.default_rng(31)
    meshes = {}
    meshes["icosahedron"] = _icosahedron(0.6)
    V2, F2 = _subdivide(*_icosahedron(0.6))
    V2 = V2 / np.linalg.norm(V2, axis=1, keepdims=True) * 0.6 * (1 + 0.05 * rng.uniform(-1, 1, (len(V2), 1)))
    meshes["icosphere1_jitter"] = (V2, F2)
    meshes["cube"] = _box_faces((-0.3, -0.25, -0.2), (0.35, 0.3, 0.25))
    meshes["notched"] = _notched_block()
    base = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1), (0, 0, 2)]
    g_alpha = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1)]
    cases = []
    queries = {
        "icosahedron": [((0.1, 0.2, 0.35), 0.3), ((0.0, 0.0, 0.0), 0.2), ((0.05, -0.1, 0.62), 0.25),
                        ((0.3, 0.3, 0.3), 0.7), ((0.55, 0.0, 0.1), 0.15)],
        "icosphere1_jitter": [((0.1, -0.2, 0.4), 0.3), ((0.4, 0.35, -0.1), 0.2), ((-0.2, 0.1, -0.63), 0.15)],
        "cube": [((0.0, 0.0, 0.0), 0.15), ((0.3, 0.25, 0.2), 0.2), ((0.33, 0.0, 0.0), 0.1), ((0.5, 0.4, 0.3), 0.3),
                 ((0.02, -0.03, 0.1), 0.6)],
        "notched": [((0.5, 0.5, 0.25), 0.2), ((0.38, 0.42, 0.1), 0.15), ((0.2, 0.2, 0.45), 0.3),
                    ((0.6, 0.2, 0.25), 0.12)],
    }
    for name, (V, F) in meshes.items():
        for q, h in queries[name]:
            for k in KERNELS:
                with mp.workdps(dps):
                    cs = ref.ClosedSurface([tuple(float(x) for x in v) for v in V], F, q)
                    vals = [cs.moment(k, a, h) for a in base]
                    for a in g_alpha:
                        vals.extend(cs.kernel_gradient(k, a, h))
                    H = cs.kernel_hessian(k, (0, 0, 0), h)
                    vals.extend(H[i][j] for i in range(3) for j in range(i, 3))
                    cases.append({"mesh": name, "kernel": k, "h": h, "query": list(q),
                                  "values": [mp.nstr(v, 30) for v in vals]})
            print("mesh3d", name, q, "done", flush=True)
    out = {"meta": {"source": "mesh3d/reference.py ClosedSurface of the reference (mpmath, %d digits)" % dps,
                    "values": "28 baseline channels in the request order of the 3-D contract: value moments "
                              "alpha in (000,100,010,001,200,110,101,020,011,002), kernel-gradient moments "
                              "(alpha, j) for alpha in (000,100,010,001), j = 0..2, Hessian (00,01,02,11,12,22); "
                              "physical units (y = vertex - query, support h)"},
           "meshes": {n: {"vertices": [[float(x) for x in v] for v in V], "faces": [list(map(int, f)) for f in F]}
                      for n, (V, F) in meshes.items()},
           "cases": cases}
    (HERE / "mesh3d_golden.json").write_text(json.dumps(out, indent=1))
    print("mesh3d_golden.json:", len(cases), "cases")


def triangle_golden(root, names=("triangle-size-1e-09", "triangle-size-0.01", "triangle-size-1e-05",
                                 "triangle-angle-0.1", "triangle-angle-179", "sliver-1e-07", "sliver-0.001")):
    adv = importlib.import_module("warpSPHBoundaries.validation.adversarial")
    out = {"meta": {"source": "validation/adversarial.py of the reference: polygon_cases, probes, "
                              "precision_polygon_reference (70 digits), kernel w4, support 1",
                    "channels": "m00 m10 m01 m20 m11 m02 Gx Gy g1xx g1xy g1yx g1yy"}, "cases": []}
    for c in adv.polygon_cases():
        if c.name not in names:
            continue
        pts = c.probes()
        target = adv.precision_polygon_reference(c.vertices, pts, "w4")
        out["cases"].append({"name": c.name, "vertices": c.vertices.tolist(), "points": pts.tolist(),
                             "target": [[repr(float(v)) for v in row] for row in target]})
        print("triangle", c.name, len(pts), "probes", flush=True)
    (HERE / "triangle_golden.json").write_text(json.dumps(out, indent=1))


WALL_KERNELS = ["cone", "lw2", "lw4"]
POWERED_KERNELS = ["w2p5", "w4p5"]


def wall_kernel_golden(root, dps=40):
    """the wall-operator kernels -- cone (the kernel of the free-surface cover vector) and lw2 / lw4 (W'/r of the wall
    Laplacian, registered by scene/viscosity.py:_register) -- on the element cases of the 2-D golden subset: value,
    moments |alpha| <= 2, gradient and moment gradients by the reference's own mpmath edge reduction
    (edge/core.py:219-262), 40 digits; with the reference's registered normalisation and block coefficients."""
    import mpmath as mp
    core = importlib.import_module("warpSPHBoundaries.edge.core")
    kernels = importlib.import_module("warpSPHBoundaries.edge.kernels")
    visc = importlib.import_module("warpSPHBoundaries.scene.viscosity")
    for fam in ("w2", "w4"):
        visc._register(fam)
        # the tensile kernel W^5, registered as scene/tensile.py:_register does (its warpbc import needs warp)
        kernels.KERNELS[fam + "p5"] = kernels._from_terms(fam + "p5", kernels.power_terms(5, fam))
    sub = json.loads((HERE / "edge2d_golden_subset.json").read_text())
    moms = [(1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]
    grads = [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]
    s = lambda v: mp.nstr(v, 36)
    out = {"meta": {"source": "edge/core.py value / gradient / moment / moment_gradient of the reference, 40 digits, "
                              "on the element cases of edge2d_golden_subset.json", "kernels": WALL_KERNELS},
           "kernels": {k: {"c2_pi": str(kernels.KERNELS[k].c2_pi),
                           "blocks": [[str(b.R), [str(c) for c in b.coeffs]] for b in kernels.KERNELS[k].blocks]}
                       for k in WALL_KERNELS + POWERED_KERNELS},
           "cases": []}
    for c in sub["cases"]:
        P, x, h = c["polygon"], c["x"], c["h"]
        rec = {"id": c["id"], "kernels": {}}
        for k in WALL_KERNELS:
            e = {"value": s(core.value(P, x, k, h=h, dps=dps)),
                 "grad": [s(g) for g in core.gradient(P, x, k, h=h, dps=dps)],
                 "moments": {f"{a},{b}": s(core.moment(P, x, k, (a, b), h=h, dps=dps)) for a, b in moms},
                 "moment_grad": {f"{a},{b}": [s(g) for g in core.moment_gradient(P, x, k, (a, b), h=h, dps=dps)]
                                 for a, b in grads}}
            rec["kernels"][k] = e
        # the tensile kernels: the gradient only (their group's G channels)
        rec["powered_grad"] = {k: [s(g) for g in core.gradient(P, x, k, h=h, dps=dps)] for k in POWERED_KERNELS}
        out["cases"].append(rec)
    (HERE / "edge2d_wall_kernels.json").write_text(json.dumps(out, indent=1))
    print("edge2d_wall_kernels.json:", len(out["cases"]), "cases")


def _cone_reps():
    """three body-frame polygons (solid on the left): an L-shape with a reflex corner, a thin bar and a tank (the
    clockwise outline of a box, background 1: the solid is the outside)."""
    L = np.array([[0.0, 0.0], [2.0, 0.0], [2.0, 0.6], [0.7, 0.6], [0.7, 1.8], [0.0, 1.8]])
    bar = np.array([[-0.6, -0.05], [0.6, -0.05], [0.6, 0.05], [-0.6, 0.05]])
    tank = np.array([[-1.0, -0.8], [-1.0, 2.6], [3.1, 2.6], [3.1, -0.8]])
    out = []
    for P, bg in ((L, 0), (bar, 0), (tank, 1)):
        n = len(P)
        out.append((P, np.stack([np.arange(n), (np.arange(n) + 1) % n], 1), bg))
    return out


def cone_area_golden(root, n=160, seed=11):
    """cone_area_golden.json: the reference's own vectorised closed form (scene/cone_area.py `cone_area`, float64
    torch on the CPU) for the three polygons of _cone_reps, seeded points inside / near / far and random axes, at
    H = 0.5 and H = 0.23 and half angles pi/6, pi/3, 2, pi (the full disk)."""
    import importlib.util
    import torch
    spec = importlib.util.spec_from_file_location(
        "ref_cone_area", str(Path(root) / "src" / "warpSPHBoundaries" / "scene" / "cone_area.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    rng = np.random.default_rng(seed)
    reps, cases = [], []
    for ri, (V, E, bg) in enumerate(_cone_reps()):
        lo, hi = V.min(0) - 0.6, V.max(0) + 0.6
        pts = rng.uniform(lo, hi, (n, 2))
        axes = rng.normal(size=(n, 2))
        reps.append({"vertices": V.tolist(), "edges": E.tolist(), "background": bg, "points": pts.tolist(),
                     "axes": axes.tolist()})
        for H in (0.5, 0.23):
            for al in (math.pi / 6, math.pi / 3, 2.0, math.pi):
                val = mod.cone_area(torch.tensor(pts), torch.tensor(axes), al, H, torch.tensor(V), torch.tensor(E), bg)
                cases.append({"rep": ri, "H": H, "half_angle": al, "value": val.numpy().tolist()})
    with open(HERE / "cone_area_golden.json", "w") as fh:
        json.dump({"source": "src/warpSPHBoundaries/scene/cone_area.py cone_area (float64, CPU)", "reps": reps,
                   "cases": cases}, fh)


def sdf_grids():
    """(name, d [nx, ny], origin, spacing) of the sampled distances of the contour fixture: a disk obstacle, a tank
    (the outside of a rounded box), two merging disks (saddle cells) and a ring (a hole in the solid)."""
    sp = 0.05
    xs = -1.2 + sp * np.arange(49)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    disk = np.hypot(X - 0.03, Y + 0.02) - 0.61
    qx, qy = np.abs(X) - 0.7, np.abs(Y) - 0.5
    box = np.hypot(np.maximum(qx, 0), np.maximum(qy, 0)) + np.minimum(np.maximum(qx, qy), 0) - 0.2
    tank = -box
    two = np.minimum(np.hypot(X + 0.36, Y) - 0.4, np.hypot(X - 0.36, Y - 0.03) - 0.37)
    r = np.hypot(X, Y)
    ring = np.maximum(r - 0.8, 0.35 - r)
    out = [(n, d, (-1.2, -1.2), sp) for n, d in (("disk", disk), ("tank", tank), ("two_disks", two), ("ring", ring))]
    for name, a in (("saddle_joined", -0.9), ("saddle_split", -0.3)):      # a diagonal solid pair: the cell mean decides
        d = np.ones((4, 4))
        d[1, 1], d[2, 2], d[1, 2], d[2, 1] = a, a, 0.5, 0.45
        out.append((name, d, (0.0, 0.0), 0.1))
    return out


def sdf_contour_golden(root):
    """sdf_contour_golden.json: the reference's marching squares (scene/scene.py _marching_squares, read from the
    source and run on its own with a stand-in SurfaceRep that records vertices / edges / background) on sdf_grids."""
    import ast
    src = (Path(root) / "src" / "warpSPHBoundaries" / "scene" / "scene.py").read_text()
    node = next(n for n in ast.parse(src).body if isinstance(n, ast.FunctionDef) and n.name == "_marching_squares")

    class Recorder:
        def __init__(self, vertices, edges, background=0):
            self.vertices, self.edges, self.background = vertices, edges, background

    ns = {"np": np, "SurfaceRep": Recorder}
    exec(compile(ast.Module(body=[node], type_ignores=[]), "scene.py", "exec"), ns)
    cases = []
    for name, d, origin, sp in sdf_grids():
        rep = ns["_marching_squares"](d, np.asarray(origin), sp)
        cases.append({"name": name, "vertices": np.asarray(rep.vertices).tolist(),
                      "edges": np.asarray(rep.edges).tolist(), "background": int(rep.background)})
    with open(HERE / "sdf_contour_golden.json", "w") as fh:
        json.dump({"source": "src/warpSPHBoundaries/scene/scene.py _marching_squares", "cases": cases}, fh)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the warpSPHBoundaries source tree>")
    root = sys.argv[1]
    np2d, torch2d = load_reference(root)
    golden_subset(root)
    np2d_c1(np2d)
    torch2d_grads(torch2d)
    torch2d_c4(torch2d)
    fluxbridge_subset(root)
    radial_golden(root)
    mesh3d_golden(root)
    triangle_golden(root)
    wall_kernel_golden(root)
    cone_area_golden(root)
    sdf_contour_golden(root)
