"""Closed triangle surfaces (3-D) on the GPU through wsb_mesh_channels: against the reference's mpmath values, the
float64 restatement of the reference's reduction (the oracle), and exact inside tests."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import mesh3d as M3

pytestmark = pytest.mark.gpu
G = json.loads((Path(__file__).parent / "golden" / "mesh3d_golden.json").read_text())
DEV = torch.device("cuda")


def _run(V, Fc, Q, h, kernel, smax=None):
    from warpsphboundaries_b200.mesh3d import ClosedMesh
    Q = np.asarray(Q, float).reshape(-1, 3)
    hh = np.broadcast_to(np.asarray(h, float), (len(Q),)).copy()
    m = ClosedMesh(V, Fc, float(hh.max()) if smax is None else smax, DEV)
    pos = torch.tensor(Q, dtype=torch.float64, device=DEV)
    sup = torch.tensor(hh, dtype=torch.float64, device=DEV)
    ind = torch.empty(len(Q), dtype=torch.int32, device=DEV)
    out = m.channels(pos, sup, kernel, inside=ind)
    torch.cuda.synchronize()
    return out.cpu().numpy(), ind.cpu().numpy()


def test_reference_fixture():
    worst = 0.0
    for c in G["cases"]:
        m = G["meshes"][c["mesh"]]
        got, _ = _run(m["vertices"], m["faces"], [c["query"]], c["h"], c["kernel"])
        ref = np.array([float(v) for v in c["values"]])
        e = np.abs(got[0] - ref).max() / (1 + np.abs(ref).max())
        worst = max(worst, e)
        assert e < 1e-10, (c["mesh"], c["kernel"], c["query"], c["h"], e, np.argmax(np.abs(got[0] - ref)))
    print("worst scaled error", worst)


def test_many_queries_one_launch_against_oracle():
    """a jittered 320-face icosphere; queries near the surface, inside, outside, close to faces, edges and vertices,
    several supports, in one launch; every row against the oracle."""
    from warpsphboundaries_b200 import workloads as W
    V, Fc = W.icosphere(2, 0.6, 0.05, seed=3)
    rng = np.random.default_rng(7)
    d = rng.normal(size=(48, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    Q = list(d * rng.uniform(0.45, 0.7, (48, 1)))
    Q += list(V[rng.choice(len(V), 6)] * (1 + rng.choice([-1e-7, 1e-7], (6, 1))))                # near vertices
    mids = (V[Fc[:6, 0]] + V[Fc[:6, 1]]) / 2
    Q += list(mids * 1.001)                                                                     # near edges
    cen = V[Fc[6:12]].mean(1)
    nrm = np.cross(V[Fc[6:12, 1]] - V[Fc[6:12, 0]], V[Fc[6:12, 2]] - V[Fc[6:12, 0]])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    Q += list(cen + 1e-9 * nrm) + list(cen - 1e-6 * nrm)                                       # near face planes
    Q = np.array(Q)
    h = rng.uniform(0.08, 0.2, len(Q))
    for kernel in ("cubic", "w6"):
        got, ind = _run(V, Fc, Q, h, kernel, smax=0.2)
        for k in range(len(Q)):
            ref = M3.channels(V, Fc, Q[k], h[k], kernel)
            e = np.abs(got[k] - ref).max() / (1 + np.abs(ref).max())
            assert e < 1e-8, (kernel, k, Q[k], h[k], e)


def test_inside_against_winding_number():
    """the vertical-ray parity equals the solid-angle winding number on random points and on points whose vertical
    lines pass exactly through the box's vertices and edges (the tie rules)."""
    from warpsphboundaries_b200 import workloads as W
    from warpsphboundaries_b200.mesh3d import ClosedMesh
    cases = [W.icosphere(2, 0.6, 0.05, seed=3), W.box_mesh((-0.3, -0.25, -0.2), (0.35, 0.3, 0.25))]
    m = G["meshes"]["notched"]
    cases.append((np.array(m["vertices"]), np.array(m["faces"])))
    rng = np.random.default_rng(9)
    for V, Fc in cases:
        lo, hi = V.min(0) - 0.1, V.max(0) + 0.1
        Q = rng.uniform(lo, hi, (4000, 3))
        xs, ys = np.unique(V[:, 0]), np.unique(V[:, 1])
        grid = np.array([[x, y, z] for x in xs[:6] for y in ys[:6] for z in rng.uniform(lo[2], hi[2], 3)])
        Q = np.concatenate([Q, grid])
        cm = ClosedMesh(V, Fc, 0.1, DEV)
        ind = cm.inside(torch.tensor(Q, dtype=torch.float64, device=DEV)).cpu().numpy()
        a, b, c = (V[Fc[:, k]][None] - Q[:, None] for k in range(3))
        la, lb, lc = (np.linalg.norm(t, axis=2) for t in (a, b, c))
        det = np.einsum("qfi,qfi->qf", a, np.cross(b, c))
        den = la * lb * lc + np.einsum("qfi,qfi->qf", a, b) * lc + np.einsum("qfi,qfi->qf", b, c) * la + \
            np.einsum("qfi,qfi->qf", c, a) * lb
        raw = (2 * np.arctan2(det, den)).sum(1) / (4 * np.pi)
        wind = np.rint(raw).astype(int)
        # points on the surface (in a face's plane and within its box): the inside test is a convention there, and
        # so is the solid-angle sum
        nrm = np.cross(V[Fc[:, 1]] - V[Fc[:, 0]], V[Fc[:, 2]] - V[Fc[:, 0]])
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        inplane = np.abs(np.einsum("fi,qfi->qf", nrm, -a)) < 1e-12
        flo, fhi = V[Fc].min(1) - 1e-12, V[Fc].max(1) + 1e-12
        inbox = ((Q[:, None] >= flo[None]) & (Q[:, None] <= fhi[None])).all(2)
        on_surface = (inplane & inbox).any(1) | (np.abs(raw - wind) > 0.05)
        ok = (ind == wind) | on_surface
        assert ok.all(), (Q[~ok][:5], ind[~ok][:5], wind[~ok][:5])


def test_whole_support_inside_and_outside_constants():
    from warpsphboundaries_b200 import workloads as W
    V, Fc = W.box_mesh((-1, -1, -1), (1, 1, 1))
    Q = np.array([[0.0, 0.0, 0.0], [0.3, -0.2, 0.1], [3.0, 0.0, 0.0]])
    for kernel in ("cubic", "w2", "w4", "w6"):
        got, ind = _run(V, Fc, Q, 0.25, kernel)
        assert ind.tolist() == [1, 1, 0]
        ref = M3.channels(V, Fc, Q[1], 0.25, kernel)
        assert np.abs(got[1] - ref).max() < 1e-10 * (1 + np.abs(ref).max())
        assert abs(got[0, 0] - 1.0) < 1e-14 and np.abs(got[2]).max() == 0.0
        assert np.allclose(got[0, 13:22].reshape(3, 3), np.eye(3), atol=1e-14)    # d/dx_j (y_i W) = delta_ij


def test_invalid_rows_and_determinism():
    from warpsphboundaries_b200.mesh3d import ClosedMesh
    from warpsphboundaries_b200 import workloads as W
    V, Fc = W.icosphere(1, 0.6)
    m = ClosedMesh(V, Fc, 0.1, DEV)
    pos = torch.tensor([[0.0, 0.0, 0.5], [0.0, 0.0, 0.5], [0.0, 0.0, 0.5]], dtype=torch.float64, device=DEV)
    sup = torch.tensor([0.1, 0.2, -1.0], dtype=torch.float64, device=DEV)
    ind = torch.empty(3, dtype=torch.int32, device=DEV)
    a = m.channels(pos, sup, "w4", inside=ind).clone()
    b = m.channels(pos, sup, "w4").clone()
    torch.cuda.synchronize()
    assert ind.tolist() == [1, -1, -1]
    assert torch.isfinite(a[0]).all() and torch.isnan(a[1:]).all()
    assert torch.equal(a[0], b[0])


def test_evaluator_subset_and_physical_units():
    from warpsphboundaries_b200.mesh3d import Evaluator, Geometry
    from warpsphboundaries_b200.radial import Request
    c = next(c for c in G["cases"] if c["mesh"] == "icosahedron" and c["kernel"] == "w6")
    m = G["meshes"]["icosahedron"]
    g = Geometry.closed_surface(m["vertices"], m["faces"])
    reqs = [Request((0, 0, 0), (2, 1)), Request((1, 0, 1)), Request((0, 0, 0))]
    got = Evaluator(g, reqs, kernel="w6").evaluate([c["query"]], c["h"])[0]
    ref = np.array([float(v) for v in c["values"]])
    want = np.array([ref[26], ref[6], ref[0]])
    assert np.abs(got - want).max() < 1e-10 * (1 + np.abs(want).max())


def test_tetrahedral_mesh_equals_its_surface():
    """a tetrahedral mesh (fluxbridge Geometry(elements, 3, 'volume')) is served through the boundary of its union:
    the fan of a jittered icosphere from its centre equals the icosphere's closed surface, and a cube of five
    tetrahedra the oracle's box, within 1e-12 (1 + |v|); the reference's tetrahedral method names are accepted."""
    from warpsphboundaries_b200 import workloads as W
    from warpsphboundaries_b200.mesh3d import Evaluator, Geometry
    V, Fc = W.icosphere(2, 0.6, 0.03, seed=5)
    fan = Geometry.from_elements([np.stack([np.zeros(3), V[a], V[b], V[c]]) for a, b, c in Fc])
    rng = np.random.default_rng(11)
    Q = rng.uniform(-0.8, 0.8, (400, 3))
    h = rng.uniform(0.05, 0.2, len(Q))
    a = Evaluator(fan, kernel="w4", method="tet_quadrature").evaluate(Q, h)
    b = Evaluator(Geometry.closed_surface(V, Fc), kernel="w4").evaluate(Q, h)
    a, b = np.asarray(a), np.asarray(b)
    assert np.abs(a - b).max() / (1 + np.abs(b).max()) < 1e-12
    C = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float) * 0.5 - 0.25
    i = lambda x, y, z: x * 4 + y * 2 + z
    tets = [[i(0, 0, 0), i(1, 0, 0), i(0, 1, 0), i(0, 0, 1)], [i(1, 1, 0), i(1, 0, 0), i(0, 1, 0), i(1, 1, 1)],
            [i(1, 0, 1), i(1, 0, 0), i(1, 1, 1), i(0, 0, 1)], [i(0, 1, 1), i(0, 1, 0), i(0, 0, 1), i(1, 1, 1)],
            [i(1, 0, 0), i(0, 1, 0), i(0, 0, 1), i(1, 1, 1)]]
    cube = Geometry.from_elements([C[t] for t in tets])
    Qc = rng.uniform(-0.4, 0.4, (24, 3))
    hc = np.full(len(Qc), 0.15)
    Evaluator(cube, kernel="w2", method="conditioned_boundary").evaluate(Qc, hc)      # the reference's method name
    got, _ = _run(cube.vertices, cube.faces, Qc, hc, "w2", smax=0.15)
    for k in range(len(Qc)):
        ref = M3.channels(cube.vertices, cube.faces, Qc[k], hc[k], "w2")
        assert np.abs(got[k] - ref).max() / (1 + np.abs(ref).max()) < 1e-8


def test_queries_outside_the_face_grid():
    """queries beyond the surface's box along each axis, from within the support (0.1) to several cells out (0.3 /
    0.6: at and past the grid's one-cell margin; 2.0: settled by the first row pass as outside with no face in reach):
    all outside, channels equal to the oracle (zero beyond the support)."""
    from warpsphboundaries_b200 import workloads as W
    V, Fc = W.box_mesh((-1, -1, -1), (1, 1, 1))
    Q = []
    for axis in range(3):
        for sign in (-1.0, 1.0):
            for d in (0.1, 0.3, 0.6, 2.0):
                q = np.array([0.13, -0.07, 0.21])
                q[axis] = sign * (1.0 + d)
                Q.append(q)
    Q = np.array(Q)
    got, ind = _run(V, Fc, Q, 0.25, "w4")
    assert (ind == 0).all()
    for k, q in enumerate(Q):
        ref = M3.channels(V, Fc, q, 0.25, "w4")
        assert np.abs(got[k] - ref).max() < 1e-10 * (1 + np.abs(ref).max()), k
    far = np.abs(Q).max(axis=1) > 1.25
    assert np.abs(got[far]).max() == 0.0 and np.abs(got[~far]).max() > 0.0
