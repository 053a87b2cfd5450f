"""The Scene route to the twelve moments (SurfaceRep.topology / moments, Scene.adjacency / precompute / restrict,
AnalyticBoundary.aggregate(fixedAdjacency=False)) through wsb_pair_channels, against the oracle and the fused route.

Tolerances: the oracle within 1e-10 in units of h (channels O(1)); the fused route within 1e-12 (the same closed form,
summed in another order)."""
import numpy as np
import pytest
import torch

from oracle import edge2d as O
from tests.helpers import DEV, small_c2
from warpsphboundaries_b200 import workloads
from warpsphboundaries_b200.provider import AnalyticBoundary, FusedGroup, FusedWall
from warpsphboundaries_b200.scene import Body, BoxRep, Scene, SurfaceRep
from warpsphboundaries_b200.shim import KernelFunctions, OperationProperties, ParticleState

pytestmark = pytest.mark.gpu
KF = {"cubic": KernelFunctions.CubicSpline, "w2": KernelFunctions.Wendland2, "w4": KernelFunctions.Wendland4,
      "w6": KernelFunctions.Wendland6}


def _oracle_world(rep, body, X, h, kernel):
    """world outputs of one representation of a posed body at world points X (oracle, physical units)."""
    V = rep.vertices.detach().cpu().numpy()
    E = rep.edges.cpu().numpy().astype(np.int64)
    ang = float(body.angle)
    lpos = O.to_local(X, body.center.cpu().numpy(), ang)
    lo, hi = V.min(0), V.max(0)
    d = np.maximum(lo - lpos, 0) + np.maximum(lpos - hi, 0)
    valid = np.hypot(d[:, 0], d[:, 1]) < h if rep.background == 0 else np.ones(len(X), bool)
    out = O.local_twelve(V, E, rep.background, lpos, np.full(len(X), h), kernel, h, valid)
    return O.to_world(out, ang)


def _scene():
    loops, X, h = small_c2(n_particles=4000, n_polys=4, seed=11)
    r0 = SurfaceRep.loops(loops[:3])
    r1 = BoxRep((0.35, 0.35), (0.6, 0.55))
    r2 = SurfaceRep.loops(loops[3:])
    b0 = Body(center=(0.0, 0.0), angle=0.0, reps=[r0, r1])
    b1 = Body(center=(0.05, -0.03), angle=0.7, reps=[r2])
    return Scene([b0, b1], DEV), X, h


def test_topology_pair_lists_equal_the_oracle():
    """SurfaceRep.topology (scene.py:374-382): the (query, edge) pairs with segment distance < support, rows ascending
    and a row's edges in cell-list order, equal to the oracle's neighbour slots flattened, near-tangent rows
    included."""
    loops, X, h = small_c2()
    rep = SurfaceRep.loops(loops)
    lpos = torch.tensor(X, dtype=torch.float64, device=DEV)
    lsup = torch.full((len(X),), h, dtype=torch.float64, device=DEV)
    topo = rep.topology(lpos, lsup)
    V, E = workloads.edges_of(loops)
    slots = O.fixed_slots(V, E, O.build_cell_list(V, E, h), X, np.full(len(X), h))
    qi = np.concatenate([np.full(len(s), r) for r, s in enumerate(slots)])
    e = np.concatenate(slots)
    assert np.array_equal(topo.qi.cpu().numpy(), qi) and np.array_equal(topo.e.cpu().numpy(), e)
    assert len(e) > 1000


@pytest.mark.parametrize("kernel", ["cubic", "w4", "w6"])
def test_precompute_matches_the_oracle(kernel):
    """Scene.adjacency + Scene.precompute (scene.py:1400-1433) on two posed bodies (three polygon loops and a box on
    one, a rotated star on the other): per body the world-frame moments of every representation, summed, against the
    oracle."""
    scene, X, h = _scene()
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    props = OperationProperties(kernel=KF[kernel])
    adj = scene.adjacency(ps, props)
    pm = scene.precompute(adj, props)
    assert pm.kernel == kernel and pm.numQueries == len(X)
    for bi, (ent, body) in enumerate(zip(pm.entries, scene.bodies)):
        got = {k: np.zeros(s) for k, s in (("lam", (len(X),)), ("G", (len(X), 2)), ("Cov", (len(X), 2, 2)),
                                            ("m1", (len(X), 2)), ("m2", (len(X), 2, 2)))}
        for m in ent["surface"]:
            q = m.q.cpu().numpy()
            for k, v in (("lam", m.lam), ("G", m.g0), ("Cov", m.g1), ("m1", m.m1), ("m2", m.m2)):
                np.add.at(got[k], q, v.cpu().numpy())
            assert int(m.quadrature_status.abs().sum()) == 0
        ref = None
        for rep in body.reps:
            r = _oracle_world(rep, body, X, h, kernel)
            ref = r if ref is None else {k: ref[k] + r[k] for k in ref}
        sc = {"lam": 1.0, "G": h, "Cov": 1.0, "m1": 1.0 / h, "m2": 1.0 / h ** 2}
        for k in sc:
            assert np.abs((got[k] - ref[k]) * sc[k]).max() < 1e-10, (bi, k)
    assert pm.stats["pairs"] > 1000


def test_channel_subsets_zero_the_rest():
    """an explicit channel subset zeroes the channels not asked for (scene.py:384-416); m2 is None without 9..11."""
    scene, X, h = _scene()
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    props = OperationProperties(kernel=KernelFunctions.Wendland4)
    adj = scene.adjacency(ps, props)
    full = scene.precompute(adj, props)
    part = scene.precompute(adj, props, channels=(0, 3, 4))
    assert part.channels == frozenset({0, 3, 4})
    for ef, ep in zip(full.entries, part.entries):
        for mf, mp in zip(ef["surface"], ep["surface"]):
            assert torch.equal(mf.lam, mp.lam) and torch.equal(mf.g0, mp.g0)
            assert float(mp.m1.abs().max()) == 0.0 and float(mp.g1.abs().max()) == 0.0 and mp.m2 is None
    with pytest.raises(ValueError):
        scene.precompute(adj, props, channels=(12,))


def test_restricted_adjacency_gives_the_same_rows():
    """SceneAdjacency.restrict (scene.py:1090-1108): the adjacency of a subset of the queries, renumbered, gives the
    same moments for those queries as the full adjacency."""
    scene, X, h = _scene()
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    props = OperationProperties(kernel=KernelFunctions.Wendland2)
    adj = scene.adjacency(ps, props)
    idx = torch.tensor(np.sort(np.random.default_rng(3).choice(len(X), 900, replace=False)), device=DEV)
    sub = scene.precompute(adj.restrict(idx), props)
    full = scene.precompute(adj, props)
    for ef, es in zip(full.entries, sub.entries):
        for mf, ms in zip(ef["surface"], es["surface"]):
            lf = torch.zeros(len(X), dtype=torch.float64, device=DEV).index_add_(0, mf.q.long(), mf.lam)
            ls = torch.zeros(len(idx), dtype=torch.float64, device=DEV).index_add_(0, ms.q.long(), ms.lam)
            assert float((lf[idx] - ls).abs().max()) < 1e-14


@pytest.mark.parametrize("lean", [True, False])
def test_aggregate_without_fixed_adjacency_equals_the_fused_route(lean):
    """AnalyticBoundary.aggregate(fixedAdjacency=False) (provider.py:89-92: Scene.adjacency, the oracle path) gives
    the fused route's outputs: lam, G, Cov (and m1, m2 through evaluate) of the scheme kernel and, without `lean`, the
    cover (cone), Laplacian (lw2) and tensile (w2p5, G only) outputs."""
    scene, X, h = _scene()
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    ab = AnalyticBoundary(scene)
    a = ab.aggregate(ps, h, kernel=KernelFunctions.Wendland2, laplacian=True, lean=lean, fixedAdjacency=True)
    b = ab.aggregate(ps, h, kernel=KernelFunctions.Wendland2, laplacian=True, lean=lean, fixedAdjacency=False)
    assert a.route == "fused" and b.route == "scene"
    assert set(a.out) == set(b.out)
    for k in a.out:
        d = float((a.out[k] - b.out[k]).abs().max())
        scale = h if k in ("G", "cover", "tens") else 1.0
        assert d * scale < 1e-12, (k, d)
    for k in ("m1", "m2"):
        d = float((a.res[0][k] - b.res[0][k]).abs().max())
        assert d / h ** (1 if k == "m1" else 2) < 1e-12, (k, d)


def test_conditioned_triangle_on_the_scene_route():
    """a single sliver triangle (the conditioned area quadrature, warptriangle.py:126-201): SurfaceRep.moments takes
    the quadrature rows like the fused route, with their status and estimate."""
    tri = np.array([[0.3, 0.3], [0.3 + 0.02, 0.3 + 1e-6], [0.3 + 0.01, 0.3 + 2e-6]])
    rep = SurfaceRep.polygon(tri, conditioned=True)
    scene = Scene([Body(reps=[rep])], DEV)
    rng = np.random.default_rng(4)
    X = np.array([0.31, 0.3]) + rng.normal(scale=0.01, size=(300, 2))
    h = 0.02
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    fw = FusedWall(scene, ps, h, (FusedGroup("w4"),))
    pm = scene.pairMoments(ps, OperationProperties(kernel=KernelFunctions.Wendland4))
    m = pm.entries[0]["surface"][0]
    q = m.q.long()
    assert int((m.quadrature_status != 0).sum()) > 0
    assert float((m.lam - fw.res[0]["lam"][0][q]).abs().max()) < 1e-12
    assert float((m.g0 - fw.res[0]["G"][0][q]).abs().max()) * h < 1e-12
    st = fw.qstatus[(0, 0, 0)][q]
    assert torch.equal(st, m.quadrature_status)
