"""Signed distance, kinematics, multi-body / multi-surface scenes, query kinds, a1g1, the provider's error paths."""
import numpy as np
import pytest
import torch

from oracle import edge2d as O
from tests.helpers import DEV, gpu_outputs, oracle_outputs, scaled_errors
from warpsphboundaries_b200 import workloads
from warpsphboundaries_b200.provider import AnalyticBoundary, FusedWall, FusedGroup, WallOutput
from warpsphboundaries_b200.scene import Body, BodyKinematics, Scene, SurfaceRep
from warpsphboundaries_b200.shim import KernelFunctions, ParticleState

pytestmark = pytest.mark.gpu


def test_signed_distance_matches_brute_force():
    loops = workloads.stars(3, (32, 96), seed=4, box=1.0)
    rep = SurfaceRep.loops(loops)
    scene = Scene([Body(center=(0.05, -0.02), angle=0.3, reps=[rep])], DEV)
    rng = np.random.default_rng(2)
    P = rng.uniform(-0.2, 1.2, size=(5000, 2))
    d, n, hit = scene.signed_distance(torch.tensor(P, device=DEV))
    lp = O.to_local(P, (0.05, -0.02), 0.3)
    V, E = workloads.edges_of(loops)
    a, b = V[E[:, 0]], V[E[:, 1]]
    e = b - a
    t = np.clip((((lp[:, None, :] - a[None]) * e[None]).sum(2)) / (e * e).sum(1)[None], 0, 1)
    c = a[None] + t[..., None] * e[None]
    dist = np.linalg.norm(lp[:, None, :] - c, axis=2)
    dmin = dist.min(1)
    ins = O.indicator(V, E, 0, lp) > 0.5
    ref = np.where(ins, -dmin, dmin)
    assert np.abs(d.cpu().numpy() - ref).max() < 1e-14
    assert bool(hit.all())
    nn = n.cpu().numpy()
    assert np.abs(np.linalg.norm(nn, axis=1) - 1).max() < 1e-12


@pytest.mark.parametrize("support", [0.004, 0.05])
def test_signed_distance_ring_search_equals_the_scan(support):
    """wsb_signed_distance searches rings of grid cells around the point (every edge is listed in the cells it
    crosses): the distance, closest point and edge of every point equal a scan over all edges -- points near and far
    inside the grid (up to ~100 rings at support 0.004) and outside it (the scan)."""
    from warpsphboundaries_b200 import _lib
    from warpsphboundaries_b200.scene import _stream
    loops = workloads.stars(3, (32, 96), seed=4, box=1.0)
    rep = SurfaceRep.loops(loops)
    ns = rep.native(support, DEV)
    rng = np.random.default_rng(5)
    P = np.concatenate([rng.uniform(-0.3, 1.3, size=(6000, 2)), rng.uniform(-3.0, 4.0, size=(500, 2))])
    m = len(P)
    lp = torch.tensor(P, dtype=torch.float64, device=DEV)
    d = torch.empty(m, dtype=torch.float64, device=DEV)
    cp = torch.empty((m, 2), dtype=torch.float64, device=DEV)
    nl = torch.empty((m, 2), dtype=torch.float64, device=DEV)
    ed = torch.empty(m, dtype=torch.int32, device=DEV)
    _lib.check(_lib.lib.wsb_signed_distance(ns.handle, _lib.ptr(lp), m, support, _lib.ptr(d), _lib.ptr(cp),
                                            _lib.ptr(nl), _lib.ptr(ed), _stream()), "wsb_signed_distance")
    V, E = rep.vertices.cpu().numpy(), rep.edges.cpu().numpy().astype(np.int64)
    a, b = V[E[:, 0]], V[E[:, 1]]
    e = b - a
    t = np.clip((((P[:, None, :] - a[None]) * e[None]).sum(2)) / (e * e).sum(1)[None], 0, 1)
    c = a[None] + t[..., None] * e[None]
    dist = np.linalg.norm(P[:, None, :] - c, axis=2)
    k = dist.argmin(1)
    dmin = dist[np.arange(m), k]
    srt = np.sort(dist, axis=1)
    unique = srt[:, 1] - srt[:, 0] > 1e-12
    got = d.cpu().numpy()
    assert np.abs(np.abs(got) - dmin).max() < 1e-14
    assert np.array_equal(ed.cpu().numpy()[unique], k[unique])
    assert np.abs(cp.cpu().numpy()[unique] - c[np.arange(m), k][unique]).max() < 1e-14
    ins = O.indicator(V, E, 0, P) > 0.5
    assert np.array_equal(got < 0, ins & (dmin > 0))


def test_kinematics_bit_exact():
    bodies = [Body(center=(0.3, -0.2), angle=0.4, linearVelocity=(1.0, -0.5), angularVelocity=2.5,
                   linearAcceleration=(0.1, 0.2), angularAcceleration=-0.7),
              Body(center=(-1.0, 2.0), angle=-1.1, linearVelocity=(0.0, 0.25), angularVelocity=-0.3)]
    x = torch.tensor(np.random.default_rng(1).uniform(-2, 2, size=(4000, 2)), dtype=torch.float64, device=DEV)
    kin = BodyKinematics(bodies, x)
    for b, bd in enumerate(bodies):
        c, s = bd.pose._cs()
        C = bd.center.to(DEV)
        d = x - C
        loc = torch.stack([d[:, 0] * c + d[:, 1] * s, d[:, 1] * c - d[:, 0] * s], 1)
        assert torch.equal(kin.local[b], loc)
        assert torch.equal(kin.rel[b], d)
        w = float(bd.angularVelocity)
        v = bd.linearVelocity.to(DEV) + w * torch.stack([-d[:, 1], d[:, 0]], 1)
        assert torch.equal(kin.velocity[b], v)
        al = float(bd.angularAcceleration)
        a = bd.linearAcceleration.to(DEV) + al * torch.stack([-d[:, 1], d[:, 0]], 1) - (w * w) * d
        assert torch.equal(kin.acceleration[b], a)


def test_multi_body_multi_surface_scene():
    """two bodies, the first with two separate surfaces (they add), the second rotated: every body's outputs against
    the oracle's sum over its surfaces."""
    h = 0.03
    loopsA = workloads.stars(2, (40, 80), seed=7, box=1.0)
    loopsB = workloads.stars(1, (60, 60), seed=8, box=1.0)
    loopsC = workloads.stars(2, (30, 50), seed=9, box=1.0)
    repA, repB, repC = SurfaceRep.loops(loopsA), SurfaceRep.loops(loopsB), SurfaceRep.loops(loopsC)
    b0 = Body(center=(0.0, 0.0), angle=0.0, reps=[repA, repB])
    b1 = Body(center=(0.1, 0.05), angle=-0.6, reps=[repC])
    scene = Scene([b0, b1], DEV)
    X = np.random.default_rng(3).uniform(-0.1, 1.1, size=(6000, 2))
    ps = ParticleState(torch.tensor(X, device=DEV), torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    fw = FusedWall(scene, ps, h, (FusedGroup("w2"),))
    got0 = {k: v[0].cpu().numpy() for k, v in fw.res[0].items()}
    got1 = {k: v[1].cpu().numpy() for k, v in fw.res[0].items()}
    # body 0: the broadphase box is the union of both surfaces' boxes
    refA = oracle_outputs(loopsA, X, h, "w2", h)
    refB = oracle_outputs(loopsB, X, h, "w2", h)
    VA, _ = workloads.edges_of(loopsA + loopsB)
    lo, hi = VA.min(0), VA.max(0)
    d = np.maximum(lo - X, 0) + np.maximum(X - hi, 0)
    valid = np.sqrt(d[:, 0] ** 2 + d[:, 1] ** 2) < h
    ref0 = {k: np.where(valid.reshape((-1,) + (1,) * (refA[k].ndim - 1)), refA[k] + refB[k], 0.0) for k in refA}
    assert max(scaled_errors(got0, ref0, h).values()) < 1e-10
    ref1 = oracle_outputs(loopsC, X, h, "w2", h, center=(0.1, 0.05), angle=-0.6)
    assert max(scaled_errors(got1, ref1, h).values()) < 1e-10


def test_query_kinds_and_a1g1():
    loops = workloads.stars(2, (64, 64), seed=12, box=1.0)
    h = 0.02
    rep = SurfaceRep.loops(loops)
    scene = Scene([Body(reps=[rep])], DEV)
    X = np.random.default_rng(4).uniform(0, 1, size=(5000, 2))
    kinds = torch.tensor(np.random.default_rng(5).integers(0, 3, len(X)), device=DEV)
    ps = ParticleState(torch.tensor(X, device=DEV), torch.full((len(X),), h, dtype=torch.float64, device=DEV),
                       kinds=kinds)
    ab = AnalyticBoundary(scene)
    fw = ab.aggregate(ps, h, kernel=KernelFunctions.Wendland2, lean=True)
    lam = fw.out["lam"][0].cpu().numpy()
    fluid = (kinds == 0).cpu().numpy()
    assert np.all(lam[~fluid] == 0.0)
    ref = oracle_outputs(loops, X, h, "w2", h)
    assert np.abs(lam[fluid] - ref["lam"][fluid]).max() < 1e-10
    a1 = torch.tensor(np.random.default_rng(6).normal(size=(1, len(X), 2)), device=DEV)
    A = fw.evaluate([WallOutput("A", 0, "a1g1")], a1=a1)["A"][0].cpu().numpy()
    refA = np.einsum("nd,ndj->nj", a1[0].cpu().numpy(), ref["Cov"])
    assert np.abs(A[fluid] - refA[fluid]).max() < 1e-10


def test_routes_agree_and_error_paths():
    loops = workloads.stars(2, (64, 128), seed=13, box=1.0)
    h = 0.02
    scene = Scene([Body(reps=[SurfaceRep.loops(loops)])], DEV)
    X = np.random.default_rng(7).uniform(0, 1, size=(4000, 2))
    ps = ParticleState(torch.tensor(X, device=DEV), torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    fused = AnalyticBoundary(scene).aggregate(ps, h, kernel=KernelFunctions.Wendland6, lean=True)
    plain = AnalyticBoundary(scene, route="plain").aggregate(ps, h, kernel=KernelFunctions.Wendland6, lean=True)
    for k in ("lam", "G", "Cov"):
        assert (fused.out[k] - plain.out[k]).abs().max().item() < 1e-9
    dp = AnalyticBoundary(scene).aggregate(ps, h, kernel=KernelFunctions.Wendland2)      # the delta+ layout
    assert set(dp.out) == {"lam", "G", "Cov", "cover", "tens"}
    with pytest.raises(NotImplementedError):
        AnalyticBoundary(scene).aggregate(ps, h, kernel=KernelFunctions.Wendland6)          # C2 / C4 only
    ax = torch.tensor(np.random.default_rng(8).normal(size=(len(X), 2)), device=DEV)
    assert torch.equal(fused.cone_area(ax, 0.5), plain.cone_area(ax, 0.5))   # one detector path for both routes
    with pytest.raises(ValueError):
        fused.evaluate([WallOutput("L", 0, "lap")])                  # 'lap' needs an lw2 / lw4 group
    with pytest.raises(NotImplementedError):
        AnalyticBoundary(scene).aggregate(ps, h, kernel=KernelFunctions.Gaussian, lean=True)
    # a conditioned single triangle is served on the fused route (its small / sliver rows by the area quadrature),
    # not on the plain one
    tri = Scene([Body(reps=[SurfaceRep.polygon([(0, 0), (0.01, 0), (0, 0.01)])])], DEV)
    fw_tri = AnalyticBoundary(tri).aggregate(ps, h, kernel=KernelFunctions.Wendland2, lean=True)
    assert torch.isfinite(fw_tri.out["lam"]).all()
    with pytest.raises(NotImplementedError):
        AnalyticBoundary(tri, route="plain").aggregate(ps, h, kernel=KernelFunctions.Wendland2, lean=True)
    # copy_from carries a new position set into the buffers of an existing aggregate
    X2 = X + 0.003
    ps2 = ParticleState(torch.tensor(X2, device=DEV), ps.supports)
    other = AnalyticBoundary(scene).aggregate(ps2, h, kernel=KernelFunctions.Wendland6, lean=True)
    fused.copy_from(other)
    assert torch.equal(fused.out["lam"], other.out["lam"])


def test_particles_on_edges_and_edge_lines():
    """rows exactly on edges (midpoints), on vertices and on the extension of edge lines: the pair orientation and the
    indicator take the same rounded form, so the channels stay within tolerance of the oracle."""
    rng = np.random.default_rng(17)
    loops = [workloads.star(rng, (0.5, 0.5), 0.3, 64, jitter=0.1)]
    V, E = workloads.edges_of(loops)
    a, b = V[E[:, 0]], V[E[:, 1]]
    X = np.concatenate([(a + b) / 2, V, a + 0.3 * (b - a), b + 0.2 * (b - a), a - 0.001 * (b - a)])
    h = 0.02
    scene = Scene([Body(reps=[SurfaceRep.loops(loops)])], DEV)
    for kernel in ("w4", "cubic"):
        got = gpu_outputs(scene, X, h, kernel, h)
        ref = oracle_outputs(loops, X, h, kernel, h)
        err = scaled_errors(got, ref, h)
        assert max(err.values()) < 1e-10, err
