"""ImplicitRep and SdfRep bodies on the fused wall path: each is integrated as its exact polygon form (a cavity disk
its area-preserving polygon with edges <= h/16, a sampled distance its marching-squares contour or its fallback),
so FusedWall on the implicit body equals FusedWall on that polygon bit for bit, and the oracle on it within 1e-10.
The contour of a sampled disk agrees with the analytic disk polygon to the contour error (O(spacing^2 kappa):
2e-3 of the scale at spacing h/16, the reference's bound for the same comparison).  Bodies without an exact form
(a half plane) are refused."""
import numpy as np
import pytest
import torch

from helpers import DEV
from oracle import edge2d as O
from warpsphboundaries_b200.implicit import DiskBody, HalfPlaneBody
from warpsphboundaries_b200.provider import FusedGroup, FusedWall, WallOutput
from warpsphboundaries_b200.scene import Body, ImplicitRep, Scene, SdfRep, SurfaceRep
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu

H = 0.3
OUTS = (WallOutput("lam", 0, "lam"), WallOutput("G", 0, "g0"), WallOutput("Cov", 0, "cov"))


def _queries(n=400, seed=3, lo=-1.3, hi=1.3):
    return np.random.default_rng(seed).uniform(lo, hi, (n, 2))


def _wall(scene, X, groups=(FusedGroup("w2"),)):
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), H, dtype=torch.float64, device=DEV))
    return FusedWall(scene, ps, H, groups)


def test_cavity_disk_is_its_polygon():
    cav = ImplicitRep(DiskBody((0.1, -0.05), 1.1, solid="outside"))
    body = Body(center=(0.2, 0.1), angle=0.4, reps=[cav])
    scene = Scene([body], DEV)
    X = _queries()
    got = _wall(scene, X).evaluate(OUTS)
    poly = cav.lowered(H, DEV)
    assert len(poly.edges) == max(24, int(np.ceil(2 * np.pi * 1.1 / (H / 16))))
    ref_scene = Scene([Body(center=(0.2, 0.1), angle=0.4, reps=[poly])], DEV)
    ref = _wall(ref_scene, X).evaluate(OUTS)
    for o in OUTS:
        assert torch.equal(got[o.name], ref[o.name]), o.name
    V, E = poly.vertices.cpu().numpy(), poly.edges.cpu().numpy()
    lpos = O.to_local(X, (0.2, 0.1), 0.4)
    orc = O.to_world(O.local_twelve(V, E, 1, lpos, np.full(len(X), H), "w2", H, np.ones(len(X), bool)), 0.4)
    assert np.abs(got["lam"][0].cpu().numpy() - orc["lam"]).max() <= 1e-10
    assert np.abs(got["G"][0].cpu().numpy() - orc["G"]).max() * H <= 1e-10
    lam = got["lam"][0].cpu().numpy()
    r = np.hypot(*(lpos - np.array([0.1, -0.05])).T)
    assert np.allclose(lam[r > 1.1 + H], 1.0, atol=1e-12) and np.allclose(lam[r < 1.1 - H], 0.0, atol=1e-12)
    # the signed distance of the body is the disk's closed form
    d, n, hit = scene.signed_distance(torch.tensor(X, device=DEV))
    assert np.allclose(d.cpu().numpy(), 1.1 - r, atol=1e-12) and bool(hit.all())


@pytest.mark.parametrize("solid", ["inside", "outside"])
def test_sampled_disk_contour(solid):
    R, c = 0.7, (0.05, -0.02)
    sgn = 1.0 if solid == "inside" else -1.0
    sdf = SdfRep.fromFunction(lambda p: sgn * ((p - torch.tensor(c, dtype=torch.float64)).norm(dim=1) - R),
                              (-1.2, -1.2), (1.2, 1.2), H / 16)
    scene = Scene([Body(center=(0.3, 0.2), angle=-0.6, reps=[sdf])], DEV)
    X = _queries(seed=4)
    got = _wall(scene, X).evaluate(OUTS)
    contour = sdf.lowered(H, DEV)
    assert contour.background == (0 if solid == "inside" else 1)
    ref = _wall(Scene([Body(center=(0.3, 0.2), angle=-0.6, reps=[contour])], DEV), X).evaluate(OUTS)
    for o in OUTS:
        assert torch.equal(got[o.name], ref[o.name]), o.name
    disk = SurfaceRep.regularPolygon(c, R, 2048, solid=solid)
    exact = _wall(Scene([Body(center=(0.3, 0.2), angle=-0.6, reps=[disk])], DEV), X).evaluate(OUTS)
    for o in OUTS:
        scale = float(exact[o.name].abs().max())
        assert float((got[o.name] - exact[o.name]).abs().max()) <= 2e-3 * max(scale, 1.0), o.name
    assert float(got["lam"].max()) > 0.9


def test_sdf_fallback_is_used():
    fb = SurfaceRep.box((-0.4, -0.3), (0.5, 0.2))
    sdf = SdfRep(np.ones((4, 4)), (0, 0), 0.1, fallback=fb)        # the samples are never contoured
    X = _queries(seed=5)
    a = _wall(Scene([Body(reps=[sdf])], DEV), X).evaluate(OUTS)
    b = _wall(Scene([Body(reps=[SurfaceRep.box((-0.4, -0.3), (0.5, 0.2))])], DEV), X).evaluate(OUTS)
    for o in OUTS:
        assert torch.equal(a[o.name], b[o.name]), o.name


def test_bodies_without_an_exact_form_are_refused():
    scene = Scene([Body(reps=[ImplicitRep(HalfPlaneBody((0.0, 0.0), (0.0, 1.0)))])], DEV)
    assert not FusedWall.supported(scene)
    with pytest.raises(NotImplementedError):
        _wall(scene, _queries(n=8))
