"""BoxRep on the GPU: a box is the exact polygon of its outline, so every output equals the SurfaceRep of the same
outline bit for bit, and the oracle (the reference's algorithm on that polygon) within 1e-10 in units of h.  The
reference's own box scene (tests/scene/test_fused_wall.py:101-112): a rotated, translated box -- an obstacle
('inside') or a tank ('outside') -- and a thin box body, constant support 0.5, the delta+ groups w2, lw2, cone, w2p5;
cone_area against the oracle (1e-11 H^2); signed distances from the box's own closed form."""
import math

import numpy as np
import pytest
import torch

from helpers import DEV
from oracle import cone_area as C
from oracle import edge2d as O
from warpsphboundaries_b200.provider import FusedGroup, FusedWall, WallOutput
from warpsphboundaries_b200.scene import Body, BoxRep, Scene, SurfaceRep
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu

H = 0.5
GROUPS = (FusedGroup("w2"), FusedGroup("lw2"), FusedGroup("cone", (3, 4)), FusedGroup("w2p5", (3, 4)))
OUTS = (WallOutput("lam", 0, "lam"), WallOutput("G", 0, "g0"), WallOutput("Cov", 0, "cov"),
        WallOutput("lap", 1, "lap"), WallOutput("cover", 2, "g0"), WallOutput("tens", 3, "g0"))


def _scene(solid, as_box=True):
    mk = (lambda lo, hi, s="inside": BoxRep(lo, hi, s)) if as_box else \
        (lambda lo, hi, s="inside": SurfaceRep.box(lo, hi, s))
    return Scene([Body(bodyId=0, center=(0.3, -0.2), angle=0.7, reps=[mk((0.1, -0.2), (2.3, 1.1), solid)]),
                  Body(bodyId=1, center=(3.0, 1.0), angle=-0.4, reps=[mk((-0.6, -0.05), (0.6, 0.05))])], DEV)


def _points(n=500, seed=2):
    return np.random.default_rng(seed).uniform(-1.2, 4.2, (n, 2))


def _wall(scene, X):
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), H, dtype=torch.float64, device=DEV))
    return FusedWall(scene, ps, H, GROUPS)


@pytest.mark.parametrize("solid", ["inside", "outside"])
def test_box_equals_its_polygon_and_the_oracle(solid):
    X = _points()
    box, poly = _scene(solid), _scene(solid, as_box=False)
    fb, fp = _wall(box, X), _wall(poly, X)
    gb, gp = fb.evaluate(OUTS), fp.evaluate(OUTS)
    for o in OUTS:
        assert torch.equal(gb[o.name], gp[o.name]), o.name
    for bi, body in enumerate(box.bodies):
        rep = body.reps[0]
        V, E = rep.vertices.cpu().numpy(), rep.edges.cpu().numpy()
        lpos = O.to_local(X, body.center.cpu().numpy(), float(body.angle))
        lo, hi = V.min(0), V.max(0)
        d = np.maximum(lo - lpos, 0) + np.maximum(lpos - hi, 0)
        valid = np.ones(len(X), bool) if rep.background else np.hypot(d[:, 0], d[:, 1]) < H
        ref = O.to_world(O.local_twelve(V, E, rep.background, lpos, np.full(len(X), H), "w2", H, valid),
                         float(body.angle))
        got = {k: fb.res[0][k][bi].cpu().numpy() for k in ("lam", "G", "Cov")}
        assert np.abs(got["lam"] - ref["lam"]).max() <= 1e-10
        assert np.abs(got["G"] - ref["G"]).max() * H <= 1e-10
        assert np.abs(got["Cov"].reshape(-1, 2, 2) - ref["Cov"].reshape(-1, 2, 2)).max() <= 1e-10
    assert float(gb["lam"].abs().max()) > 0.5


@pytest.mark.parametrize("solid", ["inside", "outside"])
def test_box_cone_area_and_signed_distance(solid):
    X = _points()
    scene = _scene(solid)
    fw = _wall(scene, X)
    axes = np.random.default_rng(9).uniform(-1, 1, (len(X), 2))
    orc = [(body.center.cpu().numpy(), float(body.angle),
            [(r.vertices.cpu().numpy(), r.edges.cpu().numpy(), r.background) for r in body.reps])
           for body in scene.bodies]
    for al in (math.pi / 6, math.pi):
        got = fw.cone_area(torch.tensor(axes, device=DEV), al).cpu().numpy()
        assert np.abs(got[0] - C.cone_area_scene(orc, X, axes, al, H)).max() <= 1e-11 * H * H
    d, n, hit, b = scene.signed_distance(torch.tensor(X, device=DEV), want_body=True)
    ref_d = np.full(len(X), np.inf)
    for bi, body in enumerate(scene.bodies):
        dd, _ = body.reps[0].signed(body.toLocal(torch.tensor(X, device=DEV)))
        ref_d = np.minimum(ref_d, dd.cpu().numpy())
    assert np.abs(d.cpu().numpy() - ref_d).max() == 0.0
    assert torch.allclose(n.norm(dim=1), torch.ones(len(X), dtype=torch.float64, device=DEV))
