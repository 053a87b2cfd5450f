"""The detector inputs of the delta+ scheme on the GPU: FusedWall.cone_area (wsb_cone_area) and FusedWall.dir_extreme
(wsb_dir_extreme) against the oracle (oracle/cone_area.py, pinned to the reference's closed form).

cone_area: the GPU evaluates the local form (indicator sector minus the chord deficits of the neighbour edges), the
oracle the non-local per-edge form over every edge; both are float64 closed forms of O(H^2) numbers, so they differ by
round-off only: tolerance 1e-11 H^2 (the reference's own tolerance for the same comparison).  dir_extreme: the same
closed form as the oracle's local restatement, tolerance 1e-12; the polar-grid oracle at the reference's 1.5e-2.
Scenes: an L-shape with a reflex corner and a thin bar as two posed bodies, a tank (the outside of a box); constant
and per-query supports; an `allowed` mask; complementary wedges at a million queries.
"""
import math

import numpy as np
import pytest
import torch

from helpers import DEV
from oracle import cone_area as C
from warpsphboundaries_b200.provider import FusedGroup, FusedWall
from warpsphboundaries_b200.scene import Body, Scene, SurfaceRep
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu

L_SHAPE = [(0.0, 0.0), (2.0, 0.0), (2.0, 0.6), (0.7, 0.6), (0.7, 1.8), (0.0, 1.8)]
BAR = [(-0.6, -0.05), (0.6, -0.05), (0.6, 0.05), (-0.6, 0.05)]


def _two_bodies():
    """(Scene, oracle bodies): the L-shape at (0.3, -0.2) turned by 0.7 and the bar at (1.6, 1.9) turned by -0.4."""
    specs = [((0.3, -0.2), 0.7, SurfaceRep.polygon(L_SHAPE)), ((1.6, 1.9), -0.4, SurfaceRep.polygon(BAR))]
    return _scene(specs)


def _tank():
    return _scene([((0.1, 0.2), 0.3, SurfaceRep.box((-1.0, -0.8), (3.1, 2.6), solid="outside"))])


def _scene(specs):
    bodies, orc = [], []
    for center, angle, rep in specs:
        bodies.append(Body(center=center, angle=angle, reps=[rep]))
        orc.append((center, angle, [(rep.vertices.cpu().numpy(), rep.edges.cpu().numpy(), rep.background)]))
    return Scene(bodies, DEV), orc


def _points(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    return rng.uniform(lo, hi, (n, 2)), rng.uniform(-1, 1, (n, 2))


def _wall(scene, X, H, allowed=None):
    n = len(X)
    h = torch.as_tensor(np.broadcast_to(H, (n,)).copy(), dtype=torch.float64, device=DEV)
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV), h)
    al = None if allowed is None else torch.as_tensor(allowed, device=DEV)
    return FusedWall(scene, ps, float(np.max(H)), (FusedGroup("w2"),), allowed=al)


@pytest.mark.parametrize("half_angle", [math.pi / 6, math.pi / 3, 2.0])
def test_cone_area_matches_the_oracle(half_angle):
    H = 0.5
    scene, orc = _two_bodies()
    X, axes = _points(500, (-1.5, -1.5), (3.5, 3.5), 2)
    fw = _wall(scene, X, H)
    got = fw.cone_area(torch.tensor(axes, device=DEV), half_angle)
    assert got.shape == (2, len(X))
    g = got.cpu().numpy()
    for row, al in ((0, half_angle), (1, math.pi)):
        ref = C.cone_area_scene(orc, X, axes, al, H)
        assert np.abs(g[row] - ref).max() <= 1e-11 * H * H, (row, np.abs(g[row] - ref).max())
    assert g[1].max() > 0.1 * H * H and (g[1] == 0).sum() > 10         # near and far queries
    assert torch.equal(got, fw.cone_area(torch.tensor(axes, device=DEV), half_angle))      # deterministic


def test_cone_area_tank_per_query_support_and_mask():
    """a tank (the solid is the outside: rows far inside the fluid see nothing, rows outside the box the whole disk),
    per-query supports in [0.2, 0.5], and an `allowed` mask: a masked-out row adds the whole sector of the background
    solid (fused.py:826-833)."""
    scene, orc = _tank()
    X, axes = _points(600, (-1.8, -1.4), (4.0, 3.6), 3)
    H = np.random.default_rng(4).uniform(0.2, 0.5, len(X))
    allowed = np.ones(len(X), bool)
    allowed[::7] = False
    fw = _wall(scene, X, H, allowed)
    for al in (0.4, 1.3, math.pi):
        g = fw.cone_area(torch.tensor(axes, device=DEV), al).cpu().numpy()
        W = 2 * al if al < math.pi else 2 * math.pi
        for row, a in ((0, al), (1, math.pi)):
            ref = C.cone_area_scene(orc, X, axes, a, H)
            Wr = W if row == 0 else 2 * math.pi
            ref = np.where(allowed, ref, 0.5 * H * H * Wr)
            assert np.abs(g[row] - ref).max() <= 1e-11 * 0.25, (al, row)
        assert (g[1] < 1e-12).sum() > 10 and (np.abs(g[1] - math.pi * H * H) < 1e-12).sum() > 10


def test_cone_area_complementary_wedges_at_a_million_queries():
    """at 2^20 queries (too many for the oracle): the wedges (axis a, half angle al) and (axis -a, half angle
    pi - al) tile the disk, so their areas sum to the full-disk area (1e-11 H^2); 0 <= wedge <= full <= pi H^2;
    half angle pi equals the full-disk row."""
    H = 0.05
    scene, _ = _two_bodies()
    X, axes = _points(1 << 20, (-1.5, -1.5), (3.5, 3.5), 6)
    fw = _wall(scene, X, H)
    ax = torch.tensor(axes, device=DEV)
    a1 = fw.cone_area(ax, 1.1)
    a2 = fw.cone_area(-ax, math.pi - 1.1)
    tol = 1e-11 * H * H
    assert float((a1[0] + a2[0] - a1[1]).abs().max()) <= tol
    assert torch.equal(a1[1], a2[1])
    assert float(a1[0].min()) >= -tol and float((a1[0] - a1[1]).max()) <= tol
    assert float(a1[1].max()) <= math.pi * H * H + tol
    full = fw.cone_area(ax, math.pi)
    assert torch.equal(full[0], full[1]) and torch.equal(full[1], a1[1])
    assert int((a1[1] > 0).sum()) > 1000


def test_cone_area_rejects_bad_arguments():
    scene, _ = _two_bodies()
    X, axes = _points(8, (0, 0), (1, 1), 1)
    fw = _wall(scene, X, 0.5)
    ax = torch.tensor(axes, device=DEV)
    for bad in (-0.1, float("nan"), float("inf")):
        with pytest.raises(ValueError):
            fw.cone_area(ax, bad)
    with pytest.raises(ValueError):
        fw.cone_area(ax[:4], 0.5)


@pytest.mark.parametrize("kind", ["two_bodies", "tank"])
def test_dir_extreme_matches_the_oracle(kind):
    H = 0.5
    scene, orc = _two_bodies() if kind == "two_bodies" else _tank()
    X, _ = _points(300 if kind == "two_bodies" else 200, (-1.5, -1.5), (3.8, 3.5), 7)
    B = len(orc)
    vec = np.random.default_rng(5).normal(size=(B, len(X), 2))
    vec[0, 3] = 0.0
    fw = _wall(scene, X, H)
    got = fw.dir_extreme(torch.tensor(vec, device=DEV))
    assert got.shape == (B, len(X))
    g = got.cpu().numpy()
    for b, (center, angle, reps) in enumerate(orc):
        lp = C.to_local(X, center, angle)
        lv = C.axes_to_local(vec[b], angle)
        V, E, bg = reps[0]
        ref = C.dir_extreme_local(lp, lv, H, V, E, bg)
        assert np.abs(g[b] - ref).max() <= 1e-12, (b, np.abs(g[b] - ref).max())
        sub = slice(0, 40)
        polar = C.dir_extreme_polar(lp[sub], lv[sub], H, V, E, bg, nr=150)
        assert (g[b][sub] >= polar - 1e-9).all() and np.abs(g[b][sub] - polar).max() <= 1.5e-2
    assert g[0, 3] == 0.0
    assert (g > 0.5).sum() > 5 and (g == 0).sum() > 5
    assert torch.equal(got, fw.dir_extreme(torch.tensor(vec, device=DEV)))    # deterministic


def test_dir_extreme_mask_on_a_tank():
    """rows outside `allowed` see the background solid everywhere: 1 for a non-zero vector, 0 for a zero one."""
    scene, orc = _tank()
    X, _ = _points(256, (-1.5, -1.2), (3.8, 3.3), 8)
    allowed = np.ones(len(X), bool)
    allowed[::5] = False
    vec = np.random.default_rng(9).normal(size=(1, len(X), 2))
    vec[0, 5] = 0.0                                   # masked out and zero
    fw = _wall(scene, X, 0.4, allowed)
    g = fw.dir_extreme(torch.tensor(vec, device=DEV)).cpu().numpy()[0]
    center, angle, reps = orc[0]
    V, E, bg = reps[0]
    ref = C.dir_extreme_local(C.to_local(X, center, angle), C.axes_to_local(vec[0], angle), 0.4, V, E, bg,
                              allowed=allowed)
    assert np.abs(g - ref).max() <= 1e-12
    assert g[5] == 0.0 and (g[~allowed] == 1.0).sum() == (~allowed).sum() - 1
