"""The disk element on the GPU (wsb_disk_aggregate through FusedWall): solid disks (a DiskArrayRep fibre bundle, a
solid ImplicitRep disk) integrated exactly along their circles.

Parity: against the oracle (oracle/disk.py: the radial integrals by adaptive quadrature, pinned to area-preserving
polygons) within 1e-10 in units of the support, on a posed bundle of disks with radii from 0.05 h to 5 h, particles
inside, near and far and near-tangent ones (|D - R| = h eps, eps down to 1e-9), for kernels with one to three
blocks; at 2^20 particles against the polygon route on area-preserving 4096-gons of the same disks (an independent
GPU path whose geometric error is O(n^-4) ~ 1e-13): 1e-9.  The detector inputs of disks: the cone area against the
oracle's angular integration (1e-12 H^2), the direction extreme against its closed form (1e-12) and the polar grid
(1.5e-2).  Refusals: tensile groups."""
import math

import numpy as np
import pytest
import torch

from helpers import DEV
from oracle import disk as Dk
from oracle import edge2d as O
from warpsphboundaries_b200.implicit import DiskBody
from warpsphboundaries_b200.provider import FusedGroup, FusedWall
from warpsphboundaries_b200.scene import Body, DiskArrayRep, ImplicitRep, Scene, SurfaceRep
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu

H = 0.1
CENTER, ANGLE = (0.4, -0.3), 0.5
NAMES = ("lam", "G", "Cov", "m1", "m2")


def _bundle():
    """twelve non-overlapping disks in the body frame, radii 0.05 h .. 5 h."""
    rng = np.random.default_rng(21)
    C, R = [], []
    radii = [0.005, 0.01, 0.02, 0.05, 0.08, 0.1, 0.15, 0.2, 0.3, 0.5, 0.04, 0.12]
    while len(C) < len(radii):
        r = radii[len(C)]
        c = rng.uniform(-1.5, 1.5, 2)
        if all(np.hypot(*(c - c2)) > r + r2 + 0.01 for c2, r2 in zip(C, R)):
            C.append(c)
            R.append(r)
    return np.array(C), np.array(R)


def _wall(scene, X, kernels, h=H):
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    return FusedWall(scene, ps, h, tuple(FusedGroup(k) for k in kernels))


def _world(X):
    c, s = math.cos(ANGLE), math.sin(ANGLE)
    return X @ np.array([[c, s], [-s, c]]) + np.array(CENTER)


def _queries(C, R, n_random=60, seed=4):
    """body-frame particles: random ones, and near-tangent ones at distance R + h eps from a circle."""
    rng = np.random.default_rng(seed)
    pts = [rng.uniform(-1.6, 1.6, (n_random, 2))]
    for k, (c, r) in enumerate(zip(C, R)):
        for eps in (1e-3, -1e-6, 1e-9, -0.5):
            a = rng.uniform(0, 2 * np.pi)
            d = max(r + H * eps, 0.0)
            pts.append((c + d * np.array([np.cos(a), np.sin(a)]))[None])
        pts.append(c[None])                                   # the centre itself
    return np.concatenate(pts)


def _compare(fw, gi, lp, C, R, kernel):
    ref = O.to_world(Dk.disks_local_twelve(C, R, lp, np.full(len(lp), H), kernel), ANGLE)
    got = {k: fw.res[gi][k][0].cpu().numpy() for k in NAMES}
    scale = {"lam": 1.0, "G": H, "Cov": 1.0, "m1": 1 / H, "m2": 1 / H ** 2}
    for k in NAMES:
        g = got[k].reshape(len(lp), -1)
        r = ref[k].reshape(len(lp), -1)
        err = np.abs(g - r).max() * scale[k]
        assert err <= 1e-10, (kernel, k, err)


@pytest.mark.parametrize("kernels", [("cubic", "w4"), ("w2", "quartic")])
def test_disk_bundle_matches_the_oracle(kernels):
    C, R = _bundle()
    scene = Scene([Body(center=CENTER, angle=ANGLE, reps=[DiskArrayRep(C, R)])], DEV)
    lp = _queries(C, R)
    fw = _wall(scene, _world(lp), kernels)
    for gi, k in enumerate(kernels):
        _compare(fw, gi, lp, C, R, k)
    lam = fw.res[0]["lam"][0].cpu().numpy()
    assert lam.max() > 0.99 and (lam == 0).sum() > 5


def test_solid_implicit_disk_is_a_one_disk_set():
    X = _world(np.random.default_rng(6).uniform(-0.8, 0.8, (300, 2)))
    a = _wall(Scene([Body(center=CENTER, angle=ANGLE, reps=[ImplicitRep(DiskBody((0.1, 0.05), 0.42))])], DEV), X,
              ("w2", "cone", "lw2"))
    b = _wall(Scene([Body(center=CENTER, angle=ANGLE, reps=[DiskArrayRep([[0.1, 0.05]], [0.42])])], DEV), X,
              ("w2", "cone", "lw2"))
    for gi in range(3):
        for k in NAMES:
            assert torch.equal(a.res[gi][k], b.res[gi][k]), (gi, k)


def test_disks_match_fine_polygons_at_a_million_particles():
    C, R = _bundle()
    n = 1 << 20
    X = _world(np.random.default_rng(8).uniform(-1.7, 1.7, (n, 2)))
    disks = _wall(Scene([Body(center=CENTER, angle=ANGLE, reps=[DiskArrayRep(C, R)])], DEV), X, ("w4",))
    polys = [SurfaceRep.polygon(Dk.area_preserving_polygon(c, r, 4096)) for c, r in zip(C, R)]
    poly = _wall(Scene([Body(center=CENTER, angle=ANGLE, reps=polys)], DEV), X, ("w4",))
    scale = {"lam": 1.0, "G": H, "Cov": 1.0, "m1": 1 / H, "m2": 1 / H ** 2}
    for k in NAMES:
        err = float((disks.res[0][k] - poly.res[0][k]).abs().max()) * scale[k]
        assert err <= 1e-9, (k, err)
    lam = disks.res[0]["lam"][0]
    assert float(lam.min()) >= -1e-12 and float(lam.max()) <= 1 + 1e-12 and int((lam > 0.5).sum()) > 1000


def test_disk_refusals():
    scene = Scene([Body(reps=[DiskArrayRep([[0.0, 0.0]], [0.3])])], DEV)
    X = np.random.default_rng(1).uniform(-0.5, 0.5, (16, 2))
    with pytest.raises(NotImplementedError):
        _wall(scene, X, ("w2p5",))
    fw = _wall(scene, X, ("w2",))
    with pytest.raises(ValueError):
        fw.cone_area(torch.zeros((16, 2), dtype=torch.float64, device=DEV), -0.5)


@pytest.mark.parametrize("half_angle", [math.pi / 6, 2.0])
def test_disk_cone_area_matches_the_numerical_integral(half_angle):
    """the closed-form areas of solid cap disk(x, H) cap wedge (per disk: the swept-area antiderivatives) against the
    oracle's adaptive angular integration of the ray lengths: 1e-12 H^2 (the reference's own test: 1e-7 H^2 against a
    200 000-angle midpoint rule); row 1 is the full disk; particles on a circle included."""
    C, R = _bundle()
    scene = Scene([Body(center=CENTER, angle=ANGLE, reps=[DiskArrayRep(C, R)])], DEV)
    lp = _queries(C, R, n_random=40)
    lp = np.concatenate([lp, C[:3] + R[:3, None] * np.array([[1.0, 0.0], [0.0, -1.0], [0.6, 0.8]])])   # on circles
    rng = np.random.default_rng(2)
    ax_local = rng.normal(size=(len(lp), 2))
    c, s = math.cos(ANGLE), math.sin(ANGLE)
    ax_world = ax_local @ np.array([[c, s], [-s, c]])
    fw = _wall(scene, _world(lp), ("w2",))
    got = fw.cone_area(torch.tensor(ax_world, device=DEV), half_angle).cpu().numpy()
    ref = Dk.disks_cone_area(lp, ax_local, half_angle, H, C, R)
    assert np.abs(got - ref).max() <= 1e-12 * H * H, np.abs(got - ref).max()
    assert got[1].max() > 0.9 * math.pi * H * H and (got[1] == 0).sum() > 5
    assert np.all(got[0] <= got[1] + 1e-15)


def test_disk_dir_extreme():
    C, R = _bundle()
    scene = Scene([Body(center=CENTER, angle=ANGLE, reps=[DiskArrayRep(C, R)])], DEV)
    lp = _queries(C, R, n_random=40)
    rng = np.random.default_rng(3)
    v_local = rng.normal(size=(len(lp), 2))
    v_local[5] = 0.0
    c, s = math.cos(ANGLE), math.sin(ANGLE)
    v_world = v_local @ np.array([[c, s], [-s, c]])
    fw = _wall(scene, _world(lp), ("w2",))
    got = fw.dir_extreme(torch.tensor(v_world[None], device=DEV)).cpu().numpy()[0]
    ref = Dk.disks_dir_extreme(lp, v_local, H, C, R)
    assert np.abs(got - ref).max() <= 1e-12
    polar = Dk.disks_dir_extreme_polar(lp, v_local, H, C, R)
    # a disk that only just enters the support leaves a sliver thinner than the grid's radial step: skip those rows
    gap = np.hypot(lp[:, None, 0] - C[None, :, 0], lp[:, None, 1] - C[None, :, 1]) - R[None] - H
    ok = ~((gap < 0) & (gap > -0.02 * H)).any(1)
    assert (got >= polar - 1e-9).all() and np.abs(got - polar)[ok].max() <= 1.5e-2
    assert got[5] == 0.0 and (got == 1.0).sum() > 5 and (got == 0.0).sum() > 5
