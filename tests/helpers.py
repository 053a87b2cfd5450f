"""Shared helpers of the GPU parity tests: build a scene from loops, run the GPU routes, run the oracle."""
import numpy as np
import torch

from oracle import edge2d as O
from warpsphboundaries_b200 import workloads
from warpsphboundaries_b200.provider import AnalyticBoundary, FusedWall, FusedGroup, WallOutput
from warpsphboundaries_b200.scene import Body, Scene, SurfaceRep
from warpsphboundaries_b200.shim import ParticleState

DEV = "cuda"


def make_scene(loops, center=(0.0, 0.0), angle=0.0, background=0):
    rep = SurfaceRep.loops(loops, solid="inside" if background == 0 else "outside")
    body = Body(center=center, angle=angle, reps=[rep])
    return Scene([body], DEV), rep, body


def gpu_outputs(scene, X, h, kernel, support, route="fused", precision="fp64"):
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), float(h), dtype=torch.float64, device=DEV))
    fw = FusedWall(scene, ps, support, (FusedGroup(kernel),), route=route, precision=precision)
    r = fw.res[0]
    return {k: v[0].cpu().numpy() for k, v in r.items()}


def oracle_outputs(loops, X, h, kernel, support, center=(0.0, 0.0), angle=0.0, background=0):
    V, E = workloads.edges_of(loops)
    lpos = O.to_local(X, center, angle)
    lo, hi = V.min(0), V.max(0)
    d = np.maximum(lo - lpos, 0) + np.maximum(lpos - hi, 0)
    valid = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) < h if background == 0 else np.ones(len(X), bool)
    hh = np.full(len(X), float(h))
    out12 = O.local_twelve(V, E, background, lpos, hh, kernel, support, valid)
    w = O.to_world(out12, angle)
    return {"lam": w["lam"], "G": w["G"], "Cov": w["Cov"], "m1": w["m1"], "m2": w["m2"]}


def scaled_errors(a, b, h):
    """max |a - b| per output in units of h (G * h, m1 / h, m2 / h^2): the channel scale is O(1)."""
    sc = {"lam": 1.0, "G": h, "Cov": 1.0, "m1": 1.0 / h, "m2": 1.0 / (h * h)}
    return {k: float(np.abs((np.asarray(a[k]) - np.asarray(b[k])) * sc[k]).max()) for k in sc}


def small_c2(n_particles=6000, n_polys=6, seed=5, h=0.02):
    """a few stars of the c2 kind and particles concentrated around them (most pairs near walls)."""
    loops = workloads.stars(n_polys, (32, 256), seed, box=1.0, rmin=0.05, rmax=0.3)
    rng = np.random.default_rng(seed + 100)
    X = rng.uniform(-0.1, 1.1, size=(n_particles, 2))
    # near-tangent and endpoint-on-circle particles
    V, E = workloads.edges_of(loops)
    pick = rng.choice(len(E), size=min(200, len(E)), replace=False)
    a, b = V[E[pick, 0]], V[E[pick, 1]]
    d = b - a
    nrm = np.stack([d[:, 1], -d[:, 0]], 1) / np.linalg.norm(d, axis=1, keepdims=True)
    eps = np.array([1e-3, 1e-6, 1e-9])[rng.integers(0, 3, len(pick))]
    X[: len(pick)] = a + rng.uniform(0.1, 0.9, len(pick))[:, None] * d + (h * (1 - eps))[:, None] * nrm
    vs = rng.choice(len(V), size=50, replace=False)
    X[len(pick): len(pick) + 50] = V[vs] + np.array([h, 0.0])
    X[len(pick) + 50: len(pick) + 60] = V[vs[:10]]                     # particles exactly on vertices
    return loops, X, h
