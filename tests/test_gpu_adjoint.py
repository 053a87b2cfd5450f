"""The adjoint kernel (wsb_aggregate_backward behind BoundaryMoments) against the oracle's analytic gradients, the
reference's torch autograd gradients (tests/golden/torch2d_grad.npz) and central finite differences of the forward.

Tolerances: analytic / autograd comparisons 1e-10 in units of h^(|alpha| - 1); finite differences (step 1e-6 in
float64, the gradient workload's convention) 1e-6 relative to the gradient's scale."""
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import edge2d as O
from warpsphboundaries_b200 import workloads
from warpsphboundaries_b200.autograd import aggregate_moments
from warpsphboundaries_b200.scene import Body, SurfaceRep

pytestmark = pytest.mark.gpu
DEV = "cuda"
ALPHAS = [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]


def _scene(loops, center=(0.0, 0.0), angle=0.0):
    rep = SurfaceRep.loops(loops)
    return Body(center=center, angle=angle, reps=[rep]), rep


def _loss(out, wl, w1, w2):
    return (out["lam"] * wl).sum() + (out["m1"] * w1).sum() + (out["m2"] * w2).sum()


def _near_wall_particles(loops, n, h, seed):
    rng = np.random.default_rng(seed)
    V, E = workloads.edges_of(loops)
    pick = rng.integers(0, len(E), n)
    a, b = V[E[pick, 0]], V[E[pick, 1]]
    t = rng.uniform(0, 1, n)[:, None]
    ang = rng.uniform(0, 2 * np.pi, n)
    rad = rng.uniform(0, 0.95 * h, n)
    return a + t * (b - a) + np.stack([rad * np.cos(ang), rad * np.sin(ang)], 1)


def oracle_grads(loops, X, h, kernel, wl, w1, w2):
    """d loss / dx [N, 2] and d loss / d vertex [V, 2] from the oracle's per-pair chord integrals (identity pose)."""
    V, E = workloads.edges_of(loops)
    cl = O.build_cell_list(V, E, h)
    slots = O.fixed_slots(V, E, cl, X, np.full(len(X), h))
    rows = np.concatenate([np.full(len(s), r) for r, s in enumerate(slots)]).astype(np.int64)
    es = np.concatenate(slots).astype(np.int64)
    p = (V[E[es, 0]] - X[rows]) / h
    q = (V[E[es, 1]] - X[rows]) / h
    u = {(0, 0): wl[rows], (1, 0): w1[rows, 0], (0, 1): w1[rows, 1], (2, 0): w2[rows, 0, 0],
         (1, 1): w2[rows, 0, 1] + w2[rows, 1, 0], (0, 2): w2[rows, 1, 1]}
    dx = np.zeros((len(X), 2))
    dv = np.zeros((len(V), 2))
    for al in ALPHAS:
        a0, (n0, n1, s0, s1) = O._edge_integral(p, q, kernel, al)
        a1s, _ = O._edge_integral(p, q, kernel, al, extra_s=1)
        sc = O.INV_PI * h ** (al[0] + al[1] - 1) * u[al]
        np.add.at(dx[:, 0], rows, -n0 * a0 * sc)
        np.add.at(dx[:, 1], rows, -n1 * a0 * sc)
        ell = s1 - s0
        t1 = (a1s - s0 * a0) / ell
        t0 = a0 - t1
        for c, nrm in enumerate((n0, n1)):
            np.add.at(dv[:, c], E[es, 0], nrm * t0 * sc)
            np.add.at(dv[:, c], E[es, 1], nrm * t1 * sc)
    return dx, dv


@pytest.mark.parametrize("kernel", ["w4", "cubic", "w6"])
def test_adjoint_matches_oracle(kernel):
    loops = workloads.stars(3, (64, 128), seed=21, box=1.0, rmin=0.1, rmax=0.3)
    h = 0.02
    X = _near_wall_particles(loops, 1500, h, 3)
    body, rep = _scene(loops)
    rng = np.random.default_rng(5)
    wl, w1, w2 = rng.normal(size=len(X)), rng.normal(size=(len(X), 2)), rng.normal(size=(len(X), 2, 2))
    pos = torch.tensor(X, dtype=torch.float64, device=DEV, requires_grad=True)
    rep.vertices.requires_grad_(True)
    sup = torch.full((len(X),), h, dtype=torch.float64, device=DEV)
    out = aggregate_moments(body, rep, pos, sup, kernel, h)
    loss = _loss(out, *(torch.tensor(w, device=DEV) for w in (wl, w1, w2)))
    gx, gv = torch.autograd.grad(loss, [pos, rep.vertices])
    rep.vertices.requires_grad_(False)
    dx, dv = oracle_grads(loops, X, h, kernel, wl, w1, w2)
    assert np.abs(gx.cpu().numpy() - dx).max() * h < 1e-10
    assert np.abs(gv.cpu().numpy() - dv).max() * h < 1e-10


def test_adjoint_matches_reference_torch_autograd():
    """per moment: d m_alpha / dx per particle and the vertex gradient of sum_i m_alpha(x_i) against torch autograd
    through the reference's torch2d (w4, star polygon of 128 vertices, h = 0.02)."""
    g = np.load(Path(__file__).parent / "golden" / "torch2d_grad.npz")
    P, X, h = g["polygon"], g["particles"], float(g["h"])
    body, rep = _scene([P])
    sup = torch.full((len(X),), h, dtype=torch.float64, device=DEV)
    for al in ALPHAS:
        key = f"{al[0]}{al[1]}"
        pos = torch.tensor(X, dtype=torch.float64, device=DEV, requires_grad=True)
        rep.vertices.requires_grad_(True)
        out = aggregate_moments(body, rep, pos, sup, "w4", h)
        if al == (0, 0):
            m = out["lam"]
        elif sum(al) == 1:
            m = out["m1"][:, 0 if al == (1, 0) else 1]
        else:
            m = {(2, 0): out["m2"][:, 0, 0], (1, 1): out["m2"][:, 0, 1], (0, 2): out["m2"][:, 1, 1]}[al]
        gx, gv = torch.autograd.grad(m.sum(), [pos, rep.vertices])
        rep.vertices.requires_grad_(False)
        sc = h ** (al[0] + al[1] - 1)
        assert np.abs(m.detach().cpu().numpy() - g["m_" + key]).max() / (sc * h) < 1e-10
        assert np.abs(gx.cpu().numpy() - g["dx_" + key]).max() / sc < 1e-10, al
        # the (1,1) autograd of the reference differentiates m11 itself; the m2 output's off-diagonal is m11
        assert np.abs(gv.cpu().numpy() - g["dv_" + key].sum(0)).max() / sc < 1e-10, al


def test_adjoint_matches_central_differences():
    """d loss / dx of a few particles and d loss / d vertex of a few vertices against central differences of the GPU
    forward with step 1e-6 (float64)."""
    loops = workloads.stars(2, (64, 64), seed=33, box=1.0, rmin=0.15, rmax=0.25)
    h = 0.02
    X = _near_wall_particles(loops, 400, h, 8)
    body, rep = _scene(loops)
    rng = np.random.default_rng(9)
    wl, w1, w2 = rng.normal(size=len(X)), rng.normal(size=(len(X), 2)), rng.normal(size=(len(X), 2, 2))
    W = [torch.tensor(w, device=DEV) for w in (wl, w1, w2)]
    sup = torch.full((len(X),), h, dtype=torch.float64, device=DEV)

    def f(Xa, verts=None):
        if verts is not None:
            r = SurfaceRep(verts, rep.edges.cpu().numpy(), conditioned=False)
            b = Body(reps=[r])
        else:
            r, b = rep, body
        out = aggregate_moments(b, r, torch.tensor(Xa, dtype=torch.float64, device=DEV), sup, "w4", h)
        return float(_loss(out, *W))

    pos = torch.tensor(X, dtype=torch.float64, device=DEV, requires_grad=True)
    rep.vertices.requires_grad_(True)
    out = aggregate_moments(body, rep, pos, sup, "w4", h)
    gx, gv = torch.autograd.grad(_loss(out, *W), [pos, rep.vertices])
    rep.vertices.requires_grad_(False)
    gx, gv = gx.cpu().numpy(), gv.cpu().numpy()
    step = 1e-6
    scale_x = np.abs(gx).max()
    for i in range(0, len(X), 37):
        for c in range(2):
            Xp, Xm = X.copy(), X.copy()
            Xp[i, c] += step
            Xm[i, c] -= step
            fd = (f(Xp) - f(Xm)) / (2 * step)
            assert abs(fd - gx[i, c]) < 1e-6 * scale_x, (i, c, fd, gx[i, c])
    V0 = rep.vertices.detach().cpu().numpy()
    scale_v = np.abs(gv).max()
    for k in range(0, len(V0), 17):
        for c in range(2):
            Vp, Vm = V0.copy(), V0.copy()
            Vp[k, c] += step
            Vm[k, c] -= step
            fd = (f(X, Vp) - f(X, Vm)) / (2 * step)
            assert abs(fd - gv[k, c]) < 1e-6 * scale_v, (k, c, fd, gv[k, c])


def test_lambda_gradient_equals_G():
    """grad_x lambda = int grad_x W = G: the adjoint of lam against the forward's own G channel."""
    loops = workloads.stars(3, (32, 256), seed=2, box=1.0)
    h = 0.02
    X = _near_wall_particles(loops, 2000, h, 1)
    body, rep = _scene(loops, center=(0.2, 0.1), angle=0.9)
    Xw = X @ np.array([[np.cos(0.9), np.sin(0.9)], [-np.sin(0.9), np.cos(0.9)]]) + np.array([0.2, 0.1])
    pos = torch.tensor(Xw, dtype=torch.float64, device=DEV, requires_grad=True)
    sup = torch.full((len(X),), h, dtype=torch.float64, device=DEV)
    out = aggregate_moments(body, rep, pos, sup, "cubic", h)
    (g,) = torch.autograd.grad(out["lam"].sum(), [pos])
    assert (g - out["G"]).abs().max().item() * h < 1e-11
