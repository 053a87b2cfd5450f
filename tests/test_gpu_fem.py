"""Finite-element pair weights of P1 triangles (wsb_pair_weights, fem.pair_weights) against the oracle
(oracle/fem.py: the triangle's exact channels from the pinned polygon oracle, combined with the barycentric
functions): pairs on the exact closed-form route within 1e-10 of the scale, pairs on the reference's far-field 8 x 8
rule within 1e-8; both element orientations; and at full size the partition of unity: over a conforming mesh of a
square the weights of all elements and vertices add up to the square's own kernel mass and gradient (FusedWall on
the square's outline) within 1e-10."""
import numpy as np
import pytest
import torch

from helpers import DEV
from oracle import fem as OF
from warpsphboundaries_b200.fem import pair_weights
from warpsphboundaries_b200.provider import FusedGroup, FusedWall
from warpsphboundaries_b200.scene import Body, Scene, SurfaceRep
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu


def _mesh(n, jitter=0.0, seed=0):
    """a conforming triangulation of [0, 1]^2: n x n squares, each cut along a diagonal; every other element listed
    clockwise (the weights do not depend on the orientation)."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, 1.0, n + 1)
    X, Y = np.meshgrid(xs, xs, indexing="ij")
    V = np.stack([X.ravel(), Y.ravel()], 1)
    inner = (V[:, 0] > 0) & (V[:, 0] < 1) & (V[:, 1] > 0) & (V[:, 1] < 1)
    V[inner] += rng.uniform(-jitter, jitter, (inner.sum(), 2)) / n
    vid = lambda i, j: i * (n + 1) + j
    E = []
    for i in range(n):
        for j in range(n):
            a, b, c, d = vid(i, j), vid(i + 1, j), vid(i + 1, j + 1), vid(i, j + 1)
            E += [[a, b, c], [a, d, c]] if (i + j) % 2 else [[a, b, d], [b, c, d]]
    return V, np.array(E)


def _pairs(V, E, X, h):
    T = V[E]
    lo, hi = T.min(1), T.max(1)
    q, e = [], []
    for i, x in enumerate(X):
        d = np.maximum(lo - x, 0) + np.maximum(x - hi, 0)
        near = np.nonzero(np.hypot(d[:, 0], d[:, 1]) < h[i])[0]
        q += [i] * len(near)
        e += list(near)
    return np.array(q), np.array(e)


@pytest.mark.parametrize("kernel", ["cubic", "w4", "quintic"])
def test_pair_weights_match_the_oracle(kernel):
    V, E = _mesh(6, jitter=0.3, seed=1)
    rng = np.random.default_rng(2)
    X = rng.uniform(-0.1, 1.1, (60, 2))
    h = rng.uniform(0.12, 0.3, len(X))
    q, e = _pairs(V, E, X, h)
    w, G = pair_weights(q, e, X, h, V, E, kernel, device=DEV)
    rw, rG = OF.pair_weights(q, e, X, h, V, E, kernel)
    # which pairs took the far-field rule (the reference's test, restated)
    r = (V[E[e]] - X[q][:, None, :]) / h[q][:, None, None]
    rho = np.linalg.norm(r.mean(1), axis=1)
    emax = np.max(np.linalg.norm(r - np.roll(r, -1, axis=1), axis=2), axis=1)
    far = rho >= emax
    err_w = np.abs(w - rw).max(1)
    err_G = np.abs(G - rG).max((1, 2)) * h[q]
    assert err_w[~far].max() <= 1e-10 and err_G[~far].max() <= 1e-10
    assert err_w.max() <= 1e-8 and err_G.max() <= 1e-8
    assert (~far).sum() > 20 and far.sum() > 20


def test_partition_of_unity_over_a_square():
    V, E = _mesh(32, jitter=0.25, seed=3)
    n = 1 << 14
    X = np.random.default_rng(4).uniform(-0.05, 1.05, (n, 2))
    h = np.full(n, 0.05)
    q, e = _pairs(V, E, X, h)
    w, G = pair_weights(q, e, X, h, V, E, "w2", device=DEV, as_torch=True)
    qt = torch.tensor(q, device=DEV, dtype=torch.int64)
    lam = torch.zeros(n, dtype=torch.float64, device=DEV).index_add_(0, qt, w.sum(1))
    grad = torch.zeros((n, 2), dtype=torch.float64, device=DEV).index_add_(0, qt, G.sum(1))
    sq = Scene([Body(reps=[SurfaceRep.box((0.0, 0.0), (1.0, 1.0))])], DEV)
    fw = FusedWall(sq, ParticleState(torch.tensor(X, device=DEV), torch.tensor(h, device=DEV)), 0.05,
                   (FusedGroup("w2"),))
    assert float((lam - fw.res[0]["lam"][0]).abs().max()) <= 1e-10
    assert float((grad - fw.res[0]["G"][0]).abs().max()) * 0.05 <= 1e-10
