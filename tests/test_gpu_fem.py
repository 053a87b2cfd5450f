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


def _on_mesh(V, E, rng, n):
    """queries exactly on mesh vertices and on edge midpoints (the winding indicator's edge and vertex cases)."""
    vs = V[rng.choice(len(V), n, replace=False)]
    k = rng.choice(len(E), n, replace=False)
    j = rng.integers(0, 3, n)
    mids = (V[E[k, j]] + V[E[k, (j + 1) % 3]]) / 2
    return np.concatenate([vs, mids])


@pytest.mark.parametrize("kernel", ["cubic", "w4", "quintic"])
def test_pair_weights_match_the_oracle(kernel):
    V, E = _mesh(6, jitter=0.3, seed=1)
    rng = np.random.default_rng(2)
    X = np.concatenate([rng.uniform(-0.1, 1.1, (60, 2)), _on_mesh(V, E, rng, 8)])
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
    """sum_k w_k and sum_k G_k over all pairs give the square's lam and G (partition of unity), and sum_k (V_k - x) w_k,
    sum_k (V_k - x)_a G_kj its first moment m1 and Cov (linear reproduction: sum_k V_k phi_k(x') = x'), which checks
    the barycentric gradient terms g_k of every closed-form pair, at queries on vertices and edge midpoints too."""
    V, E = _mesh(32, jitter=0.25, seed=3)
    rng = np.random.default_rng(4)
    X = np.concatenate([rng.uniform(-0.05, 1.05, ((1 << 14) - 400, 2)), _on_mesh(V, E, rng, 200)])
    n = len(X)
    h = np.full(n, 0.05)
    q, e = _pairs(V, E, X, h)
    w, G = pair_weights(q, e, X, h, V, E, "w2", device=DEV, as_torch=True)
    qt = torch.tensor(q, device=DEV, dtype=torch.int64)
    lam = torch.zeros(n, dtype=torch.float64, device=DEV).index_add_(0, qt, w.sum(1))
    grad = torch.zeros((n, 2), dtype=torch.float64, device=DEV).index_add_(0, qt, G.sum(1))
    Xt = torch.tensor(X, device=DEV)
    Vt = torch.tensor(V, device=DEV)
    Et = torch.tensor(E, device=DEV, dtype=torch.int64)
    et = torch.tensor(e, device=DEV, dtype=torch.int64)
    m1 = torch.zeros((n, 2), dtype=torch.float64, device=DEV)
    cov = torch.zeros((n, 2, 2), dtype=torch.float64, device=DEV)
    for k in range(3):
        d = Vt[Et[et, k]] - Xt[qt]
        m1.index_add_(0, qt, d * w[:, k:k + 1])
        cov.index_add_(0, qt, d[:, :, None] * G[:, k, None, :])
    sq = Scene([Body(reps=[SurfaceRep.box((0.0, 0.0), (1.0, 1.0))])], DEV)
    fw = FusedWall(sq, ParticleState(Xt, torch.tensor(h, device=DEV)), 0.05, (FusedGroup("w2"),))
    r = fw.res[0]
    assert float((lam - r["lam"][0]).abs().max()) <= 1e-10
    assert float((grad - r["G"][0]).abs().max()) * 0.05 <= 1e-10
    assert float((m1 - r["m1"][0]).abs().max()) / 0.05 <= 1e-10
    assert float((cov - r["Cov"][0]).abs().max()) <= 1e-10


def test_out_of_range_indices_are_refused_without_a_read():
    """a query, element or vertex index outside its array: the Python call raises ValueError before the launch; the C
    entry point itself writes NaN for that pair, sets the status word and reads nothing out of range."""
    from warpsphboundaries_b200 import _lib
    V, E = _mesh(2)
    X = np.array([[0.3, 0.3], [0.6, 0.2]])
    h = np.array([0.5, 0.5])
    for q, e, EE in (([0, 2], [0, 1], E), ([0, 1], [0, len(E)], E), ([0, 1], [0, 1], np.where(E == 3, 99, E))):
        with pytest.raises(ValueError):
            pair_weights(q, e, X, h, V, EE, "w2", device=DEV)
    dev = torch.device(DEV)
    q = torch.tensor([0, 1, 5, 1], dtype=torch.int32, device=dev)
    e = torch.tensor([0, -1, 2, 3], dtype=torch.int32, device=dev)
    pos = torch.tensor(X, device=dev)
    sup = torch.tensor(h, device=dev)
    Vt = torch.tensor(V, device=dev)
    Et = torch.tensor(E, dtype=torch.int32, device=dev)
    w = torch.zeros((4, 3), dtype=torch.float64, device=dev)
    G = torch.zeros((4, 3, 2), dtype=torch.float64, device=dev)
    st = torch.zeros(1, dtype=torch.int32, device=dev)
    _lib.check(_lib.lib.wsb_pair_weights(1, _lib.ptr(q), _lib.ptr(e), 4, _lib.ptr(pos), _lib.ptr(sup), 2, _lib.ptr(Vt),
                                         len(V), _lib.ptr(Et), len(E), _lib.ptr(w), _lib.ptr(G), _lib.ptr(st),
                                         _lib.ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    assert int(st.item()) == 1
    bad = torch.isnan(w).all(1).cpu().numpy()
    assert bad.tolist() == [False, True, True, False]
    rw, _ = pair_weights([0, 1], [0, 3], X, h, V, E, "w2", device=DEV)
    assert np.allclose(w[[0, 3]].cpu().numpy(), rw, rtol=0, atol=0)


@pytest.mark.skipif(not torch.cuda.is_available() or torch.cuda.device_count() < 2, reason="needs two devices")
def test_pair_weights_on_a_device_that_is_not_current():
    """device='cuda:1' with device 0 current: the launch runs in device 1's context and device 0 stays current."""
    V, E = _mesh(4, jitter=0.2, seed=1)
    X = np.random.default_rng(5).uniform(0.0, 1.0, (50, 2))
    h = np.full(len(X), 0.2)
    q, e = _pairs(V, E, X, h)
    torch.cuda.set_device(0)
    w1, G1 = pair_weights(q, e, X, h, V, E, "w4", device="cuda:1")
    assert torch.cuda.current_device() == 0
    w0, G0 = pair_weights(q, e, X, h, V, E, "w4", device="cuda:0")
    assert np.array_equal(w0, w1) and np.array_equal(G0, G1)
