"""Seeded synthetic workloads with the shapes of the reference's benchmark configurations (no dataset is involved).

c1  one closed regular 256-gon (radius 0.45, centre (0.5, 0.5), vertices at angles 2 pi k / 256), 4096 particles
    uniform in [0.05, 0.95]^2 kept inside the polygon; w4, h = 0.05.
c2  2^20 particles uniform in [0, 4]^2, h = 0.02; 64 star polygons (centre uniform in [0, 4]^2, mean radius log-uniform
    in [0.05, 0.4], 32..512 vertices, radial jitter +-15 %) in ONE multi-loop surface of one body; about 1 % of the edges
    get a particle at distance h (1 - eps) from the edge line (eps in {1e-3, 1e-6, 1e-9}) and some vertices a particle
    at distance h along an axis: near-tangent chords and endpoints on the support circle.
c4  2^18 particles uniform in [0, 4]^2, 16 star polygons of 128 vertices, h = 0.02, w4 (the gradient workload).
"""
import numpy as np


def star(rng, center, rbar, n, jitter=0.15):
    t = 2 * np.pi * np.arange(n) / n
    r = rbar * (1 + rng.uniform(-jitter, jitter, n))
    return np.stack([center[0] + r * np.cos(t), center[1] + r * np.sin(t)], 1)


def inside_polygon(x, P):
    """even-odd crossing test of points x [M, 2] against one closed polygon P [n, 2] (workload generation only)."""
    a, b = P, np.roll(P, -1, 0)
    cnt = np.zeros(len(x), dtype=np.int64)
    for i in range(len(P)):
        ay, by = a[i, 1], b[i, 1]
        straddle = (ay > x[:, 1]) != (by > x[:, 1])
        xc = a[i, 0] + (x[:, 1] - ay) * (b[i, 0] - a[i, 0]) / np.where(by == ay, 1, by - ay)
        cnt += straddle & (x[:, 0] < xc)
    return cnt % 2 == 1


def c1(n_particles=4096, seed=0):
    """(loops, particles [N, 2], h) of the regular 256-gon scene."""
    k = np.arange(256)
    P = np.stack([0.5 + 0.45 * np.cos(2 * np.pi * k / 256), 0.5 + 0.45 * np.sin(2 * np.pi * k / 256)], 1)
    rng = np.random.default_rng(seed)
    pts = []
    while len(pts) < n_particles:
        c = rng.uniform(0.05, 0.95, size=(4 * n_particles, 2))
        pts.extend(c[inside_polygon(c, P)][: n_particles - len(pts)])
    return [P], np.asarray(pts[:n_particles]), 0.05


def stars(n_polys, n_vertices, seed, box=4.0, rmin=0.05, rmax=0.4):
    rng = np.random.default_rng(seed)
    loops = []
    for _ in range(n_polys):
        c = rng.uniform(0, box, 2)
        rbar = float(np.exp(rng.uniform(np.log(rmin), np.log(rmax))))
        n = int(rng.integers(n_vertices[0], n_vertices[1] + 1))
        loops.append(star(rng, c, rbar, n))
    return loops


def c2(n_particles=1 << 20, seed=0, h=0.02, n_polys=64, tangent_fraction=0.01):
    """(loops, particles [N, 2], h) of the large mixed-precision scene."""
    loops = stars(n_polys, (32, 512), seed)
    rng = np.random.default_rng(seed + 1)
    X = rng.uniform(0, 4.0, size=(n_particles, 2))
    # near-tangent particles: distance h (1 - eps) from the line of ~1 % of the edges, foot point inside the edge
    V = np.concatenate(loops)
    E = np.concatenate([np.stack([o + np.arange(len(L)), o + (np.arange(len(L)) + 1) % len(L)], 1)
                        for L, o in zip(loops, np.cumsum([0] + [len(L) for L in loops[:-1]]))])
    m = max(1, int(tangent_fraction * len(E)))
    pick = rng.choice(len(E), size=m, replace=False)
    a, b = V[E[pick, 0]], V[E[pick, 1]]
    d = b - a
    nrm = np.stack([d[:, 1], -d[:, 0]], 1) / np.linalg.norm(d, axis=1, keepdims=True)       # the fluid side (outward)
    eps = np.array([1e-3, 1e-6, 1e-9])[rng.integers(0, 3, m)]
    tpar = rng.uniform(0.1, 0.9, m)
    Xt = a + tpar[:, None] * d + (h * (1 - eps))[:, None] * nrm
    # endpoints on the support circle: a particle h away from a vertex along +x
    mv = max(1, m // 4)
    vsel = rng.choice(len(V), size=mv, replace=False)
    Xv = V[vsel] + np.array([h, 0.0])
    slots = rng.choice(n_particles, size=m + mv, replace=False)
    X[slots[:m]] = Xt
    X[slots[m:]] = Xv
    return loops, X, h


def c4(n_particles=1 << 18, seed=0, h=0.02):
    loops = stars(16, (128, 128), seed + 11)
    rng = np.random.default_rng(seed + 12)
    return loops, rng.uniform(0, 4.0, size=(n_particles, 2)), h


def edges_of(loops):
    """(vertices [V, 2], edges [E, 2]) of counter-clockwise loops concatenated."""
    V, E, off = [], [], 0
    for L in loops:
        n = len(L)
        V.append(L)
        E.append(np.stack([off + np.arange(n), off + (np.arange(n) + 1) % n], 1))
        off += n
    return np.concatenate(V), np.concatenate(E)
