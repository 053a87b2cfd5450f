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


def c2(n_particles=1 << 20, seed=0, h=0.02, n_polys=64, tangent_fraction=0.01, return_special=False):
    """(loops, particles [N, 2], h) of the large mixed-precision scene; with `return_special` also the row indices of
    the near-tangent particles and of the particles one support away from a vertex."""
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
    if return_special:
        return loops, X, h, {"tangent": slots[:m], "vertex": slots[m:]}
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


# ------------------------------------------------------------------ 3-D closed surfaces
def icosphere(subdivisions, radius=0.6, jitter=0.0, seed=0):
    """(vertices [V, 3], faces [F, 3]) of an icosahedron subdivided `subdivisions` times (20 * 4^k outward faces),
    projected to the sphere of `radius`, each vertex radius then scaled by (1 + jitter U(-1, 1)) (seeded)."""
    t = (1 + 5 ** 0.5) / 2
    V = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    V = [tuple(np.asarray(v, float) / np.linalg.norm(v)) for v in V]
    Fc = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
          (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
          (8, 6, 7), (9, 8, 1)]
    for _ in range(subdivisions):
        mid = {}

        def m(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                p = (np.asarray(V[a]) + np.asarray(V[b])) / 2
                mid[key] = len(V)
                V.append(tuple(p / np.linalg.norm(p)))
            return mid[key]
        out = []
        for a, b, c in Fc:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            out += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        Fc = out
    V = np.asarray(V) * radius
    if jitter:
        rng = np.random.default_rng(seed)
        V = V * (1 + jitter * rng.uniform(-1, 1, (len(V), 1)))
    return V, np.asarray(Fc, dtype=np.int32)


def box_mesh(lo, hi):
    """(vertices, faces) of an axis-aligned box, two outward triangles per side."""
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    V = np.array([[x0, y0, z0], [x1, y0, z0], [x1, y1, z0], [x0, y1, z0], [x0, y0, z1], [x1, y0, z1], [x1, y1, z1],
                  [x0, y1, z1]], float)
    Fc = np.array([(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (1, 2, 6), (1, 6, 5), (2, 3, 7),
                   (2, 7, 6), (3, 0, 4), (3, 4, 7)], dtype=np.int32)
    return V, Fc


def c3(n_particles=1 << 21, seed=0, h=0.03, subdivisions=5):
    """the 3-D scene: 2^21 particles uniform in [-1, 1]^3, h = 0.03, an icosphere of 20 * 4^5 = 20480 faces, radius
    0.6, vertex radii jittered by 5 % (seeded)."""
    V, Fc = icosphere(subdivisions, 0.6, 0.05, seed + 21)
    rng = np.random.default_rng(seed + 22)
    return V, Fc, rng.uniform(-1.0, 1.0, size=(n_particles, 3)), h
