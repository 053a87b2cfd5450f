"""ORACLE -- test infrastructure only, never shipped and never on a product path.

A CPU (numpy, float64) restatement of the reference's 2-D boundary-integral
path of wi-re/warpSPHBoundaries, used by the tests, by `__graft_entry__.smoke()`
and by the `cpu_baseline` / `--impl reference` legs of `bench.py` as the checker
and the CPU baseline.  It follows the reference algorithm step by step:

* kernel blocks (truncated monomials)   src/warpSPHBoundaries/edge/kernels.py:96-121
* exact compact-potential plan            src/warpSPHBoundaries/edge/np2d.py:45-95
* twelve-channel term plan (truncated)    src/warpSPHBoundaries/edge/warpbc.py:40-129, 970-991
* closed-form primitives I_m, S_{j,m}     src/warpSPHBoundaries/edge/np2d.py:226-264
* per-pair channel evaluation             src/warpSPHBoundaries/edge/warpbc.py:619-661
* cell list / segment-distance predicate  src/warpSPHBoundaries/scene/scene.py:100-139
* fixed-capacity slots, cell-list order   src/warpSPHBoundaries/scene/fixedadj.py:67-97
* winding-number indicator                src/warpSPHBoundaries/scene/scene.py:350-396
* contraction, physical scaling, frame    src/warpSPHBoundaries/scene/fused.py:69-154,
                                          src/warpSPHBoundaries/scene/scene.py:384-416
* moment gradient / shape gradient        src/warpSPHBoundaries/edge/np2d.py:554-565, 626-652

Parity is pinned: `tests/test_oracle_golden.py` checks this module against the
reference's 40-digit golden vectors (`tests/golden/edge2d_golden_subset.json`,
made by `tests/golden/make_golden.py` from the reference fixture file) and
against the reference's own numpy implementation run in the build container
(`tests/golden/np2d_*.npz`, same script).
"""
from fractions import Fraction as F
from functools import lru_cache
from math import comb

import numpy as np

INV_PI = 1.0 / np.pi

# ----------------------------------------------------------------------------- kernels
# pi*W pieces of the normalised kernels (h = 1), the shapes of
# src/warpSPHBoundaries/curvbound/kernels.py:1-14 and src/warpSPHBoundaries/edge/kernels.py:124-181


def _pmul(a, b):
    out = [F(0)] * (len(a) + len(b) - 1)
    for i, x in enumerate(a):
        for j, y in enumerate(b):
            out[i + j] += x * y
    return out


def _ppow(a, k):
    out = [F(1)]
    for _ in range(k):
        out = _pmul(out, a)
    return out


def _padd(a, b):
    n = max(len(a), len(b))
    return [(a[i] if i < len(a) else 0) + (b[i] if i < len(b) else 0) for i in range(n)]


@lru_cache(maxsize=None)
def blocks(name):
    """[(R, {n: c})] pi-free truncated blocks of the kernel, R descending (edge/kernels.py:96-109)."""
    om = [F(1), F(-1)]
    if name == "cubic":
        C = F(80, 7)
        inner = _padd(_ppow(om, 3), [-4 * x for x in _ppow([F(1, 2), F(-1)], 3)])
        pieces = [(F(1, 2), [C * x for x in inner]), (F(1), [C * x for x in _ppow(om, 3)])]
    elif name in ("w2", "w4", "w6"):
        n, poly, C = {"w2": (4, [F(1), F(4)], F(7)), "w4": (6, [F(1), F(6), F(35, 3)], F(9)),
                      "w6": (8, [F(1), F(8), F(25), F(32)], F(78, 7))}[name]
        pieces = [(F(1), [C * x for x in _pmul(_ppow(om, n), poly)])]
    elif name == "poly6":
        pieces = [(F(1), [F(4) * x for x in [F(1), F(0), F(-3), F(0), F(3), F(0), F(-1)]])]
    elif name in ("cone", "lw2", "lw4"):
        # the wall-operator kernels: cone 3 (1 - r) (edge/kernels.py:179-181); W'/r of w2 / w4 registered as
        # 10 (1 - r)^3 and 28/3 (6 u^5 - 5 u^6), u = 1 - r (scene/viscosity.py:48-61; normalisation of edge/kernels.py:141-156)
        shape, C = {"cone": (om, F(3)), "lw2": (_ppow(om, 3), F(10)),
                    "lw4": (_padd([6 * x for x in _ppow(om, 5)], [-5 * x for x in _ppow(om, 6)]), F(28, 3))}[name]
        pieces = [(F(1), [C * x for x in shape])]
    else:
        terms, C = {"quartic": ([(1, F(1), 4), (-5, F(3, 5), 4), (10, F(1, 5), 4)], F(46875, 2398)),
                    "quintic": ([(1, F(1), 5), (-6, F(2, 3), 5), (15, F(1, 3), 5)], F(15309, 478))}[name]
        out = {}
        for c, R, p in terms:
            out[R] = _padd(out.get(R, [F(0)]), [F(c) * C * x for x in _ppow([R, F(-1)], p)])
        return tuple((R, {n: c for n, c in enumerate(out[R]) if c != 0}) for R in sorted(out, reverse=True))
    res = []
    for j in range(len(pieces) - 1, -1, -1):
        R, c = pieces[j]
        cc = c if j == len(pieces) - 1 else _padd(c, [-x for x in pieces[j + 1][1]])
        res.append((R, {n: x for n, x in enumerate(cc) if x != 0}))
    return tuple(res)


def kernel_mass_and_plane(name):
    """(int W, int y_x^2 W) over the whole plane, h = 1, exact (warptriangle.py:220-231)."""
    mass, p2 = F(0), F(0)
    for R, P in blocks(name):
        mass += 2 * sum(c * R ** (n + 2) / (n + 2) for n, c in P.items())
        p2 += sum(c * R ** (n + 4) / (n + 4) for n, c in P.items())
    return mass, p2


def plane_channels(name):
    m, p2 = kernel_mass_and_plane(name)
    m, p2 = float(m), float(p2)
    return np.array([m, 0, 0, 0, 0, m, 0, 0, m, p2, 0, p2])


# ----------------------------------------------------------------------------- exact plan (np2d.py:45-95)
def _phi(P, R):
    out, const = {}, F(0)
    for n, c in P.items():
        out[n + 2] = out.get(n + 2, 0) + c / (n + 2)
        const -= c * F(R) ** (n + 2) / (n + 2)
    out[0] = out.get(0, 0) + const
    return {n: c for n, c in out.items() if c != 0}


def _compile(P, R, alpha, mult, edges, values):
    a, b = alpha
    if a + b == 0:
        d = values.setdefault(R, {})
        for n, c in P.items():
            d[n] = d.get(n, 0) + mult * c
        return
    i = 0 if a > 0 else 1
    beta = (a - 1, b) if i == 0 else (a, b - 1)
    Ph = _phi(P, R)
    d = edges.setdefault((i, beta, R), {})
    for n, c in Ph.items():
        d[n] = d.get(n, 0) + mult * c
    if beta[i] >= 1:
        bm = (beta[0] - (i == 0), beta[1] - (i == 1))
        _compile(Ph, R, bm, -mult * beta[i], edges, values)


@lru_cache(maxsize=None)
def compile_moment(name, alpha):
    edges, values = {}, {}
    for R, P in blocks(name):
        _compile(dict(P), R, tuple(alpha), F(1), edges, values)
    return ({k: {n: c for n, c in d.items() if c != 0} for k, d in edges.items()},
            {R: {n: c for n, c in d.items() if c != 0} for R, d in values.items() if any(d.values())})


@lru_cache(maxsize=None)
def plan(name):
    """twelve-channel truncated term plan: edge terms (ch, i, (a, b), R, {n: c}) and value terms (ch, R, {n: c}, mR)
    (warpbc.py:98-117 with the var/gate filter of warpbc.py:637-661, plus warpbc.py:970-991 as channels 9..11)."""
    E, V = [], []

    def moment(ch, al, scale):
        edges, vals = compile_moment(name, al)
        for (i, beta, R), P in edges.items():
            E.append((ch, i, beta, R, {n: c * scale for n, c in P.items()}))
        for R, P in vals.items():
            mR = sum(c * F(R) ** (n + 2) / (n + 2) for n, c in P.items())
            V.append((ch, R, {n: c * scale / (n + 2) for n, c in P.items()}, mR * scale))

    for ch, al in enumerate([(0, 0), (1, 0), (0, 1)]):
        moment(ch, al, F(1))
    for k, al in enumerate([(0, 0), (1, 0), (0, 1)]):
        for j in (0, 1):
            ch = 3 + 2 * k + j
            for R, P in blocks(name):
                E.append((ch, j, al, R, {n: -c for n, c in P.items()}))
            if al[j]:
                moment(ch, (al[0] - (j == 0), al[1] - (j == 1)), F(al[j]))
    for ch, al in zip((9, 10, 11), [(2, 0), (1, 1), (0, 2)]):
        moment(ch, al, F(1))
    return E, V


# ----------------------------------------------------------------------------- primitives (np2d.py:226-264)
def _I_all(M, s, z):
    """[I_0 .. I_M]: I_m(s) = int_0^s r^m ds, r = sqrt(s^2 + z^2) (parity recurrence, z = 0 guarded)."""
    zz = z * z
    r = np.sqrt(s * s + zz)
    out = [s]
    if M >= 1:
        safe = np.where(z == 0, 1.0, np.abs(z))
        out.append((s * r + np.where(z == 0, 0.0, zz * np.arcsinh(s / safe))) / 2)
    for m in range(2, M + 1):
        out.append((s * r ** m + m * zz * out[m - 2]) / (m + 1))
    return out


def _S(j, m, s, z):
    """int s^j r^m ds (closed form)."""
    zz = z * z
    if j % 2 == 0:
        h = j // 2
        I = _I_all(m + 2 * h, s, z)
        return sum(comb(h, i) * (-zz) ** (h - i) * I[m + 2 * i] for i in range(h + 1))
    h = (j - 1) // 2
    r = np.sqrt(s * s + zz)
    return sum(comb(h, i) * (-zz) ** (h - i) * r ** (m + 2 * i + 2) / (m + 2 * i + 2) for i in range(h + 1))


def _ycoef(a, b, z, n0, n1, t0, t1):
    """coefficients (in s) of (z n0 + s t0)^a (z n1 + s t1)^b."""
    out = [np.ones_like(z)]

    def mul(p, q):
        r = [0] * (len(p) + len(q) - 1)
        for i, x in enumerate(p):
            for j, y in enumerate(q):
                r[i + j] = r[i + j] + x * y
        return r
    for _ in range(a):
        out = mul(out, [z * n0, t0])
    for _ in range(b):
        out = mul(out, [z * n1, t1])
    return out


def _dangle(z, lo, hi):
    y = z * (hi - lo)
    x = z * z + lo * hi
    return np.where((z == 0) | ((y == 0) & (x == 0)), 0.0, np.arctan2(y, x))


def cross2(ax, ay, bx, by):
    """a x b with each product rounded before the subtraction (predicates.py:21-31)."""
    return ax * by - ay * bx          # numpy float64: no FMA contraction


def pair_geometry(p, q):
    """edge frame of pairs: p, q [P, 2] relative vertex positions in units of h (warpbc.py:628-643)."""
    d = q - p
    ell = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1])
    ok = ell > 0
    ell_s = np.where(ok, ell, 1.0)
    t0, t1 = d[:, 0] / ell_s, d[:, 1] / ell_s
    z = cross2(p[:, 0], p[:, 1], q[:, 0], q[:, 1]) / ell_s
    s0 = (d[:, 0] * p[:, 0] + d[:, 1] * p[:, 1]) / ell_s
    s1 = (d[:, 0] * q[:, 0] + d[:, 1] * q[:, 1]) / ell_s
    return ok, t0, t1, t1, -t0, z, s0, s1


def edge_channels(p, q, name):
    """[P, 12] edge-local channels (units of h, x 1/pi applied) of pairs with relative vertices p, q (units of h):
    0 lam, 1-2 m1, 3-4 G, 5-8 g1, 9-11 m20 m11 m02 (warpbc.py:619-661 and 970-991)."""
    p = np.asarray(p, dtype=np.float64).reshape(-1, 2)
    q = np.asarray(q, dtype=np.float64).reshape(-1, 2)
    ok, t0, t1, n0, n1, z, s0, s1 = pair_geometry(p, q)
    az = np.abs(z)
    E, V = plan(name)
    out = np.zeros((len(p), 12))
    chords = {}
    for R in {float(t[3]) for t in E} | {float(t[1]) for t in V}:
        L = np.sqrt(np.maximum((R - az) * (R + az), 0.0))
        lo = np.maximum(s0, -L)
        hi = np.minimum(s1, L)
        m = ok & (az < R) & (lo < hi)
        chords[R] = (np.where(m, lo, 0.0), np.where(m, hi, 0.0), m)
    memo = {}

    def sdiff(j, n, R):
        key = (j, n, R)
        if key not in memo:
            lo, hi, m = chords[R]
            memo[key] = np.where(m, _S(j, n, hi, z) - _S(j, n, lo, z), 0.0)
        return memo[key]
    for ch, i, (a, b), R, P in E:
        R = float(R)
        yc = _ycoef(a, b, z, n0, n1, t0, t1)
        tot = 0.0
        for j, cj in enumerate(yc):
            tot = tot + cj * sum(float(c) * sdiff(j, n, R) for n, c in P.items())
        ni = n0 if i == 0 else n1
        out[:, ch] += np.where(chords[R][2], ni * tot, 0.0)
    for ch, R, Q, mR in V:
        R = float(R)
        lo, hi, m = chords[R]
        poly = sum(float(c) * sdiff(0, n, R) for n, c in Q.items())
        out[:, ch] += np.where(m, z * poly - float(mR) * _dangle(z, lo, hi), 0.0)
    return out * INV_PI


# ----------------------------------------------------------------------------- adjacency (scene.py:100-139, fixedadj.py:67-97)
def build_cell_list(verts, edges, support_max):
    """static edge cell list of a surface: every edge in all cells its (bbox +- support_max) overlaps; cell = support_max.
    Returns (lo[2], cell, (nx, ny), start[nx*ny+1], items[]) with items in (cell, edge) order (scene.py:100-119, 273-279)."""
    a, b = verts[edges[:, 0]], verts[edges[:, 1]]
    blo, bhi = np.minimum(a, b) - support_max, np.maximum(a, b) + support_max
    gmin, gmax = blo.min(0), bhi.max(0)
    dims = np.maximum(np.ceil((gmax - gmin) / support_max).astype(np.int64), 1)
    nx, ny = int(dims[0]), int(dims[1])
    i0 = np.maximum(np.floor((blo - gmin) / support_max).astype(np.int64), 0)
    i1 = np.minimum(np.floor((bhi - gmin) / support_max).astype(np.int64), dims - 1)
    cells, items = [], []
    for e in range(len(edges)):
        for cy in range(i0[e, 1], i1[e, 1] + 1):
            for cx in range(i0[e, 0], i1[e, 0] + 1):
                cells.append(cx * ny + cy)
                items.append(e)
    cells = np.asarray(cells, dtype=np.int64)
    items = np.asarray(items, dtype=np.int64)
    order = np.argsort(cells, kind="stable")
    counts = np.bincount(cells, minlength=nx * ny)
    start = np.concatenate([[0], np.cumsum(counts)])
    return gmin, float(support_max), (nx, ny), start, items[order]


def segment_distance_lt(px, py, ax, ay, bx, by, h):
    """the neighbour predicate |x - seg(a, b)| < h in float64 (scene.py:135-139, fixedadj.py:92-96)."""
    dx, dy = bx - ax, by - ay
    t = np.clip(((px - ax) * dx + (py - ay) * dy) / np.maximum(dx * dx + dy * dy, 1e-300), 0.0, 1.0)
    ex = px - (ax + t * dx)
    ey = py - (ay + t * dy)
    return np.sqrt(ex * ex + ey * ey) < h


def fixed_slots(verts, edges, cl, lpos, lsup, valid=None):
    """per query row the edges of its cell that pass the predicate, in cell-list order: list of int arrays
    (the slot contents of fixedadj.py:67-97; -1 padding omitted)."""
    lo, cell, (nx, ny), start, items = cl
    out = []
    for r in range(len(lpos)):
        if valid is not None and not valid[r]:
            out.append(np.zeros(0, dtype=np.int64))
            continue
        px, py = lpos[r]
        cx = int(np.floor((px - lo[0]) / cell))
        cy = int(np.floor((py - lo[1]) / cell))
        if not (0 <= cx < nx and 0 <= cy < ny):
            out.append(np.zeros(0, dtype=np.int64))
            continue
        cid = cx * ny + cy
        es = items[start[cid]:start[cid + 1]]
        a, b = verts[edges[es, 0]], verts[edges[es, 1]]
        keep = segment_distance_lt(px, py, a[:, 0], a[:, 1], b[:, 0], b[:, 1], lsup[r])
        out.append(es[keep])
    return out


# ----------------------------------------------------------------------------- indicator (scene.py:350-396)
def indicator(verts, edges, background, lpos, lsup=None):
    """winding number + background; on an edge / vertex the principal-value angle fraction; half-open crossings elsewhere.
    Relative coordinates normalised by the per-query support, as the edge terms (scene.py:350-396, fixedadj.py:98-145)."""
    lpos = np.asarray(lpos, dtype=np.float64)
    N = len(lpos)
    A, C = verts[edges[:, 0]], verts[edges[:, 1]]
    out = np.zeros(N)
    for r0 in range(0, N, 512):
        x = lpos[r0:r0 + 512]
        hh = np.ones(len(x)) if lsup is None else np.asarray(lsup[r0:r0 + 512], dtype=np.float64)
        arx = (A[None, :, 0] - x[:, None, 0]) / hh[:, None]
        ary = (A[None, :, 1] - x[:, None, 1]) / hh[:, None]
        crx = (C[None, :, 0] - x[:, None, 0]) / hh[:, None]
        cry = (C[None, :, 1] - x[:, None, 1]) / hh[:, None]
        cr = cross2(arx, ary, crx, cry)
        py = x[:, None, 1]
        up = (A[None, :, 1] <= py) & (py < C[None, :, 1]) & (cr > 0)
        down = (C[None, :, 1] <= py) & (py < A[None, :, 1]) & (cr < 0)
        w = up.sum(1).astype(np.float64) - down.sum(1)
        on = ((cr == 0) & (arx * crx + ary * cry <= 0)).any(1)
        if on.any():
            ang = np.where(cr == 0, 0.0, np.arctan2(cr, arx * crx + ary * cry))
            w = np.where(on, ang.sum(1) / (2 * np.pi), w)
        out[r0:r0 + 512] = w
    return out + background


def ybins(verts, edges, nbins=None):
    """y bins of the edges (scene.py:318-336): bin count 2 floor(sqrt(E)), every edge listed in each bin its y range
    meets, edge order within a bin.  Returns (y0, dy, nb, start[nb + 1], items)."""
    a, b = verts[edges[:, 0]], verts[edges[:, 1]]
    ylo, yhi = np.minimum(a[:, 1], b[:, 1]), np.maximum(a[:, 1], b[:, 1])
    nb = nbins or max(1, int(np.sqrt(len(edges))) * 2)
    y0 = float(ylo.min())
    dy = max(float(yhi.max()) - y0, 1e-300) / nb
    i0 = np.clip(np.floor((ylo - y0) / dy).astype(np.int64), 0, nb - 1)
    i1 = np.clip(np.floor((yhi - y0) / dy).astype(np.int64), 0, nb - 1)
    cnt = i1 - i0 + 1
    item = np.repeat(np.arange(len(edges)), cnt)
    st = np.cumsum(cnt) - cnt
    bins = i0[item] + np.arange(int(cnt.sum())) - np.repeat(st, cnt)
    order = np.argsort(bins, kind="stable")
    start = np.concatenate([[0], np.cumsum(np.bincount(bins[order], minlength=nb))])
    return y0, dy, nb, start, item[order]


def indicator_binned(verts, edges, background, lpos, lsup, cl, bins=None):
    """the reference's fast indicator (scene.py:281-316, 338-396): points in grid cells without edges take the winding
    of their cell centre (ray cast once per cell), points beyond the grid the background, the others a ray cast over
    their y bin's edges (half-open crossings; the principal-value angle sum over all edges for points on an edge or a
    vertex).  Equal to `indicator` (the whole-loop form) wherever the cell cache is exact."""
    verts = np.asarray(verts, dtype=np.float64)
    edges = np.asarray(edges, dtype=np.int64)
    lpos = np.asarray(lpos, dtype=np.float64)
    lsup = np.asarray(lsup, dtype=np.float64)
    lo, cell, (nx, ny), start, _ = cl
    y0, dy, nb, bstart, bitems = bins if bins is not None else ybins(verts, edges)
    cnt = np.diff(start)
    empty = np.nonzero(cnt == 0)[0]
    cind = np.zeros(nx * ny)
    if len(empty):
        centres = lo + (np.stack([empty // ny, empty % ny], 1) + 0.5) * cell
        cind[empty] = _ray_indicator(verts, edges, centres, None, (y0, dy, nb, bstart, bitems))
    cx = np.floor((lpos[:, 0] - lo[0]) / cell).astype(np.int64)
    cy = np.floor((lpos[:, 1] - lo[1]) / cell).astype(np.int64)
    inside = (cx >= 0) & (cx < nx) & (cy >= 0) & (cy < ny)
    cid = np.where(inside, cx * ny + cy, 0)
    fast = inside & (cnt[cid] == 0)
    out = np.where(fast, cind[cid], 0.0)
    out = np.where(~inside, float(background), out)
    slow = np.nonzero(~(fast | ~inside))[0]
    if len(slow):
        out[slow] = _ray_indicator(verts, edges, lpos[slow], lsup[slow], (y0, dy, nb, bstart, bitems)) + background
    out[fast] += background
    return out


def _ray_indicator(verts, edges, p, sup, bins):
    """winding number by the y-bin ray cast (scene.py:338-396), without the background."""
    y0, dy, nb, start, items = bins
    iy = np.floor((p[:, 1] - y0) / dy).astype(np.int64)
    ok = (iy >= 0) & (iy <= nb)
    b = np.where(ok, np.minimum(iy, nb - 1), 0)
    cnt = np.where(ok, start[b + 1] - start[b], 0)
    q = np.repeat(np.arange(len(p)), cnt)
    off = np.arange(int(cnt.sum())) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    e = items[start[b[q]] + off]
    a, c = verts[edges[e, 0]], verts[edges[e, 1]]
    x = p[q]
    ar, cr = a - x, c - x
    if sup is not None:
        ar, cr = ar / sup[q, None], cr / sup[q, None]
    cross = cross2(ar[:, 0], ar[:, 1], cr[:, 0], cr[:, 1])
    up = (a[:, 1] <= x[:, 1]) & (x[:, 1] < c[:, 1]) & (cross > 0)
    down = (c[:, 1] <= x[:, 1]) & (x[:, 1] < a[:, 1]) & (cross < 0)
    wn = np.zeros(len(p))
    np.add.at(wn, q, up.astype(np.float64) - down.astype(np.float64))
    on = (cross == 0) & ((ar * cr).sum(1) <= 0)
    boundary = np.zeros(len(p), dtype=np.int64)
    np.add.at(boundary, q, on.astype(np.int64))
    for r in np.nonzero(boundary > 0)[0]:
        A = verts[edges[:, 0]] - p[r]
        C = verts[edges[:, 1]] - p[r]
        if sup is not None:
            A, C = A / sup[r], C / sup[r]
        cr2 = cross2(A[:, 0], A[:, 1], C[:, 0], C[:, 1])
        ang = np.where(cr2 == 0, 0.0, np.arctan2(cr2, (A * C).sum(1)))
        wn[r] = ang.sum() / (2 * np.pi)
    return wn


# ----------------------------------------------------------------------------- scene composition
def local_twelve(verts, edges, background, lpos, lsup, name, support_max, valid=None, return_slots=False, ind=None,
                 cl=None):
    """[N, 12] local-frame channels in physical units, summed per row in cell-list slot order, + indicator * plane
    (scene.py:384-416 / fused.py:69-154): [lam, m10, m01, Gx, Gy, g1xx, g1xy, g1yx, g1yy, m20, m11, m02].
    `ind` / `cl`: a precomputed indicator (before the `valid` mask) and cell list of these rows, reused across
    kernels."""
    verts = np.asarray(verts, dtype=np.float64)
    edges = np.asarray(edges, dtype=np.int64)
    lpos = np.asarray(lpos, dtype=np.float64)
    lsup = np.asarray(lsup, dtype=np.float64)
    cl = build_cell_list(verts, edges, support_max) if cl is None else cl
    slots = fixed_slots(verts, edges, cl, lpos, lsup, valid)
    rows = np.concatenate([np.full(len(s), r, dtype=np.int64) for r, s in enumerate(slots)]) if slots else np.zeros(0, np.int64)
    es = np.concatenate(slots) if slots else np.zeros(0, np.int64)
    out = np.zeros((len(lpos), 12))
    if len(es):
        hq = lsup[rows][:, None]
        p = (verts[edges[es, 0]] - lpos[rows]) / hq
        q = (verts[edges[es, 1]] - lpos[rows]) / hq
        c = edge_channels(p, q, name)
        for k in range(len(es)):                 # fixed order per row: the slot order
            out[rows[k]] += c[k]
    ind = indicator(verts, edges, background, lpos, lsup) if ind is None else np.asarray(ind, dtype=np.float64)
    if valid is not None:
        ind = np.where(valid, ind, 0.0)
    out += ind[:, None] * plane_channels(name)[None, :]
    h = lsup
    phys = np.stack([np.ones_like(h), h, h, 1 / h, 1 / h, np.ones_like(h), np.ones_like(h), np.ones_like(h),
                     np.ones_like(h), h * h, h * h, h * h], 1)
    out = out * phys
    if return_slots:
        return out, slots, ind
    return out


def to_world(local12, angle):
    """world-frame outputs (lam [N], G [N,2], Cov [N,2,2], m1 [N,2], m2 [N,2,2]) from local channels (fused.py:69-154)."""
    c, s = np.cos(angle), np.sin(angle)
    R = np.array([[c, -s], [s, c]])
    lam = local12[:, 0]
    m1 = local12[:, 1:3] @ R.T
    G = local12[:, 3:5] @ R.T
    g1 = local12[:, 5:9].reshape(-1, 2, 2)
    cov = R[None] @ g1 @ R.T[None]
    m2l = np.stack([local12[:, 9], local12[:, 10], local12[:, 10], local12[:, 11]], 1).reshape(-1, 2, 2)
    m2 = R[None] @ m2l @ R.T[None]
    return dict(lam=lam, G=G, Cov=cov, m1=m1, m2=m2)


def to_local(pos, center, angle):
    """Pose.toLocal (scene.py:75-79): (p - c) R with the rotation written out."""
    c, s = np.cos(angle), np.sin(angle)
    d = np.asarray(pos, dtype=np.float64) - np.asarray(center, dtype=np.float64)
    return np.stack([d[:, 0] * c + d[:, 1] * s, d[:, 1] * c - d[:, 0] * s], 1)


# ----------------------------------------------------------------------------- whole polygons (golden-vector checks)
def polygon_moments(P, x, h, name):
    """value, m_alpha (|alpha| <= 2) of one closed polygon (any orientation) at point x, support h:
    dict {(a, b): value} in physical units (np2d.moment restricted to the truncated plan + winding indicator)."""
    P = np.asarray(P, dtype=np.float64)
    a2 = np.sum(P[:, 0] * np.roll(P[:, 1], -1) - np.roll(P[:, 0], -1) * P[:, 1])
    if a2 < 0:
        P = P[::-1].copy()
    n = len(P)
    edges = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1)
    x = np.asarray(x, dtype=np.float64).reshape(1, 2)
    p = (P[edges[:, 0]] - x) / h
    q = (P[edges[:, 1]] - x) / h
    c = edge_channels(p, q, name).sum(0)
    ind = indicator(P, edges, 0, x, np.array([h]))[0]
    c = c + ind * plane_channels(name)
    return {(0, 0): c[0], (1, 0): c[1] * h, (0, 1): c[2] * h, (2, 0): c[9] * h * h, (1, 1): c[10] * h * h,
            (0, 2): c[11] * h * h, "G": np.array([c[3], c[4]]) / h, "g1": c[5:9].reshape(2, 2)}


def _edge_integral(p, q, name, alpha, extra_s=0):
    """per edge: int_chord s^extra_s y^alpha W ds (units of h, pi-free) summed over the kernel blocks."""
    ok, t0, t1, n0, n1, z, s0, s1 = pair_geometry(p, q)
    az = np.abs(z)
    tot = np.zeros(len(p))
    for R, P in blocks(name):
        R = float(R)
        L = np.sqrt(np.maximum((R - az) * (R + az), 0.0))
        lo = np.maximum(s0, -L)
        hi = np.minimum(s1, L)
        m = ok & (az < R) & (lo < hi)
        lo, hi = np.where(m, lo, 0.0), np.where(m, hi, 0.0)
        yc = [0] * extra_s + _ycoef(alpha[0], alpha[1], z, n0, n1, t0, t1)
        acc = 0.0
        for j, cj in enumerate(yc):
            if isinstance(cj, int):
                continue
            acc = acc + cj * sum(float(c) * (_S(j, nn, hi, z) - _S(j, nn, lo, z)) for nn, c in P.items())
        tot += np.where(m, acc, 0.0)
    return tot, (n0, n1, s0, s1)


def moment_gradient(P, x, h, name, alpha):
    """grad_x m_alpha = -sum_e n_e int_chord y^alpha W ds  (np2d.py:554-565), physical units: [2]."""
    P = np.asarray(P, dtype=np.float64)
    a2 = np.sum(P[:, 0] * np.roll(P[:, 1], -1) - np.roll(P[:, 0], -1) * P[:, 1])
    if a2 < 0:
        P = P[::-1].copy()
    n = len(P)
    x = np.asarray(x, dtype=np.float64).reshape(1, 2)
    p = (P - x) / h
    q = (np.roll(P, -1, 0) - x) / h
    integ, (n0, n1, _, _) = _edge_integral(p, q, name, alpha)
    k = alpha[0] + alpha[1]
    sc = INV_PI * h ** (k - 1)
    return np.array([-(n0 * integ).sum() * sc, -(n1 * integ).sum() * sc])


def shape_gradient(P, x, h, name, alpha):
    """d m_alpha / d vertex_k for every vertex [K, 2] of a polygon given in ccw order (np2d.py:626-652)."""
    P = np.asarray(P, dtype=np.float64)
    x = np.asarray(x, dtype=np.float64).reshape(1, 2)
    p = (P - x) / h
    q = (np.roll(P, -1, 0) - x) / h
    a0, (n0, n1, s0, s1) = _edge_integral(p, q, name, alpha)
    a1s, _ = _edge_integral(p, q, name, alpha, extra_s=1)
    ell = s1 - s0
    a1 = (a1s - s0 * a0) / ell
    out = np.zeros((len(P), 2))
    for comp, nrm in enumerate((n0, n1)):
        out[:, comp] += nrm * (a0 - a1) + np.roll(nrm * a1, 1)
    k = alpha[0] + alpha[1]
    return out * INV_PI * h ** (k - 1)


# ----------------------------------------------------------------------------- powered kernels (tensile group)
# pi*W = C u^p B(u)^5, u = 1 - r: the 5th power of the Wendland C2 / C4 shape (edge/kernels.py:214-232, registered by
# scene/tensile.py:40-47), normalised by C = 1 / (2 int_0^1 r shape^5 dr) (edge/kernels.py:141-156)
_POWERED = {"w2p5": (4, [F(5), F(-4)]), "w4p5": (6, [F(56, 3), F(-88, 3), F(35, 3)])}


@lru_cache(maxsize=None)
def powered(name):
    """(C, p, base coefficients in u) of a powered kernel, C exact."""
    p0, base = _POWERED[name]
    shape = {"w2p5": _pmul(_ppow([F(1), F(-1)], 4), [F(1), F(4)]),
             "w4p5": _pmul(_ppow([F(1), F(-1)], 6), [F(1), F(6), F(35, 3)])}[name]
    s5 = [F(1)]
    for _ in range(5):
        s5 = _pmul(s5, shape)
    integral = sum(c / (n + 2) for n, c in enumerate(s5))      # int_0^1 r shape^5 dr
    return 1 / (2 * integral), 5 * p0, base


def powered_pi_w(name, r):
    C, p, base = powered(name)
    u = 1.0 - np.minimum(r, 1.0)
    b = sum(float(c) * u ** k for k, c in enumerate(base))
    return float(C) * u ** p * b ** 5


def _powered_chord(name, lo, hi, z):
    """int_lo^hi pi*W(sqrt(s^2 + z^2)) ds by adaptive Gauss-Kronrod (QUADPACK), split at the foot s = 0."""
    from scipy.integrate import quad
    f = lambda s: powered_pi_w(name, np.sqrt(s * s + z * z))
    pts = [0.0] if lo < 0.0 < hi else None
    return quad(f, lo, hi, points=pts, epsabs=1e-15, epsrel=1e-13, limit=400)[0]


def powered_gradient(P, x, h, name):
    """grad_x int_solid W dA' of a powered kernel at x = -(1 / (pi h)) sum_e n_e int_chord pi*W ds (chord in units of
    h, clipped to the support): the G channels of the tensile group, physical units [2]."""
    P = np.asarray(P, dtype=np.float64)
    a2 = np.sum(P[:, 0] * np.roll(P[:, 1], -1) - np.roll(P[:, 0], -1) * P[:, 1])
    if a2 < 0:
        P = P[::-1].copy()
    x = np.asarray(x, dtype=np.float64).reshape(1, 2)
    p = (P - x) / h
    q = (np.roll(P, -1, 0) - x) / h
    ok, t0, t1, n0, n1, z, s0, s1 = pair_geometry(p, q)
    g = np.zeros(2)
    for e in range(len(p)):
        az = abs(z[e])
        if not ok[e] or az >= 1.0:
            continue
        L = np.sqrt((1.0 - az) * (1.0 + az))
        lo, hi = max(s0[e], -L), min(s1[e], L)
        if lo < hi:
            w = _powered_chord(name, lo, hi, z[e])
            g -= np.array([n0[e], n1[e]]) * w
    return g * INV_PI / h


def powered_gradient_local(V, E, lpos, h, name):
    """powered_gradient of every body-frame position lpos [N, 2] over the edges E of vertices V (the whole surface,
    one call per particle over the edges within the support), [N, 2]."""
    a, b = V[E[:, 0]], V[E[:, 1]]
    out = np.zeros((len(lpos), 2))
    for i, xq in enumerate(np.asarray(lpos, dtype=np.float64)):
        d = b - a
        t = np.clip(((xq - a) * d).sum(1) / np.maximum((d * d).sum(1), 1e-300), 0.0, 1.0)
        dist = np.linalg.norm(a + t[:, None] * d - xq, axis=1)
        near = np.flatnonzero(dist < h)
        if len(near) == 0:
            continue
        p = (a[near] - xq) / h
        q = (b[near] - xq) / h
        ok, t0, t1, n0, n1, z, s0, s1 = pair_geometry(p, q)
        for e in range(len(near)):
            az = abs(z[e])
            if not ok[e] or az >= 1.0:
                continue
            L = np.sqrt((1.0 - az) * (1.0 + az))
            lo, hi = max(s0[e], -L), min(s1[e], L)
            if lo < hi:
                w = _powered_chord(name, lo, hi, z[e])
                out[i] -= np.array([n0[e], n1[e]]) * w
    return out * INV_PI / h
