"""CPU oracle (test infrastructure only) for the two detector inputs of the delta+ scheme: the wedge area of the solid
inside the support disk and the largest direction cosine towards the solid.  Only tests/, the smoke check and the CPU
baseline of bench.py use this module, as the checker; the product never imports it.

cone_area     the NON-LOCAL per-edge closed form of src/warpSPHBoundaries/scene/cone_area.py:20-60 (`_edge_sector_area`)
              and :91-135 (`cone_area`, vectorised over points and edges): on a ray at angle phi the solid's measure in
              [0, H] is sum_e s_e min(t_e(phi), H), so the area is background * area(wedge cap disk) + sum_e s_e
              int 1/2 min(t_e, H)^2 dphi over the swept angles of e inside the wedge -- every edge contributes, near or
              far.  The GPU evaluates the LOCAL form (indicator sector minus the chord deficits of the edges within
              one support, src/warpSPHBoundaries/scene/fused.py:180-246), so the two agree to round-off only.  The
              support H may differ per point (the reference's scene function takes one H; its fused kernel one per
              row).  Pinned to the reference's own `cone_area` outputs: tests/golden/cone_area_golden.json.
dir_extreme   (a) `dir_extreme_polar`: the polar-grid oracle of the reference's test (tests/scene/test_fused_wall.py:
              193-226): the largest |cos| over the midpoints of an (nr x nphi) polar grid of the support disk whose
              points lie in the solid by even-odd membership -- independent of the closed form, accurate to the
              angular step.  (b) `dir_extreme_local`: the closed form per row (fused.py:248-308) over the edges within
              one support, with the winding indicator by the angle sum; pinned to (a) at the reference test's
              tolerance (1.5e-2, never below it).
"""
import math

import numpy as np

TWO_PI = 2.0 * math.pi


def _wrap(a):
    return (a + math.pi) % TWO_PI - math.pi


def _seg_integral(l, h, z, H, pn, valid):
    """int_l^h 1/2 min(t_e(phi), H)^2 dphi per (point, edge) (cone_area.py:75-88): a chord part 1/2 z^2 d tan(phi - pn)
    on [l, h] cap (pn - be, pn + be) (be = acos(z / H), the copy nearest the midpoint) and sectors 1/2 H^2 dphi on the
    rest; arrays broadcast together, H per point."""
    with np.errstate(invalid="ignore", divide="ignore"):
        inside = z < H
        be = np.where(inside, np.arccos(np.clip(z / H, None, 1.0)), 0.0)
        k = np.floor((0.5 * (l + h) - pn) / TWO_PI + 0.5)
        c_lo = np.maximum(l, pn + TWO_PI * k - be)
        c_hi = np.minimum(h, pn + TWO_PI * k + be)
        chord = valid & inside & (c_lo < c_hi)
        sector = 0.5 * H * H * np.where(chord, (c_lo - l) + (h - c_hi), h - l)
        tri = np.where(chord, 0.5 * z * z * (np.tan(c_hi - pn) - np.tan(c_lo - pn)), 0.0)
    return np.where(valid, sector + tri, 0.0)


def cone_area(points, axes, half_angle, H, vertices, edges, background=0):
    """area(solid cap disk(p, H) cap wedge(p, atan2(axis), half_angle)) [N] for one polygon (cone_area.py:91-135):
    `points` [N, 2], `axes` [N, 2], `H` scalar or [N], `vertices` [V, 2], `edges` [E, 2] (solid on the left),
    `background` 1 when the solid is the unbounded outside; half_angle >= pi is the full disk."""
    p = np.asarray(points, float).reshape(-1, 2)
    ax = np.asarray(axes, float).reshape(-1, 2)
    V = np.asarray(vertices, float).reshape(-1, 2)
    E = np.asarray(edges, np.int64).reshape(-1, 2)
    Hn = np.broadcast_to(np.asarray(H, float), (len(p),))[:, None]
    al = float(half_angle)
    a, b = V[E[:, 0]], V[E[:, 1]]
    d = b - a
    L = np.sqrt((d * d).sum(1))
    A = a[None] - p[:, None]
    B = b[None] - p[:, None]
    cr = A[..., 0] * B[..., 1] - A[..., 1] * B[..., 0]
    sgn = np.where(cr > 0, 1.0, -1.0)
    Ls = np.maximum(L, 1e-300)[None]
    z = np.abs(cr) / Ls
    pa = np.arctan2(A[..., 1], A[..., 0])
    dphi = _wrap(np.arctan2(B[..., 1], B[..., 0]) - pa)
    lo = np.where(dphi >= 0, pa, pa + dphi)
    hi = np.where(dphi >= 0, pa + dphi, pa)
    du = d / np.maximum(L, 1e-300)[:, None]
    t = (A * du[None]).sum(2, keepdims=True)
    foot = A - t * du[None]
    pn = lo + _wrap(np.arctan2(foot[..., 1], foot[..., 0]) - lo)
    if al >= math.pi:
        total = sgn * _seg_integral(lo, hi, z, Hn, pn, np.ones(lo.shape, bool))
    else:
        th = np.arctan2(ax[:, 1], ax[:, 0])[:, None]
        c = lo + _wrap(th - lo)
        total = np.zeros(lo.shape)
        for k in (-1.0, 0.0, 1.0):
            l = np.maximum(lo, c + TWO_PI * k - al)
            h = np.minimum(hi, c + TWO_PI * k + al)
            total += sgn * _seg_integral(l, h, z, Hn, pn, l < h)
    keep = (L[None] > 0) & (np.abs(cr) >= 1e-300)
    out = (total * keep).sum(1)
    W = 2.0 * al if al < math.pi else TWO_PI
    return out + background * 0.5 * Hn[:, 0] ** 2 * W


def to_local(points, center, angle):
    """Pose.toLocal: R^T (x - c)."""
    c, s = math.cos(angle), math.sin(angle)
    d = np.asarray(points, float) - np.asarray(center, float)
    return np.stack([d[:, 0] * c + d[:, 1] * s, d[:, 1] * c - d[:, 0] * s], 1)


def axes_to_local(axes, angle):
    """a world direction in the body frame: R^T a."""
    c, s = math.cos(angle), math.sin(angle)
    a = np.asarray(axes, float)
    return np.stack([a[:, 0] * c + a[:, 1] * s, a[:, 1] * c - a[:, 0] * s], 1)


def cone_area_scene(bodies, points, axes, half_angle, H):
    """the sum over posed polygons: `bodies` a list of (center, angle, [(vertices, edges, background), ...]) with
    body-frame vertices; points and axes in the world frame (cone_area.py:138-155 poses the vertices instead, which
    is the same area)."""
    out = np.zeros(len(points))
    for center, angle, reps in bodies:
        lp = to_local(points, center, angle)
        la = axes_to_local(axes, angle)
        for V, E, bg in reps:
            out += cone_area(lp, la, half_angle, H, V, E, bg)
    return out


# ------------------------------------------------------------------------------------------------ direction extreme
def winding(points, vertices, edges):
    """winding number of each point (not on an edge) by the angle sum over the edges."""
    p = np.asarray(points, float).reshape(-1, 2)
    V = np.asarray(vertices, float)
    E = np.asarray(edges, np.int64)
    A = V[E[:, 0]][None] - p[:, None]
    B = V[E[:, 1]][None] - p[:, None]
    cr = A[..., 0] * B[..., 1] - A[..., 1] * B[..., 0]
    dt = (A * B).sum(2)
    return np.rint(np.arctan2(cr, dt).sum(1) / TWO_PI)


def _seg_dist(p, a, b):
    d = b - a
    den = max(float(d @ d), 1e-300)
    t = min(max(float((p - a) @ d) / den, 0.0), 1.0)
    e = p - (a + t * d)
    return math.sqrt(float(e @ e))


def dir_extreme_local(points, vecs, H, vertices, edges, background=0, allowed=None):
    """max |v_hat . x_hat| per point (body frame, `vecs` body-frame vectors) over the directions to the solid within
    one support (fused.py:248-308): 1 inside the solid, else over the edges within H the pieces inside the disk --
    1 where the line of v crosses a piece, else the larger |cos| at its two ends; 0 for v = 0.  Points outside
    `allowed` see a background solid everywhere (fused.py:777-784) and nothing otherwise."""
    p = np.asarray(points, float).reshape(-1, 2)
    w = np.asarray(vecs, float).reshape(-1, 2)
    V = np.asarray(vertices, float)
    E = np.asarray(edges, np.int64)
    Hn = np.broadcast_to(np.asarray(H, float), (len(p),))
    ind = winding(p, V, E) + background
    out = np.zeros(len(p))
    for q in range(len(p)):
        nv = math.hypot(w[q, 0], w[q, 1])
        if nv == 0.0:
            continue
        if allowed is not None and not allowed[q]:
            out[q] = 1.0 if background else 0.0
            continue
        vx, vy = w[q] / nv
        best = 1.0 if ind[q] > 0.5 else 0.0
        for e0, e1 in E:
            if best >= 1.0:
                break
            a, b = V[e0], V[e1]
            if not _seg_dist(p[q], a, b) < Hn[q]:
                continue
            ax, ay = a - p[q]
            dx, dy = b - a
            aa = dx * dx + dy * dy
            if aa <= 0:
                continue
            bq = ax * dx + ay * dy
            disc = bq * bq - aa * (ax * ax + ay * ay - Hn[q] ** 2)
            if disc <= 0:
                continue
            sq = math.sqrt(disc)
            t0, t1 = max(0.0, (-bq - sq) / aa), min(1.0, (-bq + sq) / aa)
            if not t0 < t1:
                continue
            cd = dx * vy - dy * vx
            if cd != 0.0 and t0 <= -(ax * vy - ay * vx) / cd <= t1:
                best = 1.0
                continue
            for t in (t0, t1):
                rx, ry = ax + t * dx, ay + t * dy
                rr = math.hypot(rx, ry)
                if rr > 0:
                    best = max(best, abs(rx * vx + ry * vy) / rr)
        out[q] = best
    return out


def _even_odd(X, Y, V, E):
    inside = np.zeros(X.shape, bool)
    for e0, e1 in E:
        (x1, y1), (x2, y2) = V[int(e0)], V[int(e1)]
        cond = (y1 > Y) != (y2 > Y)
        xi = x1 + (Y - y1) * (x2 - x1) / (y2 - y1 + 1e-300)
        inside ^= cond & (X < xi)
    return inside


def dir_extreme_polar(points, vecs, H, vertices, edges, background=0, nr=300, nphi=1440):
    """the independent polar-grid oracle (body frame): the largest |cos(phi - angle(v))| over the midpoints
    (r, phi) of an nr x nphi polar grid of the disk of radius H whose points lie in the solid (even-odd rule;
    background: its complement); 0 for v = 0 or no solid point."""
    p = np.asarray(points, float).reshape(-1, 2)
    w = np.asarray(vecs, float).reshape(-1, 2)
    V = np.asarray(vertices, float)
    E = np.asarray(edges, np.int64)
    Hn = np.broadcast_to(np.asarray(H, float), (len(p),))
    ph = (np.arange(nphi) + 0.5) / nphi * TWO_PI
    out = np.zeros(len(p))
    for q in range(len(p)):
        if w[q, 0] == 0.0 and w[q, 1] == 0.0:
            continue
        rr = (np.arange(nr) + 0.5) / nr * Hn[q]
        X = p[q, 0] + rr[:, None] * np.cos(ph)[None]
        Y = p[q, 1] + rr[:, None] * np.sin(ph)[None]
        solid = _even_odd(X, Y, V, E)
        if background:
            solid = ~solid
        if solid.any():
            cosv = np.broadcast_to(np.abs(np.cos(ph - math.atan2(w[q, 1], w[q, 0])))[None], X.shape)
            out[q] = cosv[solid].max()
    return out
