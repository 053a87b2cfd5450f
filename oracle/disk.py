"""CPU oracle (test infrastructure only) for the disk element: the twelve channels of a solid disk inside the support
of a particle.  Only tests/ use this module, as the checker; the product never imports it.

The reference integrates a solid disk (DiskArrayRep, a solid ImplicitRep disk) by Chebyshev table lookup per
(query, disk) (src/warpSPHBoundaries/edge/warpdisk.py:1-12, edge/disktables.py; its test bounds the tables at 5e-6
against a high-resolution polygon, tests/scene/test_fused_implicit.py (a)).  This oracle restates the integrals
themselves, independently of the device's boundary-arc form: in the frame whose x axis points from the particle to
the disk centre (distance D, radius R, units of the support h) the disk covers, on the circle of radius r about the
particle, the angles |phi| < theta(r), cos theta = (r^2 + D^2 - R^2) / (2 r D) (pi inside, 0 outside), so with
P = pi W and P' its derivative

    lam   = 1/pi int_0^1 P r 2 theta dr            m1_x = 1/pi int P r^2 2 sin(theta) dr
    G_x   = -1/pi int P' r 2 sin(theta) dr         g1_xx, g1_yy = -1/pi int P' r^2 (theta +- sin theta cos theta) dr
    m2_xx, m2_yy = 1/pi int P r^3 (theta +- sin theta cos theta) dr

(the y components and off-diagonals vanish by symmetry), by adaptive quadrature (scipy quad) on the pieces between
the tangency radii |D - R|, D + R and the kernel's block radii, each mapped by r = a + (b - a)(1 - cos t)/2 so that
the square-root behaviour of theta at a tangency radius is smooth, then rotated to the body frame.  The channel convention
is the polygon one (oracle/edge2d.local_twelve): G = -int grad_y W, g1_dj = -int y_d d_j W, physical units.
Pinned against the polygon oracle on area-preserving 4096-gons of the same disks (error O(n^-2)).
"""
import math
import numpy as np
from scipy import integrate

from warpsphboundaries_b200 import kernels as K


def _profile(name):
    """(P(r), P'(r)) of pi W as float functions (sum of the truncated blocks)."""
    blocks = [(float(b.R), [float(x) for x in b.c]) for b in K.kernel(name).blocks]

    def P(r):
        return sum(np.polynomial.polynomial.polyval(r, c) for R, c in blocks if r <= R)

    def dP(r):
        return sum(np.polynomial.polynomial.polyval(r, np.polynomial.polynomial.polyder(c)) for R, c in blocks
                   if r <= R)
    return P, dP, [R for R, _ in blocks]


def _theta(r, D, R):
    if D == 0.0:
        return math.pi if r < R else 0.0
    c = (r * r + D * D - R * R) / (2.0 * r * D)
    return math.acos(min(1.0, max(-1.0, c)))


def disk_local(D, R, name, tol=1e-13):
    """[12] channels (h = 1, frame x along the centre direction): lam, m1 (2), G (2), g1 (4), m2 (3)."""
    P, dP, knots = _profile(name)
    pts = [0.0] + sorted({x for x in [abs(D - R), D + R] + knots if 0.0 < x < 1.0}) + [1.0]

    def q(f):
        # each piece between breakpoints through r = a + (b - a)(1 - cos t)/2: the square-root behaviour of theta at
        # a tangency radius becomes smooth in t
        tot = 0.0
        for a, b in zip(pts[:-1], pts[1:]):
            g = lambda t: f(a + 0.5 * (b - a) * (1.0 - math.cos(t))) * 0.5 * (b - a) * math.sin(t)
            tot += integrate.quad(g, 0.0, math.pi, limit=400, epsabs=tol, epsrel=tol)[0]
        return tot / math.pi

    def sc(r):
        t = _theta(r, D, R)
        return t, math.sin(t), math.cos(t)

    lam = q(lambda r: P(r) * r * 2 * sc(r)[0])
    m1x = q(lambda r: P(r) * r * r * 2 * sc(r)[1])
    Gx = -q(lambda r: dP(r) * r * 2 * sc(r)[1])
    gxx = -q(lambda r: dP(r) * r * r * (sc(r)[0] + sc(r)[1] * sc(r)[2]))
    gyy = -q(lambda r: dP(r) * r * r * (sc(r)[0] - sc(r)[1] * sc(r)[2]))
    mxx = q(lambda r: P(r) * r ** 3 * (sc(r)[0] + sc(r)[1] * sc(r)[2]))
    myy = q(lambda r: P(r) * r ** 3 * (sc(r)[0] - sc(r)[1] * sc(r)[2]))
    return np.array([lam, m1x, 0.0, Gx, 0.0, gxx, 0.0, 0.0, gyy, mxx, 0.0, myy])


def rotate(ch, a):
    """the channels of the centre-aligned frame in the frame where the centre direction has angle a."""
    c, s = math.cos(a), math.sin(a)
    Rm = np.array([[c, -s], [s, c]])
    out = np.empty(12)
    out[0] = ch[0]
    out[1:3] = Rm @ ch[1:3]
    out[3:5] = Rm @ ch[3:5]
    out[5:9] = (Rm @ ch[5:9].reshape(2, 2) @ Rm.T).reshape(4)
    m2 = np.array([[ch[9], ch[10]], [ch[10], ch[11]]])
    m2 = Rm @ m2 @ Rm.T
    out[9:12] = [m2[0, 0], m2[0, 1], m2[1, 1]]
    return out


def disks_local_twelve(centres, radii, lpos, lsup, name):
    """[N, 12] body-frame channels in physical units (the polygon convention: m1 x h, G / h, m2 x h^2) of the union
    of non-overlapping disks (centres [M, 2], radii [M], body frame) at the particles lpos [N, 2], supports [N]."""
    centres = np.asarray(centres, float).reshape(-1, 2)
    radii = np.asarray(radii, float).reshape(-1)
    out = np.zeros((len(lpos), 12))
    for i, (p, h) in enumerate(zip(np.asarray(lpos, float), np.asarray(lsup, float))):
        for c, R in zip(centres, radii):
            v = (c - p) / h
            D = math.hypot(v[0], v[1])
            if D >= 1.0 + R / h:
                continue
            out[i] += rotate(disk_local(D, R / h, name), math.atan2(v[1], v[0]) if D > 0 else 0.0)
        out[i] *= np.array([1, h, h, 1 / h, 1 / h, 1, 1, 1, 1, h * h, h * h, h * h])
    return out


def area_preserving_polygon(centre, R, n):
    """the regular n-gon with the disk's area (vertices at radius R sqrt(2 pi / (n sin(2 pi / n))))."""
    rN = R * math.sqrt(2 * math.pi / (n * math.sin(2 * math.pi / n)))
    t = 2 * np.pi * np.arange(n) / n
    return np.stack([centre[0] + rN * np.cos(t), centre[1] + rN * np.sin(t)], 1)



# ------------------------------------------------------------------------------------------------ detector inputs
def _ray_span(D, R, phi):
    """the part of the ray at angle phi (from the centre direction) inside disk cap unit ball: (lo, hi) or None."""
    sm = D * math.sin(phi)
    if abs(sm) >= R:
        return None
    q = math.sqrt(R * R - sm * sm)
    t1, t2 = D * math.cos(phi) - q, D * math.cos(phi) + q
    lo, hi = min(max(t1, 0.0), 1.0), min(max(t2, 0.0), 1.0)
    return (lo, hi) if hi > lo else None


def disk_wedge_area(D, R, g, half_angle, tol=1e-13):
    """area (support 1) of disk cap unit ball cap the wedge |phi - g| <= half_angle (phi from the centre direction;
    half_angle >= pi: the whole disk) by adaptive quadrature of 1/2 (hi^2 - lo^2) over the ray angles -- the
    reference test's independent numerical angular integration (tests/scene/test_disk_array.py:79-97) in
    adaptive form, split at the tangent rays and the rays through the circle / support-circle crossings."""
    if half_angle >= math.pi:
        a, b = -math.pi, math.pi
    else:
        a, b = g - half_angle, g + half_angle
    cuts = []
    if D >= R and D > 0:
        t = math.asin(min(R / D, 1.0))
        cuts += [t, -t]
    if D > 1e-12:
        arg = (D * D + 1.0 - R * R) / (2.0 * D)
        if abs(arg) <= 1.0:
            t = math.acos(arg)
            cuts += [t, -t]
    pts = sorted({c + 2 * math.pi * k for c in cuts for k in (-2, -1, 0, 1, 2) if a < c + 2 * math.pi * k < b})

    def f(phi):
        s = _ray_span(D, R, phi)
        return 0.0 if s is None else 0.5 * (s[1] ** 2 - s[0] ** 2)
    edges = [a] + pts + [b]
    return sum(integrate.quad(f, x0, x1, limit=400, epsabs=tol, epsrel=tol)[0] for x0, x1 in zip(edges[:-1], edges[1:]))


def disks_cone_area(lpos, axes_local, half_angle, H, centres, radii):
    """[2, N]: wedge and full-disk areas (physical units) of the solid of a disk set at body-frame particles with
    body-frame axes; H per particle."""
    lpos = np.asarray(lpos, float)
    ax = np.asarray(axes_local, float)
    Hn = np.broadcast_to(np.asarray(H, float), (len(lpos),))
    out = np.zeros((2, len(lpos)))
    for i in range(len(lpos)):
        th = math.atan2(ax[i, 1], ax[i, 0])
        for c, R in zip(np.asarray(centres, float).reshape(-1, 2), np.asarray(radii, float).reshape(-1)):
            v = (c - lpos[i]) / Hn[i]
            D = math.hypot(v[0], v[1])
            if D >= 1.0 + R / Hn[i]:
                continue
            g = th - (math.atan2(v[1], v[0]) if D > 0 else 0.0)
            out[0, i] += disk_wedge_area(D, R / Hn[i], g, half_angle) * Hn[i] ** 2
            out[1, i] += disk_wedge_area(D, R / Hn[i], 0.0, math.pi) * Hn[i] ** 2
    return out


def disks_dir_extreme(lpos, vecs_local, H, centres, radii):
    """max |v_hat . x_hat| over the directions from each body-frame particle to the points of the disks within its
    support, in closed form per disk (fused.py:440-475): the directions to one disk form [-b, b] about the centre
    direction, b = asin(R / d) when the tangent points are inside the support, else the angle of the circle's crossing
    with the support circle; the extreme is cos(max(0, psi - b)), 1 inside the disk; 0 for v = 0."""
    lpos = np.asarray(lpos, float)
    w = np.asarray(vecs_local, float)
    Hn = np.broadcast_to(np.asarray(H, float), (len(lpos),))
    out = np.zeros(len(lpos))
    for i in range(len(lpos)):
        nv = math.hypot(w[i, 0], w[i, 1])
        if nv == 0:
            continue
        best = 0.0
        for c, R in zip(np.asarray(centres, float).reshape(-1, 2), np.asarray(radii, float).reshape(-1)):
            cx, cy = c - lpos[i]
            d = math.hypot(cx, cy)
            if d <= R:
                best = 1.0
            elif d - R < Hn[i]:
                h = Hn[i]
                b = (math.asin(min(R / d, 1.0)) if d * d - R * R <= h * h else
                     math.acos(min(max((d * d + h * h - R * R) / (2 * d * h), -1.0), 1.0)))
                psi = math.acos(min(abs(cx * w[i, 0] + cy * w[i, 1]) / (d * nv), 1.0))
                best = max(best, 1.0 if psi <= b else math.cos(psi - b))
        out[i] = best
    return out


def disks_dir_extreme_polar(lpos, vecs_local, H, centres, radii, nr=150, nphi=1440):
    """the polar-grid oracle for disk sets: the largest |cos| over the midpoints of a polar grid of the support disk
    that lie inside a disk (independent of the closed form, accurate to the angular step)."""
    lpos = np.asarray(lpos, float)
    w = np.asarray(vecs_local, float)
    Hn = np.broadcast_to(np.asarray(H, float), (len(lpos),))
    C = np.asarray(centres, float).reshape(-1, 2)
    Rr = np.asarray(radii, float).reshape(-1)
    ph = (np.arange(nphi) + 0.5) / nphi * 2 * np.pi
    out = np.zeros(len(lpos))
    for i in range(len(lpos)):
        if w[i, 0] == 0.0 and w[i, 1] == 0.0:
            continue
        rr = (np.arange(nr) + 0.5) / nr * Hn[i]
        X = lpos[i, 0] + rr[:, None] * np.cos(ph)[None]
        Y = lpos[i, 1] + rr[:, None] * np.sin(ph)[None]
        solid = np.zeros(X.shape, bool)
        for c, R in zip(C, Rr):
            solid |= (X - c[0]) ** 2 + (Y - c[1]) ** 2 < R * R
        if solid.any():
            cosv = np.broadcast_to(np.abs(np.cos(ph - math.atan2(w[i, 1], w[i, 0])))[None], X.shape)
            out[i] = cosv[solid].max()
    return out
