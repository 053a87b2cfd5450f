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

