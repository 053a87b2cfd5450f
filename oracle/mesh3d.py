"""ORACLE -- test infrastructure only, never shipped and never on a product path.

A CPU (Python float64) restatement of the reference's exact closed-surface reduction
(src/warpSPHBoundaries/mesh3d/reference.py), used by the tests as the checker of the 3-D closed-surface kernels.
It follows the reference's formulation, which differs from the device one: the volume -> face step keeps the full
solid-angle flux term of every face (reference.py:256-270), and each face integral is reduced to closed-form edge
primitives (asinh / atan recurrences of edge/primitives.py:17-96 and the K function of reference.py:74-87) instead of
compact potentials and quadrature.

* kernel profile (blocks, C3 normalisation)   mesh3d/reference.py:55-63, edge/kernels.py:96-121
* edge primitives I_m, J_m, S_{j,m}, K_m      edge/primitives.py:17-96, mesh3d/reference.py:74-87
* face integral of r^n 1[r <= R]              mesh3d/reference.py:125-150 (Triangle._scalar)
* edge line moments, in-plane recursion       mesh3d/reference.py:152-188 (Triangle._line, _local)
* face monomial moments                       mesh3d/reference.py:190-200 (Triangle.block_moment)
* volume moments, gradients, Hessian          mesh3d/reference.py:256-311 (ClosedSurface)

Pinned by tests/test_oracle_mesh3d.py against the reference's own mpmath values in tests/golden/mesh3d_golden.json
(made by tests/golden/make_golden.py).  O(faces) per query: small meshes only.
"""
import math
from fractions import Fraction as F
from math import comb

import numpy as np

from oracle.edge2d import blocks

C3PI = {"cubic": F(16), "w2": F(21, 2), "w4": F(495, 32), "w6": F(1365, 64)}
C2PI = {"cubic": F(80, 7), "w2": F(7), "w4": F(9), "w6": F(78, 7)}
ZERO = (0, 0, 0)


def profile(name, h=1.0):
    """[(n, cutoff, coefficient)]: W_h(r) = sum coefficient * r^n 1[r <= cutoff] in 3-D (reference.py:55-63)."""
    ratio = float(C3PI[name] / C2PI[name]) / math.pi
    return [(n, float(R) * h, ratio * float(c) / h ** (n + 3)) for R, P in blocks(name) for n, c in sorted(P.items())]


# ------------------------------------------------------------------ edge primitives, r = sqrt(s^2 + c^2)
def I_up(M, s, c):
    """[int r^m ds for m = 0..M] (odd antiderivatives, upward recurrence; edge/primitives.py:17-35)."""
    cc = c * c
    r = math.sqrt(s * s + cc)
    out = [s]
    if M >= 1:
        out.append((s * r + (cc * math.asinh(s / abs(c)) if c != 0 else 0.0)) / 2)
    for m in range(2, M + 1):
        out.append((s * r ** m + m * cc * out[m - 2]) / (m + 1))
    return out


def Ig(m, s, c):
    """int r^m ds for any integer m (c != 0 when m < 0; edge/primitives.py:58-72)."""
    if m >= 0:
        return I_up(m, s, c)[m]
    cc = c * c
    if m == -1:
        return math.asinh(s / abs(c))
    if m == -2:
        return math.atan(s / c) / c
    return ((m + 3) * Ig(m + 2, s, c) - s * (s * s + cc) ** ((m + 2) / 2)) / ((m + 2) * cc)


def Jg(m, s, c):
    """int s r^m ds (edge/primitives.py:75-78)."""
    if m == -2:
        return math.log(s * s + c * c) / 2
    return (s * s + c * c) ** ((m + 2) / 2) / (m + 2)


def Sg(j, m, s, c):
    """int s^j r^m ds via s^2 = r^2 - c^2 (edge/primitives.py:80-86)."""
    cc = c * c
    if j % 2 == 0:
        k = j // 2
        return sum(comb(k, i) * (-cc) ** (k - i) * Ig(m + 2 * i, s, c) for i in range(k + 1))
    k = (j - 1) // 2
    return sum(comb(k, i) * (-cc) ** (k - i) * Jg(m + 2 * i, s, c) for i in range(k + 1))


def Kfun(m, s, w, a):
    """int r^m / (s^2 + w^2) ds with r^2 = s^2 + w^2 + a^2, w != 0 (reference.py:74-87)."""
    b = abs(w)
    c = math.sqrt(w * w + a * a)
    if m == 0:
        return math.atan(s / b) / b
    if m == -1:
        r = math.sqrt(s * s + c * c)
        return math.atan(a * s / (b * r)) / (a * b) if a else s / (b * b * r)
    if m == 1:
        return math.asinh(s / c) + a * a * Kfun(-1, s, w, a)
    if m >= 2:
        return Ig(m - 2, s, c) + a * a * Kfun(m - 2, s, w, a)
    raise ValueError("K needs m >= -1")


# ------------------------------------------------------------------ one triangle
class Triangle:
    """a planar triangle seen from a query: normal, plane distance z, in-plane frame e1 e2 and per edge
    (w, lo, hi, mu.e1, mu.e2, t.e1, t.e2) (reference.py:90-123)."""

    def __init__(self, verts, query):
        p = [np.asarray(v, float) - np.asarray(query, float) for v in verts]
        d = p[1] - p[0]
        N = np.cross(d, p[2] - p[0])
        nl = np.linalg.norm(N)
        self.normal = N / nl
        self.z = float(N @ p[0]) / nl
        self.a = abs(self.z)
        self.e1 = d / np.linalg.norm(d)
        self.e2 = np.cross(self.normal, self.e1)
        self.edges = []
        for j in range(3):
            v, q = p[j], p[(j + 1) % 3]
            D = q - v
            L = np.linalg.norm(D)
            t = D / L
            mu = np.cross(t, self.normal)
            w = float(np.cross(D, N) @ v) / (L * nl)
            self.edges.append((w, float(D @ v) / L, float(D @ q) / L, float(mu @ self.e1), float(mu @ self.e2),
                               float(t @ self.e1), float(t @ self.e2)))
        self._cache = {}

    def scalar(self, n, R):
        """int over the face of r^n 1[r <= R]; R None: the whole face (reference.py:125-150)."""
        key = ("s", n, R)
        if key in self._cache:
            return self._cache[key]
        a = self.a
        total = 0.0
        if R is None or a < R:
            for w, lo, hi, *_ in self.edges:
                if w == 0:
                    continue
                cuts = [lo, hi]
                if R is not None and R * R > a * a + w * w:
                    L = math.sqrt(R * R - a * a - w * w)
                    cuts += [s for s in (-L, L) if lo < s < hi]
                cuts.sort()
                for l, u in zip(cuts, cuts[1:]):
                    dK0 = Kfun(0, u, w, a) - Kfun(0, l, w, a)
                    if R is None or ((l + u) / 2) ** 2 + w * w + a * a < R * R:
                        term = Kfun(n + 2, u, w, a) - Kfun(n + 2, l, w, a) - a ** (n + 2) * dK0
                    else:
                        term = (R ** (n + 2) - a ** (n + 2)) * dK0
                    total += w * term / (n + 2)
        self._cache[key] = total
        return total

    def line(self, edge, beta, n, R):
        """int along an edge (clipped to the disk of radius R) of the in-plane monomial (u1, u2)^beta r^n
        (reference.py:152-172)."""
        w, lo, hi, mu1, mu2, t1, t2 = edge
        c2 = w * w + self.a * self.a
        if c2 >= R * R:
            return 0.0
        L = math.sqrt(R * R - c2)
        lo, hi = max(lo, -L), min(hi, L)
        if lo >= hi:
            return 0.0
        poly = [1.0]
        for b, mu, t in zip(beta, (mu1, mu2), (t1, t2)):
            q = [comb(b, j) * (w * mu) ** (b - j) * t ** j for j in range(b + 1)]
            new = [0.0] * (len(poly) + b)
            for i, x in enumerate(poly):
                for j, y in enumerate(q):
                    new[i + j] += x * y
            poly = new
        c = math.sqrt(c2)
        return sum(x * (Sg(j, n, hi, c) - Sg(j, n, lo, c)) for j, x in enumerate(poly) if x)

    def local(self, beta, n, R):
        """int over the face of (u1, u2)^beta r^n 1[r <= R] by the in-plane gradient recursion
        (reference.py:174-188)."""
        if not any(beta):
            return self.scalar(n, R)
        key = ("l", beta, n, R)
        if key in self._cache:
            return self._cache[key]
        i = 0 if beta[0] else 1
        b = list(beta)
        b[i] -= 1
        b = tuple(b)
        val = sum(e[3 + i] * (self.line(e, b, n + 2, R) - R ** (n + 2) * self.line(e, b, 0, R))
                  for e in self.edges) / (n + 2)
        if b[i]:
            lower = list(b)
            lower[i] -= 1
            lower = tuple(lower)
            val -= b[i] * (self.local(lower, n + 2, R) - R ** (n + 2) * self.local(lower, 0, R)) / (n + 2)
        self._cache[key] = val
        return val

    def block_moment(self, alpha, n, R):
        """int over the face of y^alpha r^n 1[r <= R] (reference.py:190-200)."""
        poly = {(0, 0): 1.0}
        for i, power in enumerate(alpha):
            lin = {(0, 0): self.z * self.normal[i], (1, 0): self.e1[i], (0, 1): self.e2[i]}
            for _ in range(power):
                new = {}
                for k1, c1 in poly.items():
                    for k2, c2 in lin.items():
                        k = (k1[0] + k2[0], k1[1] + k2[1])
                        new[k] = new.get(k, 0.0) + c1 * c2
                poly = new
        return sum(c * self.local(b, n, R) for b, c in poly.items() if c)

    def integrate(self, prof, alpha):
        return sum(c * self.block_moment(alpha, n, R) for n, R, c in prof)


# ------------------------------------------------------------------ the closed surface
class ClosedSurface:
    """volume integrals over a closed, outward-oriented triangle surface seen from one query
    (reference.py:221-311)."""

    def __init__(self, vertices, faces, query):
        V = np.asarray(vertices, float)
        self.faces = [Triangle(V[list(f)], query) for f in faces]
        self._cache = {}

    def block_moment(self, alpha, n, R):
        """int over the solid of y^alpha r^n 1[r <= R] (reference.py:256-270)."""
        key = (alpha, n, R)
        if key in self._cache:
            return self._cache[key]
        if not any(alpha):
            val = sum(f.z * (f.scalar(n, R) + R ** (n + 3) * (f.scalar(-3, None) - f.scalar(-3, R))) / (n + 3)
                      for f in self.faces if f.z)
        else:
            i = next(j for j, a in enumerate(alpha) if a)
            beta = list(alpha)
            beta[i] -= 1
            beta = tuple(beta)
            val = sum(f.normal[i] * (f.block_moment(beta, n + 2, R) - R ** (n + 2) * f.block_moment(beta, 0, R))
                      for f in self.faces) / (n + 2)
            if beta[i]:
                lower = list(beta)
                lower[i] -= 1
                lower = tuple(lower)
                val -= beta[i] * (self.block_moment(lower, n + 2, R) - R ** (n + 2) * self.block_moment(lower, 0, R)) / (n + 2)
        self._cache[key] = val
        return val

    def moment(self, name, alpha, h):
        return sum(c * self.block_moment(tuple(alpha), n, R) for n, R, c in profile(name, h))

    def kernel_gradient(self, name, alpha, h):
        """int y^alpha grad_query W_h (reference.py:280-284)."""
        alpha = tuple(alpha)
        prof = profile(name, h)
        out = []
        for j in range(3):
            g = -sum(f.normal[j] * f.integrate(prof, alpha) for f in self.faces)
            if alpha[j]:
                lower = list(alpha)
                lower[j] -= 1
                g += alpha[j] * self.moment(name, tuple(lower), h)
            out.append(g)
        return out

    def kernel_hessian(self, name, h):
        """int Hessian_query W_h (reference.py:300-311 with alpha = 0)."""
        L = [(n - 2, R, c * n) for n, R, c in profile(name, h) if n]
        return [[sum(f.normal[i] * f.integrate(L, tuple(int(k == j) for k in range(3))) for f in self.faces)
                 for j in range(3)] for i in range(3)]


BASE_ALPHA = [(0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (2, 0, 0), (1, 1, 0), (1, 0, 1), (0, 2, 0), (0, 1, 1),
              (0, 0, 2)]


def channels(vertices, faces, query, h, name):
    """the 28 baseline channels at one query: value moments, kernel-gradient moments (alpha <= 1), Hessian."""
    cs = ClosedSurface(vertices, faces, query)
    vals = [cs.moment(name, a, h) for a in BASE_ALPHA]
    for a in BASE_ALPHA[:4]:
        vals.extend(cs.kernel_gradient(name, a, h))
    H = cs.kernel_hessian(name, h)
    vals.extend(H[i][j] for i in range(3) for j in range(i, 3))
    return np.array(vals)
