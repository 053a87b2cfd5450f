"""ORACLE -- test infrastructure only, never shipped and never on a product path.

CPU (numpy / scipy, float64) restatement of the reference's independent shell quadrature for solid half-spaces and
spheres in 3-D (src/warpSPHBoundaries/fluxbridge/radial_reference.py:17-56) and its rotation of the nine axial
invariants into the Cartesian baseline requests (radial_reference.py:59-79; the request list of
src/warpSPHBoundaries/fluxbridge/contract.py:41-46).  Pinned against the reference's 70-digit fixtures in
tests/golden/radial_golden.json (tests/test_oracle_radial.py).

Unit support (h = 1): `distance` is the signed outward distance of the query from the solid (for a sphere
|x - c| - R), `radius` the sphere radius (None: half-space).
"""
from fractions import Fraction as F

import numpy as np
from scipy import integrate

from oracle.edge2d import _padd, _pmul, _ppow

C3PI = {"cubic": F(16), "w2": F(21, 2), "w4": F(495, 32), "w6": F(1365, 64)}
C2PI = {"cubic": F(80, 7), "w2": F(7), "w4": F(9), "w6": F(78, 7)}


def pieces(name):
    """3-D pieces (lo, hi, coefficients of W in r) for unit support (curvbound/kernels.py:1-14)."""
    om = [F(1), F(-1)]
    if name == "cubic":
        inner = _padd(_ppow(om, 3), [-4 * x for x in _ppow([F(1, 2), F(-1)], 3)])
        raw = [(F(0), F(1, 2), inner), (F(1, 2), F(1), _ppow(om, 3))]
    else:
        n, poly = {"w2": (4, [F(1), F(4)]), "w4": (6, [F(1), F(6), F(35, 3)]),
                   "w6": (8, [F(1), F(8), F(25), F(32)])}[name]
        raw = [(F(0), F(1), _pmul(_ppow(om, n), poly))]
    c = float(C3PI[name]) / np.pi
    return [(float(lo), float(hi), [float(x) * c for x in co]) for lo, hi, co in raw]


def invariants(distance, kernel="w2", radius=None):
    """(lam, m1_axial, m2_tangent, m2_axial, G_axial, g1_tangent, g1_axial, H_tangent, H_axial), unit support."""
    d = float(distance)
    res = np.zeros(9)
    full_end = min(1.0, max(0.0, -d))
    cap_end = 1.0 if radius is None else min(1.0, 2 * float(radius) + d)
    for lo, hi, coeff in pieces(kernel):
        for left, right, full in [(lo, min(hi, full_end), True), (max(lo, abs(d)), min(hi, cap_end), False)]:
            if right <= left:
                continue

            def entries(r):
                if full:
                    cap = 1.0
                elif radius is None:
                    cap = -d / r
                else:
                    R = float(radius)
                    cap = (-d * (2 * R + d) - r * r) / (2 * (R + d) * r)
                a0 = 2 * np.pi * (cap + 1)
                a1 = np.pi * (cap * cap - 1)
                at = np.pi * (cap - cap ** 3 / 3 + 2.0 / 3)
                an = 2 * np.pi * (cap ** 3 + 1) / 3
                w = sum(c * r ** n for n, c in enumerate(coeff))
                ell = sum(n * c * r ** (n - 2) for n, c in enumerate(coeff) if n >= 1 and c)
                q = sum(n * (n - 2) * c * r ** (n - 4) for n, c in enumerate(coeff) if n >= 1 and n != 2 and c)
                return (r * r * w * a0, r ** 3 * w * a1, r ** 4 * w * at, r ** 4 * w * an, -r ** 3 * ell * a1,
                        -r ** 4 * ell * at, -r ** 4 * ell * an, r * r * ell * a0 + r ** 4 * q * at,
                        r * r * ell * a0 + r ** 4 * q * an)
            for col in range(9):
                res[col] += integrate.quad(lambda r: entries(r)[col], left, right, epsabs=1e-15, epsrel=1e-14,
                                           limit=200)[0]
    return res


def baseline():
    """the 28 baseline requests (alpha, derivative) of contract.baseline(3), in order."""
    def lattice(d, n):
        if d == 1:
            return [(n,)]
        return [(i,) + b for i in range(n, -1, -1) for b in lattice(d - 1, n - i)]
    mon = lambda deg: [a for n in range(deg + 1) for a in lattice(3, n)]
    z = (0, 0, 0)
    return ([(a, ()) for a in mon(2)] + [(a, (j,)) for a in mon(1) for j in range(3)] +
            [(z, (i, j)) for i in range(3) for j in range(i, 3)])


def select(values, normal, requests=None):
    """the Cartesian values of the requests from the axial invariants (radial_reference.py:59-79)."""
    n = np.asarray(normal, dtype=float)
    out = []
    for alpha, ds in (requests or baseline()):
        ids = tuple(i for i, p in enumerate(alpha) for _ in range(p))
        if not ds and not ids:
            v = values[0]
        elif not ds and len(ids) == 1:
            v = values[1] * n[ids[0]]
        elif len(ds) == 1 and not ids:
            v = values[4] * n[ds[0]]
        else:
            i, j = ids if not ds else ids + tuple(ds)
            t, a = (2, 3) if not ds else ((5, 6) if len(ds) == 1 else (7, 8))
            v = (values[t] if i == j else 0.0) + (values[a] - values[t]) * n[i] * n[j]
        out.append(v)
    return np.array(out)
