"""Exact kernel algebra for the 2-D edge reductions (host side, offline).

Every SPH kernel of this package is a piecewise polynomial in r = |y|/h on [0, 1].
Written as a sum of *blocks* ("truncated monomials"),

    pi * W(r) = sum_b  P_b(r) * 1[r <= R_b],      P_b(r) = sum_n c_{b,n} r^n,

each block is integrated on its own chord (the part of an edge within r <= R_b)
and the channels are linear in the blocks.  This is the decomposition of
`src/warpSPHBoundaries/edge/kernels.py:96-109` (`_blocks_from_pieces`): the
outer piece at R = 1, and for every inner knot the difference of the two pieces
that meet there.

For one block the edge reduction needs six radial functions, all exact
rationals derived here once:

    P(r)            the profile                          (kernel gradient G, g1)
    M(r)   = int_0^r t P dt                              (odd chord integral of P)
    Psi(r) = M(r) - M(R)                                 (first moments m1, second moments m2)
    Flam   = M(r) / r^2,   singular part  -M(R) / r^2    (lambda value term)
    MPsi(r)= int_0^r t Psi dt                            (odd chord integral of Psi)
    FPsi   = MPsi(r) / r^2, singular part -MPsi(R) / r^2 (the Psi area term of m20 / m02)

`emit_header()` writes them as literal coefficients into a C++ header that the
CUDA kernels include (`csrc/kernel_tables.h`), so the per-pair code carries
every coefficient as an immediate operand.

The kernel shapes and their 2-D normalisations follow
`src/warpSPHBoundaries/curvbound/kernels.py:1-14,37-50` (cubic, Wendland C2/C4/C6)
and `src/warpSPHBoundaries/edge/kernels.py:124-181` (truncated-power kernels).
The normalisation is recomputed here from 2 * int_0^1 r (pi W) dr = 1 and checked
against the published constants.
"""
from dataclasses import dataclass, field
from fractions import Fraction as F
from functools import lru_cache
from math import comb
from typing import Dict, List, Tuple

# kernel ids of the C ABI (include/wsb.h: WSB_KERNEL_*); order is part of the ABI
KERNEL_IDS = {"cubic": 0, "w2": 1, "w4": 2, "w6": 3, "quartic": 4, "quintic": 5, "poly6": 6, "cone": 7, "lw2": 8,
              "lw4": 9}
KERNEL_NAMES = {v: k for k, v in KERNEL_IDS.items()}
# the powered kernels W^5 of the Wendland C2 / C4 shapes (the tensile group of the delta+ layout): degree 25 / 40 in r,
# evaluated by a graded Gauss-Legendre quadrature along the chord instead of the monomial closed form
QUAD_KERNEL_IDS = {"w2p5": 10, "w4p5": 11}
QUAD_GAUSS = 24
QUAD_GAUSS_FAR = 12      # panels at least their own length away from the foot (Bernstein parameter >= 5.8)
QUAD_GAUSS_CHORD = 20    # the tensile chord's panel next to the foot (parameter ~2.9: 2.9^-40 ~ 3e-19)

# published 2-D normalisations C2 * pi (src/warpSPHBoundaries/curvbound/kernels.py:5-13,
# src/warpSPHBoundaries/edge/kernels.py:183-185); only used to check the recomputed ones
_PUBLISHED_C2PI = {"cubic": F(80, 7), "w2": F(7), "w4": F(9), "w6": F(78, 7),
                   "quartic": F(46875, 2398), "quintic": F(15309, 478), "poly6": F(4),
                   # the wall-operator kernels: cone (1 - q), the cover vector's kernel, normalisation 3
                   # (src/warpSPHBoundaries/edge/kernels.py:179-181); lw2 (1 - q)^3 and lw4 6 u^5 - 5 u^6 (u = 1 - q),
                   # the kernels W'/r of the wall Laplacian (src/warpSPHBoundaries/scene/viscosity.py:48-61), normalised
                   # by the same rule C = 1 / (2 int_0^1 r shape dr)
                   "cone": F(3), "lw2": F(10), "lw4": F(28, 3)}


# ------------------------------------------------------------------ polynomial helpers (ascending coefficient lists)
def _padd(a, b):
    n = max(len(a), len(b))
    return [(a[i] if i < len(a) else 0) + (b[i] if i < len(b) else 0) for i in range(n)]


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


def _peval(a, x):
    acc = F(0)
    for c in reversed(a):
        acc = acc * x + c
    return acc


def _trim(a):
    a = list(a)
    while len(a) > 1 and a[-1] == 0:
        a.pop()
    return a


def _shape_integral(pieces):
    """int_0^1 r * shape(r) dr over the pieces [(lo, hi, coeffs)]."""
    tot = F(0)
    for lo, hi, c in pieces:
        P = [F(0)] + [F(0)] + [x / (i + 2) for i, x in enumerate(c)]     # int r^(n+1) = r^(n+2)/(n+2)
        tot += _peval(P, hi) - _peval(P, lo)
    return tot


# ------------------------------------------------------------------ kernel shapes
def _pieces(name):
    """pieces [(lo, hi, shape coefficients)] of the UNNORMALISED shape on [0, 1]."""
    one_minus = [F(1), F(-1)]
    if name == "cubic":
        half = [F(1, 2), F(-1)]
        inner = _padd(_ppow(one_minus, 3), [-4 * x for x in _ppow(half, 3)])
        return [(F(0), F(1, 2), inner), (F(1, 2), F(1), _ppow(one_minus, 3))]
    if name in ("w2", "w4", "w6"):
        n, poly = {"w2": (4, [F(1), F(4)]),
                   "w4": (6, [F(1), F(6), F(35, 3)]),
                   "w6": (8, [F(1), F(8), F(25), F(32)])}[name]
        return [(F(0), F(1), _pmul(_ppow(one_minus, n), poly))]
    if name == "poly6":
        return [(F(0), F(1), [F(1), F(0), F(-3), F(0), F(3), F(0), F(-1)])]
    if name == "cone":
        return [(F(0), F(1), one_minus)]
    if name == "lw2":
        return [(F(0), F(1), _ppow(one_minus, 3))]
    if name == "lw4":
        return [(F(0), F(1), _padd([6 * x for x in _ppow(one_minus, 5)], [-5 * x for x in _ppow(one_minus, 6)]))]
    terms = {"quartic": [(1, F(1), 4), (-5, F(3, 5), 4), (10, F(1, 5), 4)],
             "quintic": [(1, F(1), 5), (-6, F(2, 3), 5), (15, F(1, 3), 5)]}.get(name)
    if terms is None:
        raise KeyError(f"unknown kernel {name!r}; expected one of {sorted(KERNEL_IDS)}")
    knots = sorted({R for _, R, _ in terms})
    pieces, lo = [], F(0)
    for hi in knots:
        poly = [F(0)]
        for c, R, p in terms:
            if R >= hi:
                poly = _padd(poly, [F(c) * x for x in _ppow([R, F(-1)], p)])
        pieces.append((lo, hi, poly))
        lo = hi
    return pieces


@dataclass(frozen=True)
class Block:
    """one truncated block  P(r) 1[r <= R]  of pi*W and its derived exact profiles (h = 1)."""
    R: F
    c: Tuple[F, ...]          # P
    m: Tuple[F, ...]          # M(r) = int_0^r t P dt        (coefficient list in r)
    Mhat: F                   # M(R)
    psi: Tuple[F, ...]        # Psi = M - M(R)
    flam: Tuple[F, ...]       # M(r)/r^2                     (regular part of the lambda value profile)
    mpsi: Tuple[F, ...]       # MPsi(r) = int_0^r t Psi dt
    MPhat: F                  # MPsi(R)
    fpsi: Tuple[F, ...]       # MPsi(r)/r^2
    n4: Tuple[F, ...]         # N(r) = int_0^r t^3 P dt      (odd cubic chord integral, adjoint)


@dataclass(frozen=True)
class Kernel:
    name: str
    kid: int
    c2pi: F                                   # C2 * pi of the normalised kernel
    pieces: Tuple[Tuple[F, F, Tuple[F, ...]], ...]   # normalised pi*W pieces (lo, hi, coeffs)
    blocks: Tuple[Block, ...]                 # sorted by R descending
    mass: F                                   # int_plane W dA  (= 1)
    plane2: F                                 # int_plane y_x^2 W dA  (h = 1)

    @property
    def max_degree(self):
        """largest monomial power of r whose chord integral the forward channels need (Psi / FPsi)."""
        return max(max(len(b.psi), len(b.fpsi), len(b.c)) - 1 for b in self.blocks)


def _block(R, c):
    c = _trim(c)
    m = [F(0), F(0)] + [x / (n + 2) for n, x in enumerate(c)]
    Mhat = _peval(m, R)
    psi = list(m)
    psi[0] -= Mhat
    flam = [x / (n + 2) for n, x in enumerate(c)]
    mpsi = [F(0), F(0)] + [x / (n + 2) for n, x in enumerate(psi)]
    MPhat = _peval(mpsi, R)
    fpsi = [x / (n + 2) for n, x in enumerate(psi)]
    n4 = [F(0)] * 4 + [x / (n + 4) for n, x in enumerate(c)]
    t = lambda a: tuple(_trim(a))
    return Block(F(R), t(c), t(m), Mhat, t(psi), t(flam), t(mpsi), MPhat, t(fpsi), t(n4))


@lru_cache(maxsize=None)
def kernel(name: str) -> Kernel:
    """the exact kernel table of `name` (cubic, w2, w4, w6, quartic, quintic, poly6)."""
    raw = _pieces(name)
    C = 1 / (2 * _shape_integral(raw))
    if C != _PUBLISHED_C2PI[name]:
        raise AssertionError(f"normalisation of {name}: {C} != published {_PUBLISHED_C2PI[name]}")
    pieces = tuple((lo, hi, tuple(C * x for x in c)) for lo, hi, c in raw)
    blocks = []
    for j in range(len(pieces) - 1, -1, -1):          # outer piece first, then the differences at the inner knots
        lo, hi, c = pieces[j]
        coeffs = list(c) if j == len(pieces) - 1 else _padd(list(c), [-x for x in pieces[j + 1][2]])
        blocks.append(_block(hi, coeffs))
    blocks = tuple(sorted(blocks, key=lambda b: -b.R))
    mass = 2 * sum(b.Mhat for b in blocks)
    plane2 = -2 * sum(b.MPhat for b in blocks)
    if mass != 1:
        raise AssertionError(f"{name}: block masses sum to {mass}")
    return Kernel(name, KERNEL_IDS[name], C, pieces, blocks, mass, plane2)


def pi_w(name, r: F) -> F:
    """exact pi * W(r) (h = 1) from the blocks (tests)."""
    return sum((_peval(b.c, r) for b in kernel(name).blocks if r <= b.R), F(0))


# ------------------------------------------------------------------ reference term plan (the "plain" interpreter route)
def _phi(P, R):
    """Phi[f](r) = -int_r^R t f dt as {n: c} (the compact potential of src/warpSPHBoundaries/edge/np2d.py:45-52)."""
    out, const = {}, F(0)
    for n, c in P.items():
        out[n + 2] = out.get(n + 2, 0) + c / (n + 2)
        const -= c * F(R) ** (n + 2) / (n + 2)
    out[0] = out.get(0, 0) + const
    return {n: c for n, c in out.items() if c != 0}


def _compile(P, R, alpha, mult, edges, values):
    """the compact-potential recursion of src/warpSPHBoundaries/edge/np2d.py:63-79 (truncated form only)."""
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
    bi = beta[i]
    if bi >= 1:
        bm = (beta[0] - (i == 0), beta[1] - (i == 1))
        _compile(Ph, R, bm, -mult * bi, edges, values)


def compile_moment(name, alpha):
    """exact truncated plan of m_alpha: edges {(i, beta, R): {n: c}}, values {R: {n: c}} (pi-free)."""
    edges, values = {}, {}
    for blk in kernel(name).blocks:
        P = {n: c for n, c in enumerate(blk.c) if c != 0}
        _compile(P, blk.R, tuple(alpha), F(1), edges, values)
    edges = {k: {n: c for n, c in d.items() if c != 0} for k, d in edges.items()}
    values = {R: {n: c for n, c in d.items() if c != 0} for R, d in values.items()}
    return edges, {R: d for R, d in values.items() if d}


@dataclass
class TermPlan:
    """flat term tables of the twelve edge channels (the layout of the reference's per-pair interpreter,
    src/warpSPHBoundaries/edge/warpbc.py:40-129 restricted to the truncated terms its edge kernels evaluate,
    warpbc.py:637-661, plus the second-moment plan of warpbc.py:970-991 as channels 9..11)."""
    radii: List[float] = field(default_factory=list)
    cn: List[int] = field(default_factory=list)
    cc: List[float] = field(default_factory=list)
    E: List[tuple] = field(default_factory=list)     # (ch, i, a, b, Ridx, c0, c1)
    V: List[tuple] = field(default_factory=list)     # (ch, Ridx, c0, c1, mR)

    def R(self, R):
        f = float(R)
        if f not in self.radii:
            self.radii.append(f)
        return self.radii.index(f)

    def coef(self, P, scale):
        c0 = len(self.cn)
        for n, c in sorted(P.items()):
            self.cn.append(n)
            self.cc.append(float(F(c) * scale))
        return c0, len(self.cn)

    def edge(self, ch, i, beta, R, P, scale):
        self.E.append((ch, i, beta[0], beta[1], self.R(R), *self.coef(P, scale)))

    def value(self, ch, R, P, scale):
        mR = sum(c * F(R) ** (n + 2) / (n + 2) for n, c in P.items())
        self.V.append((ch, self.R(R), *self.coef({n: c / (n + 2) for n, c in P.items()}, scale), float(mR * scale)))

    def moment(self, name, ch, alpha, scale):
        edges, vals = compile_moment(name, alpha)
        for (i, beta, R), P in edges.items():
            self.edge(ch, i, beta, R, P, scale)
        for R, P in vals.items():
            self.value(ch, R, P, scale)


@lru_cache(maxsize=None)
def term_plan(name) -> TermPlan:
    """the twelve-channel truncated term plan of `name`:
    0 lam, 1-2 m1, 3-4 G, 5-8 g1 (g(1,0)_x, g(1,0)_y, g(0,1)_x, g(0,1)_y), 9-11 m20, m11, m02."""
    k = kernel(name)
    tp = TermPlan()
    for ch, al in enumerate([(0, 0), (1, 0), (0, 1)]):
        tp.moment(name, ch, al, F(1))
    for kk, al in enumerate([(0, 0), (1, 0), (0, 1)]):
        for j in (0, 1):
            ch = 3 + 2 * kk + j
            for blk in k.blocks:
                tp.edge(ch, j, al, blk.R, {n: c for n, c in enumerate(blk.c) if c != 0}, F(-1))
            if al[j]:
                beta = (al[0] - (j == 0), al[1] - (j == 1))
                tp.moment(name, ch, beta, F(al[j]))
    for ch, al in zip((9, 10, 11), [(2, 0), (1, 1), (0, 2)]):
        tp.moment(name, ch, al, F(1))
    return tp


# ------------------------------------------------------------------ C++ header generation
def _lit(x) -> str:
    v = float(x)
    if v == 0:
        return "0.0"
    return repr(v)


def _dot(coeffs, arr, start=0):
    """C expression  sum_n coeffs[n] * arr[n + start]  (zero coefficients dropped)."""
    parts = [f"{_lit(c)}*{arr}[{n + start}]" for n, c in enumerate(coeffs) if c != 0]
    return " + ".join(parts) if parts else "0.0"


def _horner(coeffs, var):
    """C expression evaluating sum_n coeffs[n] var^n by Horner's rule (leading zero coefficients
    become a power factor, so no fma(x, r, 0.0) appears)."""
    cs = list(coeffs)
    while len(cs) > 1 and cs[-1] == 0:
        cs.pop()
    low = 0
    while low < len(cs) - 1 and cs[low] == 0:
        low += 1
    cs = cs[low:]
    expr = _lit(cs[-1])
    for c in reversed(cs[:-1]):
        expr = f"fma({expr}, {var}, {_lit(c)})"
    for _ in range(low):
        expr = f"({expr})*{var}"
    return expr


def emit_header() -> str:
    """the generated C++ header with every kernel's block profiles as literal code."""
    out = ["// GENERATED by warpsphboundaries_b200/kernels.py (emit_header); do not edit by hand.",
           "// Exact rational kernel profiles rounded once to double; see that module for the algebra.",
           "#pragma once", "", "namespace wsb {", ""]
    out.append(f"constexpr int kNumKernels = {len(KERNEL_IDS)};")
    # the largest A_n index any kernel needs: forward max_degree, adjoint needs c up to deg+2 (s^2 W) on A
    amax = max(max(kernel(n).max_degree, max(len(b.c) + 1 for b in kernel(n).blocks)) for n in KERNEL_IDS)
    out.append(f"constexpr int kMaxA = {amax + 1};   // A_n, n = 0 .. kMaxA-1")
    out.append("")
    out.append("struct BlockSums {      // per (pair, block) chord sums, before the 1/pi and the edge frame")
    out.append("  double W0, W1;        // int P ds, int s P ds")
    out.append("  double P0, P1;        // int Psi ds, int s Psi ds")
    out.append("  double Lreg, Preg;    // int M/r^2 ds, int MPsi/r^2 ds (regular parts of the value terms)")
    out.append("  double Mhat, MPhat;   // singular coefficients M(R), MPsi(R)")
    out.append("};")
    out.append("")
    out.append("struct AdjSums {        // per (pair, block) chord sums of the adjoint")
    out.append("  double W0, W1, W2, W3;   // int s^j P ds, j = 0..3")
    out.append("};")
    out.append("")
    for name, kid in sorted(KERNEL_IDS.items(), key=lambda t: t[1]):
        k = kernel(name)
        out.append(f"// ---- {name}: C2*pi = {k.c2pi}, plane second moment {k.plane2}")
        out.append(f"struct Kern_{name} {{")
        out.append(f"  static constexpr int kId = {kid};")
        out.append("  static constexpr bool kQuad = false;")
        out.append(f"  static constexpr int kBlocks = {len(k.blocks)};")
        out.append(f"  static constexpr double kMass = {_lit(k.mass)};")
        out.append(f"  static constexpr double kPlane2 = {_lit(k.plane2)};")
        nA = [max(len(b.psi), len(b.fpsi), len(b.c)) for b in k.blocks]
        nAadj = [len(b.c) + 2 for b in k.blocks]
        out.append("  static constexpr double kR[kBlocks] = {" + ", ".join(_lit(b.R) for b in k.blocks) + "};")
        out.append("  static constexpr int kNA[kBlocks] = {" + ", ".join(str(n) for n in nA) + "};   // A_0..A_{kNA-1} for the forward sums")
        out.append("  static constexpr int kNAadj[kBlocks] = {" + ", ".join(str(n) for n in nAadj) + "};   // for the adjoint sums")
        out.append("  template <int B> __host__ __device__ static __forceinline__ void sums(const double* A, double rlo, double rhi, BlockSums& o);")
        out.append("  template <int B> __host__ __device__ static __forceinline__ void adj(const double* A, double rlo, double rhi, double zz, AdjSums& o);")
        out.append("};")
        for bi, b in enumerate(k.blocks):
            out.append(f"template <> __host__ __device__ __forceinline__ void Kern_{name}::sums<{bi}>(const double* A, double rlo, double rhi, BlockSums& o) {{")
            out.append(f"  // block R = {b.R}: P = {[str(x) for x in b.c]}")
            out.append(f"  o.W0 = {_dot(b.c, 'A')};")
            out.append(f"  o.W1 = ({_horner(b.m, 'rhi')}) - ({_horner(b.m, 'rlo')});")
            out.append(f"  o.P0 = {_dot(b.psi, 'A')};")
            out.append(f"  o.P1 = ({_horner(b.mpsi, 'rhi')}) - ({_horner(b.mpsi, 'rlo')});")
            out.append(f"  o.Lreg = {_dot(b.flam, 'A')};")
            out.append(f"  o.Preg = {_dot(b.fpsi, 'A')};")
            out.append(f"  o.Mhat = {_lit(b.Mhat)};")
            out.append(f"  o.MPhat = {_lit(b.MPhat)};")
            out.append("}")
            out.append(f"template <> __host__ __device__ __forceinline__ void Kern_{name}::adj<{bi}>(const double* A, double rlo, double rhi, double zz, AdjSums& o) {{")
            out.append(f"  const double a0 = {_dot(b.c, 'A')};")
            out.append(f"  const double a2 = {_dot(b.c, 'A', 2)};")
            out.append(f"  const double m1 = ({_horner(b.m, 'rhi')}) - ({_horner(b.m, 'rlo')});")
            out.append(f"  const double m3 = ({_horner(b.n4, 'rhi')}) - ({_horner(b.n4, 'rlo')});")
            out.append("  o.W0 = a0; o.W1 = m1; o.W2 = a2 - zz * a0; o.W3 = m3 - zz * m1;")
            out.append("}")
        out.append("")
    # the reference term plan tables for the plain interpreter route
    out.append("// ---- reference term plans (plain FP64 interpreter): per kernel offsets into flat tables")
    E, V, CN, CC, RAD, offs = [], [], [], [], [], []
    for name, kid in sorted(KERNEL_IDS.items(), key=lambda t: t[1]):
        tp = term_plan(name)
        e0, v0, c0, r0 = len(E), len(V), len(CN), len(RAD)
        for (ch, i, a, b, Ri, ca, cb) in tp.E:
            E.append((ch, i, a, b, r0 + Ri, c0 + ca, c0 + cb))
        for (ch, Ri, ca, cb, mR) in tp.V:
            V.append((ch, r0 + Ri, c0 + ca, c0 + cb, mR))
        CN.extend(tp.cn)
        CC.extend(tp.cc)
        RAD.extend(tp.radii)
        offs.append((e0, len(E), v0, len(V)))
    out.append(f"constexpr int kPlanEdgeTerms = {len(E)};")
    out.append(f"constexpr int kPlanValueTerms = {len(V)};")
    out.append(f"constexpr int kPlanCoeffs = {len(CN)};")
    out.append(f"constexpr int kPlanNumRadii = {len(RAD)};")
    out.append("struct PlanOffsets { int e0, e1, v0, v1; };")
    out.append("static const PlanOffsets kPlanOffsets[kNumKernels] = {" + ", ".join("{%d, %d, %d, %d}" % o for o in offs) + "};")
    out.append("static const int kPlanE[kPlanEdgeTerms][7] = {   // ch, i, a, b, radius index, c0, c1")
    out.extend("  {%d, %d, %d, %d, %d, %d, %d}," % e for e in E)
    out.append("};")
    out.append("static const int kPlanVi[kPlanValueTerms][4] = {   // ch, radius index, c0, c1")
    out.extend("  {%d, %d, %d, %d}," % v[:4] for v in V)
    out.append("};")
    out.append("static const double kPlanVmR[kPlanValueTerms] = {" + ", ".join(_lit(v[4]) for v in V) + "};")
    out.append("static const int kPlanCn[kPlanCoeffs] = {" + ", ".join(str(x) for x in CN) + "};")
    out.append("static const double kPlanCc[kPlanCoeffs] = {" + ", ".join(_lit(x) for x in CC) + "};")
    out.append("static const double kPlanRadii[kPlanNumRadii] = {" + ", ".join(_lit(x) for x in RAD) + "};")
    out.append("")
    out.extend(emit_quad())
    out.extend(emit_cheb32())
    out.extend(emit_disk())
    out.extend(emit_radial())
    out.extend(emit_mesh())
    out.extend(emit_triangle())
    out.append("}  // namespace wsb")
    out.append("")
    return "\n".join(out)


def chebyshev(coeffs, R):
    """exact Chebyshev coefficients b_k of the polynomial sum_n coeffs[n] r^n on [0, R], x = 2 r / R - 1:
    p(r) = sum_k b_k T_k(x).  Power basis in x first (r = R (x + 1) / 2), then x^n = 2^(1 - n) sum_j C(n, j) T_(n-2j)
    with the T_0 term halved."""
    R = F(R)
    deg = len(coeffs) - 1
    px = [F(0)] * (deg + 1)
    for n, c in enumerate(coeffs):
        if c:
            f = F(c) * (R / 2) ** n
            for k in range(n + 1):
                px[k] += f * comb(n, k)
    b = [F(0)] * (deg + 1)
    for n, a in enumerate(px):
        if not a:
            continue
        for j in range(n // 2 + 1):
            k = n - 2 * j
            w = F(1) if n == 0 else F(comb(n, j), 2 ** (n - 1))
            if k == 0 and n > 0:
                w /= 2
            b[k] += a * w
    return b


CHEB_PROFILES = ("c", "psi", "flam", "fpsi", "m", "mpsi")   # the four chord integrands, then the two potentials
F32_GAUSS = 8                                               # Gauss-Legendre nodes per panel of the float route


def emit_cheb32() -> list:
    """float Chebyshev tables of every exact kernel's block profiles on [0, R] (the float route of the 2-D channels):
    P, Psi, M/r^2, MPsi/r^2 (integrated along the chord by Gauss-Legendre) and the potentials M, MPsi (whose
    differences are the odd chord integrals).  Chebyshev coefficients of a bounded profile stay bounded, so Clenshaw's
    recurrence evaluates them in float to a few ulp of the profile's scale, where the monomial coefficients (up to
    ~1e4) would cancel."""
    import numpy as np
    gx, gw = np.polynomial.legendre.leggauss(F32_GAUSS)
    out = ["// ---- float Chebyshev tables of the block profiles on [0, R] (x = 2 r / R - 1), Clenshaw in float",
           f"constexpr int kF32Gauss = {F32_GAUSS};   // Gauss-Legendre nodes per panel of the float route",
           "static __device__ const float kF32Gx[kF32Gauss] = {" + ", ".join(repr(float(v)) + "f" for v in gx) + "};",
           "static __device__ const float kF32Gw[kF32Gauss] = {" + ", ".join(repr(float(v)) + "f" for v in gw) + "};",
           "template <class KT> struct ChebOf;   // the float tables of an exact kernel"]

    def clenshaw(cb, dst):
        cb = list(cb)
        while len(cb) > 1 and cb[-1] == 0:
            cb.pop()
        lit = lambda v: repr(float(v)) + "f"
        if len(cb) == 1:
            return [f"  {dst} = {lit(cb[0])};"]
        lines = ["  {", "    float b1 = 0.0f, b2 = 0.0f, t;"]
        for k in range(len(cb) - 1, 0, -1):
            lines.append(f"    t = fmaf(x2, b1, {lit(cb[k])} - b2); b2 = b1; b1 = t;")
        lines.append(f"    {dst} = fmaf(x, b1, {lit(cb[0])} - b2);")
        lines.append("  }")
        return lines

    for name, kid in sorted(KERNEL_IDS.items(), key=lambda t: t[1]):
        k = kernel(name)
        out.append(f"struct Cheb_{name} {{")
        out.append("  static constexpr double kMhat[] = {" + ", ".join(_lit(b.Mhat) for b in k.blocks) + "};")
        out.append("  static constexpr double kMPhat[] = {" + ", ".join(_lit(b.MPhat) for b in k.blocks) + "};")
        out.append("  template <int B> __device__ static __forceinline__ void integrands(float x, float& P, float& Psi, "
                   "float& Fl, float& Fp);")
        out.append("  template <int B> __device__ static __forceinline__ void potentials(float x, float& M, float& Mp);")
        out.append("};")
        out.append(f"template <> struct ChebOf<Kern_{name}> : Cheb_{name} {{}};")
        for bi, b in enumerate(k.blocks):
            cheb = {pn: chebyshev(getattr(b, pn), b.R) for pn in CHEB_PROFILES}
            out.append(f"template <> __device__ __forceinline__ void Cheb_{name}::integrands<{bi}>(float x, float& P, "
                       "float& Psi, float& Fl, float& Fp) {")
            out.append("  const float x2 = 2.0f * x;")
            for pn, dst in (("c", "P"), ("psi", "Psi"), ("flam", "Fl"), ("fpsi", "Fp")):
                out.extend(clenshaw(cheb[pn], dst))
            out.append("}")
            out.append(f"template <> __device__ __forceinline__ void Cheb_{name}::potentials<{bi}>(float x, float& M, "
                       "float& Mp) {")
            out.append("  const float x2 = 2.0f * x;")
            for pn, dst in (("m", "M"), ("mpsi", "Mp")):
                out.extend(clenshaw(cheb[pn], dst))
            out.append("}")
    out.append("")
    return out


def emit_disk() -> list:
    """the disk element's profiles per exact kernel id as literal code: disk_profile<KID>(r) gives P = pi*W, the value
    potential M(r)/r^2 (M = int_0^r t P dt) and the second potential MPsi(r)/r^2 + sum M(R)/2 summed over the
    truncated blocks (a block past its radius R continues as M(R)/r^2 and MPsi(R)/r^2), and disk_knots<KID> the
    block radii below 1 (where the profiles have kinks)."""
    out = ["// ---- disk element: pi*W, M/r^2 and the second potential of every exact kernel, summed over its blocks",
           "template <int KID> __device__ __forceinline__ void disk_profile(double r, double ir2, double& P, double& Fl,",
           "                                                             double& F2l);",
           "template <int KID> __device__ __forceinline__ int disk_knots(double* out);"]
    for kid in range(len(KERNEL_IDS)):
        k = kernel(KERNEL_NAMES[kid])
        half = sum((b.Mhat for b in k.blocks), F(0)) / 2
        body = [f"template <> __device__ __forceinline__ void disk_profile<{kid}>(double r, double ir2, double& P, "
                f"double& Fl, double& F2l) {{   // {k.name}",
                f"  P = 0.0;", f"  Fl = 0.0;", f"  F2l = {_lit(half)};"]
        for b in k.blocks:
            body.append(f"  if (r <= {_lit(b.R)}) {{")
            body.append(f"    P += {_horner(b.c, 'r')};")
            body.append(f"    Fl += {_horner(b.flam, 'r')};")
            body.append(f"    F2l += {_horner(b.fpsi, 'r')};")
            body.append("  } else {")
            body.append(f"    Fl += {_lit(b.Mhat)} * ir2;")
            body.append(f"    F2l += {_lit(b.MPhat)} * ir2;")
            body.append("  }")
        body.append("}")
        knots = sorted(b.R for b in k.blocks if b.R < 1)
        body.append(f"template <> __device__ __forceinline__ int disk_knots<{kid}>(double* out) {{")
        for j, R in enumerate(knots):
            body.append(f"  out[{j}] = {_lit(R)};")
        body.append(f"  return {len(knots)};")
        body.append("}")
        out.extend(body)
    out.append(f"constexpr int kDiskMaxKnots = {max(1, max(sum(1 for b in kernel(n).blocks if b.R < 1) for n in KERNEL_IDS))};")
    out.append("// pi*W and its derivative (the far-field rule of the finite-element pair weights)")
    out.append("template <int KID> __device__ __forceinline__ void pi_w_deriv(double r, double& P, double& dP);")
    for kid in range(len(KERNEL_IDS)):
        k = kernel(KERNEL_NAMES[kid])
        out.append(f"template <> __device__ __forceinline__ void pi_w_deriv<{kid}>(double r, double& P, double& dP) {{")
        out.append("  P = 0.0;")
        out.append("  dP = 0.0;")
        for b in k.blocks:
            der = [c * (i + 1) for i, c in enumerate(b.c[1:])] or [F(0)]
            out.append(f"  if (r <= {_lit(b.R)}) {{")
            out.append(f"    P += {_horner(b.c, 'r')};")
            out.append(f"    dP += {_horner(der, 'r')};")
            out.append("  }")
        out.append("}")
    gx, gw = __import__("numpy").polynomial.legendre.leggauss(8)
    out.append("constexpr int kFemGauss = 8;   // nodes per direction of the far-field rule, on [0, 1]")
    out.append("static __device__ const double kFemGx[kFemGauss] = {" + ", ".join(repr(float((x + 1) / 2)) for x in gx) + "};")
    out.append("static __device__ const double kFemGw[kFemGauss] = {" + ", ".join(repr(float(w / 2)) for w in gw) + "};")
    out.append("")
    return out


# the Wendland C2 / C4 shapes in u = 1 - q (src/warpSPHBoundaries/edge/kernels.py:217-219): u^p0 B(u)
_POWER_FAMILIES = {"w2": (4, [F(5), F(-4)]), "w4": (6, [F(56, 3), F(-88, 3), F(35, 3)])}


@lru_cache(maxsize=None)
def quad_kernel(name: str):
    """(C2*pi, p, B) of a powered kernel: `w2p5` / `w4p5` = the 5th power of the Wendland C2 / C4 shape
    (src/warpSPHBoundaries/edge/kernels.py:214-232, registered by scene/tensile.py:40-47), pi*W = C u^p B(u)^5 with
    u = 1 - r, p = 5 p0, B the family's base in u; normalised by the rule C = 1 / (2 int_0^1 r shape dr) of
    edge/kernels.py:141-156.  Every factor is positive on r <= 1, so the factored form is accurate to a few ulp where
    the monomial expansion (coefficients up to ~1e13 for w4p5) cancels."""
    if name not in QUAD_KERNEL_IDS:
        raise KeyError(f"unknown powered kernel {name!r}; expected one of {sorted(QUAD_KERNEL_IDS)}")
    fam = name[:2]
    p0, base = _POWER_FAMILIES[fam]
    (lo, hi, shape), = _pieces(fam)
    # the u-form equals the q-form of the smoothing kernel's shape: u^p0 B(u) expanded in q
    u = [F(1), F(-1)]
    bq = [F(0)]
    for k, c in enumerate(base):
        bq = _padd(bq, [c * x for x in _ppow(u, k)])
    if _trim(_pmul(_ppow(u, p0), bq)) != _trim(list(shape)):
        raise AssertionError(f"{fam}: the u-form of the shape differs from its q-form")
    s5 = _ppow(shape, 5)
    C = 1 / (2 * _shape_integral([(F(0), F(1), s5)]))
    return C, 5 * p0, tuple(base)


def pi_w_quad(name, r: F) -> F:
    """exact pi * W(r) of a powered kernel (h = 1, r <= 1; tests)."""
    C, p, base = quad_kernel(name)
    u = 1 - r
    return C * u ** p * sum(c * u ** k for k, c in enumerate(base)) ** 5


def emit_quad() -> list:
    """the powered kernels as quadrature kernels: pi*W(r) in the factored form, and the Gauss-Legendre rule of the
    chord panels."""
    import numpy as np
    gx, gw = np.polynomial.legendre.leggauss(QUAD_GAUSS)
    fx, fw = np.polynomial.legendre.leggauss(QUAD_GAUSS_FAR)
    cx, cw = np.polynomial.legendre.leggauss(QUAD_GAUSS_CHORD)
    out = ["// x^N by squaring",
           "template <int N>",
           "__host__ __device__ __forceinline__ double qpow(double x) {",
           "  if constexpr (N == 0) {",
           "    return 1.0;",
           "  } else if constexpr (N % 2 == 0) {",
           "    const double y = qpow<N / 2>(x);",
           "    return y * y;",
           "  } else {",
           "    return x * qpow<N - 1>(x);",
           "  }",
           "}",
           f"constexpr int kQuadGauss = {QUAD_GAUSS};",
           "static __device__ const double kQuadGx[kQuadGauss] = {" + ", ".join(repr(float(x)) for x in gx) + "};",
           "static __device__ const double kQuadGw[kQuadGauss] = {" + ", ".join(repr(float(x)) for x in gw) + "};",
           f"constexpr int kQuadGaussFar = {QUAD_GAUSS_FAR};",
           "static __device__ const double kQuadFx[kQuadGaussFar] = {" + ", ".join(repr(float(x)) for x in fx) + "};",
           "static __device__ const double kQuadFw[kQuadGaussFar] = {" + ", ".join(repr(float(x)) for x in fw) + "};",
           f"constexpr int kQuadGaussChord = {QUAD_GAUSS_CHORD};",
           "static __device__ const double kQuadCx[kQuadGaussChord] = {" + ", ".join(repr(float(x)) for x in cx) + "};",
           "static __device__ const double kQuadCw[kQuadGaussChord] = {" + ", ".join(repr(float(x)) for x in cw) + "};",
           ""]
    for name, kid in sorted(QUAD_KERNEL_IDS.items(), key=lambda t: t[1]):
        C, p, base = quad_kernel(name)
        out.append(f"// ---- {name}: C2*pi = {C}; pi*W = C u^{p} B(u)^5, u = 1 - r, on r <= 1")
        out.append(f"struct Kern_{name} {{")
        out.append(f"  static constexpr int kId = {kid};")
        out.append("  static constexpr bool kQuad = true;")
        out.append("  static constexpr int kBlocks = 1;")
        out.append("  static constexpr double kR[kBlocks] = {1.0};")
        out.append("  static constexpr int kNA[kBlocks] = {1};")
        out.append("  static constexpr double kMass = 1.0;")
        out.append("  static constexpr double kPlane2 = 0.0;")
        out.append("  __host__ __device__ static __forceinline__ double poly(double r) {")
        out.append("    const double u = 1.0 - r;")
        out.append(f"    const double b = {_horner(list(base), 'u')};")
        out.append("    const double b2 = b * b;")
        out.append(f"    return {_lit(C)} * qpow<{p}>(u) * (b2 * b2 * b);")
        out.append("  }")
        out.append("};")
        out.append("")
    return out


def plane_channels(name):
    """the twelve channel values of a solid that covers the whole support (indicator 1), h = 1:
    lam = 1, g1 diagonal = 1, m20 = m02 = plane second moment; zero elsewhere."""
    k = kernel(name)
    m, p2 = float(k.mass), float(k.plane2)
    return [m, 0.0, 0.0, 0.0, 0.0, m, 0.0, 0.0, m, p2, 0.0, p2]


# ------------------------------------------------------------------ 3-D radial profiles (solid half-space / sphere)
RADIAL_KERNELS = ("cubic", "w2", "w4", "w6")
_PUBLISHED_C3PI = {"cubic": F(16), "w2": F(21, 2), "w4": F(495, 32), "w6": F(1365, 64)}
# Gauss-Legendre order of every radial sub-interval: exact for polynomial integrands up to degree 2 * 12 - 1 = 23
# (the highest is r^4 W a_t of w6, degree 18); cubic's outer Laurent piece lives on r >= 1/2, where 12 nodes leave a
# relative error below 1e-17.
RADIAL_GAUSS = 12


@dataclass(frozen=True)
class RadialProfile:
    """f(r) = r^p (hi - r)^k g(r) with g a polynomial; exact rational coefficients."""
    p: int
    k: int
    g: Tuple[F, ...]

    def __call__(self, r: F) -> F:
        return F(r) ** self.p * (self.hi - F(r)) ** self.k * _peval(list(self.g), F(r)) if self.k else \
            F(r) ** self.p * _peval(list(self.g), F(r))


def _factor_laurent(terms, hi):
    """{n: c} (n may be negative) -> (p, k, g) with f = r^p (hi - r)^k g(r), (hi - r) divided out while g(hi) = 0."""
    terms = {n: c for n, c in terms.items() if c}
    p = min(terms)
    g = [F(0)] * (max(terms) - p + 1)
    for n, c in terms.items():
        g[n - p] = c
    k = 0
    while len(g) > 1 and _peval(g, hi) == 0:
        # synthetic division by (hi - r) = -(r - hi): g = (r - hi) q  ->  g = (hi - r) (-q)
        q = [F(0)] * (len(g) - 1)
        acc = F(0)
        for i in range(len(g) - 1, 0, -1):
            acc = acc * hi + g[i]
            q[i - 1] = acc
        g = [-x for x in q]
        k += 1
    return p, k, tuple(_trim(g))


@lru_cache(maxsize=None)
def radial(name: str):
    """the 3-D radial tables of `name` (unit support): [(lo, hi, W, L, dL)] with W = c3pi * shape (the 3-D kernel
    times pi), L = W'/r and dL = L' as RadialProfile in r, and c3pi (checked against the published constant)."""
    if name not in RADIAL_KERNELS:
        raise KeyError(f"radial family: kernel {name!r} not in {RADIAL_KERNELS}")
    raw = _pieces(name)
    tot = F(0)
    for lo, hi, c in raw:
        P = [F(0)] * 3 + [x / (i + 3) for i, x in enumerate(c)]
        tot += _peval(P, hi) - _peval(P, lo)
    c3pi = 1 / (4 * tot)
    if c3pi != _PUBLISHED_C3PI[name]:
        raise AssertionError(f"3-D normalisation of {name}: {c3pi} != published {_PUBLISHED_C3PI[name]}")
    out = []
    for lo, hi, c in raw:
        w = {n: c3pi * x for n, x in enumerate(c)}
        ell = {n - 2: n * x for n, x in w.items() if n >= 1}
        dell = {n - 1: n * x for n, x in ell.items() if n != 0}
        out.append((lo, hi, *(RadialProfile(*_factor_laurent(t, hi)) for t in (w, ell, dell))))
    return tuple(out), c3pi


# ------------------------------------------------------------------ 3-D closed surfaces (face -> edge reductions)
MESH_FUNCS = ("A_K0", "A_K1", "A_K2", "A_W", "A_L", "A2_K2")


def _leval(d, x):
    """value of the Laurent polynomial {exponent: coefficient} at x (x > 0 wherever a negative exponent is used)."""
    return sum((c * F(x) ** e for e, c in d.items() if c), F(0))


def _compact_potential(bounds, fp):
    """per piece the Laurent polynomial A_p with A' = r f and A(r) = -int_r^1 t f(t) dt (zero from r = 1 on)."""
    prims = []
    for f in fp:
        prim = {}
        for n, c in f.items():
            if n + 2 == 0:
                raise AssertionError("logarithmic term in a compact potential")
            prim[n + 2] = prim.get(n + 2, F(0)) + c / (n + 2)
        prims.append(prim)
    out = []
    for p, ((lo, hi), prim) in enumerate(zip(bounds, prims)):
        tail = sum((_leval(prims[q], bounds[q][1]) - _leval(prims[q], bounds[q][0]) for q in range(p + 1, len(bounds))),
                   F(0))
        d = dict(prim)
        d[0] = d.get(0, F(0)) - _leval(prim, hi) - tail
        out.append({e: c for e, c in d.items() if c})
    return out


@lru_cache(maxsize=None)
def mesh_tables(name: str):
    """exact tables of the closed-surface reduction of `name` (unit support, W~ = c3*pi * shape = pi * W):
    {"bounds": [(lo, hi)] per piece, "Q": (Q0(1), Q1(1), Q2(1)) with Q_k(r) = int_0^r t^(2+k) W~ dt,
     "funcs": {name: [Laurent dict per piece]} for the compact potentials
        A_K0, A_K1, A_K2  of K_k(r) = (Q_k(r) - Q_k(1)) / r^(3+k)   (volume potentials of the value moments),
        A_W, A_L          of W~ and L = W~'/r,
        A2_K2             of r -> A_K2(r) (the trace term of the in-plane second moment)}."""
    raw = _pieces(name)
    c3pi = radial(name)[1]
    bounds = [(lo, hi) for lo, hi, _ in raw]
    Wp = [{n: c3pi * c for n, c in enumerate(co) if c} for _, _, co in raw]
    Lp = [{n - 2: n * c for n, c in w.items() if n >= 1} for w in Wp]
    Q, K = [], []
    for k in range(3):
        pieces, acc = [], F(0)
        for (lo, hi), w in zip(bounds, Wp):
            prim = {n + 3 + k: c / (n + 3 + k) for n, c in w.items()}
            d = dict(prim)
            d[0] = d.get(0, F(0)) + acc - _leval(prim, lo)
            pieces.append(d)
            acc += _leval(prim, hi) - _leval(prim, lo)
        Q.append(acc)
        Kk = []
        for d in pieces:
            kd = {}
            for e, c in d.items():
                kd[e - 3 - k] = kd.get(e - 3 - k, F(0)) + c
            kd[-3 - k] = kd.get(-3 - k, F(0)) - acc
            Kk.append({e: c for e, c in kd.items() if c})
        K.append(Kk)
    funcs = {"A_K0": _compact_potential(bounds, K[0]), "A_K1": _compact_potential(bounds, K[1]),
             "A_K2": _compact_potential(bounds, K[2]), "A_W": _compact_potential(bounds, Wp),
             "A_L": _compact_potential(bounds, Lp)}
    funcs["A2_K2"] = _compact_potential(bounds, funcs["A_K2"])
    for fname, pcs in funcs.items():
        negs = {e for d in pcs for e in d if e < 0}
        if len(negs) > 1:
            raise AssertionError(f"{name} {fname}: more than one negative power {negs}")
    return {"bounds": bounds, "Q": tuple(Q), "funcs": funcs}


def mesh_negative_power(name, fname):
    pcs = mesh_tables(name)["funcs"][fname]
    negs = {e for d in pcs for e in d if e < 0}
    return -min(negs) if negs else 0


def _emit_dd(coeffs, x, a):
    """C++ statements computing (P(x) - P(a)) / (x - a) into `dd` for P = sum coeffs[n] x^n (n >= 0): the synthetic
    division by (x - a) evaluated by Horner's rule, no cancellation between P(x) and P(a)."""
    cs = list(coeffs)
    while len(cs) > 1 and cs[-1] == 0:
        cs.pop()
    D = len(cs) - 1
    if D < 1:
        return ["dd = 0.0;"]
    out = [f"double b = {_lit(cs[D])}; dd = b;"]
    for j in range(D - 2, -1, -1):
        out.append(f"b = fma({a}, b, {_lit(cs[j + 1])}); dd = fma(dd, {x}, b);")
    return out


def emit_mesh() -> list:
    """generated device code of the closed-surface family: per kernel and compact potential the polynomial part's value
    and divided difference per piece, the negative power and its coefficient."""
    import numpy as np
    x8, w8 = np.polynomial.legendre.leggauss(8)
    out = ["// ---- 3-D closed surfaces: compact potentials (unit support, W~ = c3*pi * shape); function ids:",
           "//      0 A_K0, 1 A_K1, 2 A_K2, 3 A_W, 4 A_L, 5 A2_K2",
           "template <class M, int Fn> struct MeshFn;",
           "static __device__ const double kMeshGx8[8] = {" + ", ".join(repr(float(x)) for x in x8) + "};",
           "static __device__ const double kMeshGw8[8] = {" + ", ".join(repr(float(x)) for x in w8) + "};"]
    for name in RADIAL_KERNELS:
        t = mesh_tables(name)
        bounds = t["bounds"]
        out.append(f"struct Mesh_{name} {{")
        out.append(f"  static constexpr int kPieces = {len(bounds)};")
        out.append(f"  static constexpr double kBreak = {_lit(bounds[0][1]) if len(bounds) > 1 else '2.0'};   // end of the inner piece")
        out.append(f"  static constexpr double kQ0 = {_lit(t['Q'][0])}, kQ1 = {_lit(t['Q'][1])}, kQ2 = {_lit(t['Q'][2])};")
        out.append("};")
        for fi, fname in enumerate(MESH_FUNCS):
            pcs = t["funcs"][fname]
            m = mesh_negative_power(name, fname)
            out.append(f"template <> struct MeshFn<Mesh_{name}, {fi}> {{   // {fname}")
            out.append(f"  static constexpr int kNeg = {m};")
            for p, d in enumerate(pcs):
                poly = [d.get(n, F(0)) for n in range(max([e for e in d if e >= 0], default=0) + 1)]
                nu = d.get(-m, F(0)) if m else F(0)
                out.append(f"  static constexpr double kNu{p} = {_lit(nu)};")
                out.append(f"  __host__ __device__ static __forceinline__ double poly{p}(double x) {{ return {_horner(poly, 'x')}; }}")
                body = " ".join(_emit_dd(poly, "x", "a"))
                out.append(f"  __host__ __device__ static __forceinline__ double dd{p}(double x, double a) {{ double dd; {body} return dd; }}")
                # the same divided difference in two halves: the synthetic-division coefficients b (they depend on a
                # only, so a caller forms them once per a) and Horner's rule over b at x -- the same fma sequence
                cs = list(poly)
                while len(cs) > 1 and cs[-1] == 0:
                    cs.pop()
                D = len(cs) - 1
                out.append(f"  static constexpr int kDD{p} = {max(D, 0)};")
                if D >= 1:
                    bs = [f"b[0] = {_lit(cs[D])};"] + [f"b[{k}] = fma(a, b[{k - 1}], {_lit(cs[D - k])});"
                                                       for k in range(1, D)]
                    hs = ["double dd = b[0];"] + [f"dd = fma(dd, x, b[{k}]);" for k in range(1, D)]
                else:
                    bs, hs = [], ["double dd = 0.0;"]
                out.append(f"  __host__ __device__ static __forceinline__ void ddb{p}(double a, double* b) {{ {' '.join(bs)} }}")
                out.append(f"  __host__ __device__ static __forceinline__ double ddh{p}(double x, const double* b) {{ {' '.join(hs)} return dd; }}")
            out.append("};")
    out.append("")
    return out


def _radial_eval(prof, var, hi_lit, T):
    """C++ expression of a RadialProfile at `var` in type T."""
    g = list(prof.g)
    expr = f"T({_lit(g[-1])})"
    for x in reversed(g[:-1]):
        expr = f"fma_t({expr}, {var}, T({_lit(x)}))" if x != 0 else f"({expr} * {var})"
    fac = []
    if prof.k:
        fac.append(f"ipow<{prof.k}>(T({hi_lit}) - {var})")
    if prof.p > 0:
        fac.append(f"ipow<{prof.p}>({var})")
    if prof.p < 0:
        fac.append(f"(T(1) / ipow<{-prof.p}>({var}))")
    return " * ".join([f"({expr})"] + fac)


# ------------------------------------------------------------------ 2-D conditioned triangles (area quadrature)
TRIANGLE_KERNELS = ("cubic", "w2", "w4", "w6", "poly6")


def triangle_profiles(name):
    """per piece of the 2-D kernel (pi W, unit support): (lo, hi, W, rho) with rho = -W'/r, both as RadialProfile
    r^p (hi - r)^k g(r) (exact factors keep the values accurate where W is small)."""
    if name not in TRIANGLE_KERNELS:
        raise KeyError(f"conditioned triangles: kernel {name!r} not in {TRIANGLE_KERNELS} (at most two radii)")
    out = []
    for lo, hi, co in kernel(name).pieces:
        w = {n: c for n, c in enumerate(co) if c}
        rho = {n - 2: -n * c for n, c in w.items() if n >= 1}
        out.append((lo, hi, RadialProfile(*_factor_laurent(w, hi)), RadialProfile(*_factor_laurent(rho, hi))))
    return out


def emit_triangle() -> list:
    """generated device code of the conditioned-triangle quadrature: per kernel the pieces and W, -W'/r."""
    import numpy as np
    x16, w16 = np.polynomial.legendre.leggauss(16)
    x8, w8 = np.polynomial.legendre.leggauss(8)
    out = ["// ---- 2-D conditioned triangles: pi W and rho = -pi W'/r per piece (unit support)",
           "static __device__ const double kTriGx16[16] = {" + ", ".join(repr(float(x)) for x in x16) + "};",
           "static __device__ const double kTriGw16[16] = {" + ", ".join(repr(float(x)) for x in w16) + "};",
           "static __device__ const double kTriGx8[8] = {" + ", ".join(repr(float(x)) for x in x8) + "};",
           "static __device__ const double kTriGw8[8] = {" + ", ".join(repr(float(x)) for x in w8) + "};"]
    for name in TRIANGLE_KERNELS:
        pcs = triangle_profiles(name)
        out.append(f"struct Tri_{name} {{")
        out.append(f"  static constexpr int kPieces = {len(pcs)};")
        out.append(f"  static constexpr double kPlane2 = {_lit(kernel(name).plane2)};   // int_plane y_x^2 W")
        out.append(f"  static constexpr double kKnot = {_lit(pcs[0][1]) if len(pcs) > 1 else '2.0'};   // end of the inner piece")
        out.append("  template <int P> __host__ __device__ static __forceinline__ void eval(double r, double& w, double& rho);")
        out.append("};")
        for i, (lo, hi, W, rho) in enumerate(pcs):
            out.append(f"template <> __host__ __device__ __forceinline__ void Tri_{name}::eval<{i}>(double r, double& w, double& rho) {{")
            out.append("  using T = double;")
            out.append(f"  w = {_radial_eval(W, 'r', _lit(hi), 'T')};")
            out.append(f"  rho = {_radial_eval(rho, 'r', _lit(hi), 'T')};")
            out.append("}")
    out.append("")
    return out


def emit_radial() -> list:
    """generated device code of the radial family: per kernel the pieces and W, W'/r, (W'/r)' in factored form."""
    import numpy as np
    xg, wg = np.polynomial.legendre.leggauss(RADIAL_GAUSS)
    out = ["// ---- 3-D radial family (solid half-space / sphere), unit support; W = c3*pi * shape, L = W'/r, dL = L'",
           "template <int K, typename T>",
           "__host__ __device__ __forceinline__ T ipow(T x) {",
           "  T y = x;",
           "#pragma unroll",
           "  for (int i = 1; i < K; ++i) y *= x;",
           "  return y;",
           "}",
           "__host__ __device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }",
           "__host__ __device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }",
           f"constexpr int kRadialGauss = {RADIAL_GAUSS};",
           "static __device__ const double kRadialGx[kRadialGauss] = {" + ", ".join(repr(float(x)) for x in xg) + "};",
           "static __device__ const double kRadialGw[kRadialGauss] = {" + ", ".join(repr(float(x)) for x in wg) + "};"]
    for name in RADIAL_KERNELS:
        pcs, c3pi = radial(name)
        out.append(f"struct Rad_{name} {{   // c3*pi = {c3pi}")
        out.append(f"  static constexpr int kPieces = {len(pcs)};")
        out.append("  static constexpr double kLo[kPieces] = {" + ", ".join(_lit(p[0]) for p in pcs) + "};")
        out.append("  static constexpr double kHi[kPieces] = {" + ", ".join(_lit(p[1]) for p in pcs) + "};")
        # whole-support constants (the region of the support inside the solid is the full ball)
        full = _radial_full(name)
        out.append("  template <typename T> __host__ __device__ static __forceinline__ void full(T* v) {")
        out.append("    " + " ".join(f"v[{j}] = T({_lit(x)});" for j, x in enumerate(full)))
        out.append("  }")
        out.append("  template <int P, typename T> __host__ __device__ static __forceinline__ void eval(T r, T& w, T& l, T& dl);")
        out.append("};")
        for i, (lo, hi, W, L, dL) in enumerate(pcs):
            out.append(f"template <> __host__ __device__ __forceinline__ void Rad_{name}::eval<{i}, double>(double r, double& w, double& l, double& dl) {{")
            out.append("  using T = double;")
            for var, prof in (("w", W), ("l", L), ("dl", dL)):
                out.append(f"  {var} = {_radial_eval(prof, 'r', _lit(hi), 'T')};")
            out.append("}")
            out.append(f"template <> __host__ __device__ __forceinline__ void Rad_{name}::eval<{i}, float>(float r, float& w, float& l, float& dl) {{")
            out.append("  using T = float;")
            for var, prof in (("w", W), ("l", L), ("dl", dL)):
                out.append(f"  {var} = {_radial_eval(prof, 'r', _lit(hi), 'T')};")
            out.append("}")
    out.append("")
    return out


def _radial_full(name):
    """the nine invariants (unit support, /pi folded) of a query whose whole support lies inside the solid."""
    pcs, _ = radial(name)
    def integral(prof_idx, power):
        tot = F(0)
        for lo, hi, *profs in pcs:
            prof = profs[prof_idx]
            # exact integral of r^power * prof over [lo, hi] by expanding prof into a Laurent polynomial
            poly = list(prof.g)
            if prof.k:
                poly = _pmul(poly, _ppow([hi, F(-1)], prof.k))
            for n, c in enumerate(poly):
                e = n + prof.p + power
                if c == 0:
                    continue
                if e == -1:
                    raise AssertionError("log term in a whole-support constant")
                tot += c * (hi ** (e + 1) - lo ** (e + 1)) / (e + 1)
        return tot
    w2, w4 = integral(0, 2), integral(0, 4)
    l4, l2, dl3 = integral(1, 4), integral(1, 2), integral(2, 3)
    return [4 * w2, F(0), F(4, 3) * w4, F(4, 3) * w4, F(0), -F(4, 3) * l4, -F(4, 3) * l4,
            4 * l2 + F(4, 3) * dl3, 4 * l2 + F(4, 3) * dl3]


if __name__ == "__main__":       # python -m warpsphboundaries_b200.kernels  -> regenerate the header
    import pathlib
    p = pathlib.Path(__file__).parent / "csrc" / "kernel_tables.h"
    p.write_text(emit_header())
    print("wrote", p)


# ------------------------------------------------------------------ algorithmic work per pair
def _horner_flops(coeffs):
    cs = list(coeffs)
    while len(cs) > 1 and cs[-1] == 0:
        cs.pop()
    low = 0
    while low < len(cs) - 1 and cs[low] == 0:
        low += 1
    return 2 * (len(cs) - 1 - low) + low          # one FMA per Horner step, one multiply per power factor


def pair_work(name):
    """algorithmic float64 work of one (particle, edge) neighbour pair in the closed form of the fused route, counted
    from the formulas it evaluates (FMA = 2 flops; add, sub, mul = 1): {"flops": F, "sqrt": .., "div": .., "log": ..,
    "atan2": ..} with every block's chord present (the work of a pair whose chords are all non-empty)."""
    k = kernel(name)
    flops = 2 + 3 + 2 + 3 + 4 + 4 + 4          # d, |d|^2, t, cross, s0, s1, relative vertices
    sq, dv, lg, at = 1, 6, 0, 0                  # |d|, 1/ell, z/ell, four (v - x)/h
    for b in k.blocks:
        na = max(len(b.psi), len(b.fpsi), len(b.c))
        flops += 3 + 1 + 4 + 3 + 4 + 1 + 6 + 9 * max(na - 2, 0)    # chord, zz, r_lo/r_hi, log args, angle args, A_0, A_1, A_n
        sq += 3
        dv += 1
        lg += 1
        at += 1
        nz = lambda a: sum(1 for c in a if c != 0)
        flops += (2 * nz(b.c) - 1) + (2 * nz(b.psi) - 1) + (2 * nz(b.flam) - 1) + (2 * nz(b.fpsi) - 1)
        flops += 2 * _horner_flops(b.m) + 1 + 2 * _horner_flops(b.mpsi) + 1
        flops += 50                                                  # the two value terms and the twelve accumulations
    return {"flops": flops, "sqrt": sq, "div": dv, "log": lg, "atan2": at}
