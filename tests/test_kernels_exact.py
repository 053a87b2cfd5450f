"""The package's exact kernel algebra (kernel tables compiled into the CUDA header) against the oracle's."""
from fractions import Fraction as F

import pytest

from oracle import edge2d as O
from warpsphboundaries_b200 import kernels as K

NAMES = ["cubic", "w2", "w4", "w6", "quartic", "quintic", "poly6"]


@pytest.mark.parametrize("name", NAMES)
def test_blocks_equal_oracle(name):
    k = K.kernel(name)
    ob = O.blocks(name)
    assert len(k.blocks) == len(ob)
    for b, (R, P) in zip(k.blocks, ob):
        assert b.R == R
        assert {n: c for n, c in enumerate(b.c) if c != 0} == P


@pytest.mark.parametrize("name", NAMES)
def test_derived_profiles(name):
    """M' = r P, Psi(R) = 0, the value profiles, and the whole-plane constants."""
    k = K.kernel(name)
    assert k.mass == 1
    for b in k.blocks:
        assert K._peval(list(b.psi), b.R) == 0
        for n, c in enumerate(b.c):
            assert b.m[n + 2] == c / (n + 2) if n + 2 < len(b.m) else c == 0
        assert b.Mhat == K._peval(list(b.m), b.R)
    mass, plane2 = O.kernel_mass_and_plane(name)
    assert k.plane2 == plane2


@pytest.mark.parametrize("name", NAMES)
def test_term_plan_equals_oracle_plan(name):
    tp = K.term_plan(name)
    E, V = O.plan(name)
    assert len(tp.E) == len(E) and len(tp.V) == len(V)
    for (ch, i, a, b, Ri, c0, c1), (och, oi, (oa, ob), oR, oP) in zip(tp.E, E):
        assert (ch, i, a, b, tp.radii[Ri]) == (och, oi, oa, ob, float(oR))
        assert [(n, c) for n, c in zip(tp.cn[c0:c1], tp.cc[c0:c1])] == [(n, float(c)) for n, c in sorted(oP.items())]
    for (ch, Ri, c0, c1, mR), (och, oR, oQ, omR) in zip(tp.V, V):
        assert (ch, tp.radii[Ri], mR) == (och, float(oR), float(omR))


def test_header_is_current():
    from pathlib import Path
    p = Path(K.__file__).parent / "csrc" / "kernel_tables.h"
    assert p.read_text() == K.emit_header(), "run python -m warpsphboundaries_b200.kernels"


def test_pi_w_normalised():
    for name in NAMES:
        assert K.pi_w(name, F(0)) == sum(b.c[0] for b in K.kernel(name).blocks)
        assert K.pi_w(name, F(2)) == 0
