"""Host logic of the radial family (no GPU): the request contract, argument checks, C-ABI argument errors."""
import ctypes

import numpy as np
import pytest

from oracle import radial as OR
from warpsphboundaries_b200 import _lib
from warpsphboundaries_b200.radial import RadialEvaluator, Request, baseline, monomials


def test_baseline_is_the_28_request_contract():
    b = baseline(3)
    assert len(b) == 28
    assert [(r.alpha, r.derivative) for r in b] == OR.baseline()
    assert len(baseline(2)) == 6 + 6 + 3
    assert monomials(2, 1) == ((0, 0), (1, 0), (0, 1))


def test_request_validation():
    with pytest.raises(ValueError):
        Request((1, 2, 3, 4))
    with pytest.raises(ValueError):
        Request((5, 5, 0))
    with pytest.raises(ValueError):
        Request((0, 0, 0), (3,))
    assert Request((1, 0, 1), (2,)).scale == 1


def test_evaluator_rejects_what_the_reference_rejects():
    with pytest.raises(ValueError):
        RadialEvaluator("cone")
    with pytest.raises(ValueError):
        RadialEvaluator("sphere", kernel="quintic")
    with pytest.raises(ValueError):
        RadialEvaluator("sphere", [Request((2, 1, 0))])
    with pytest.raises(ValueError):
        RadialEvaluator("sphere", precision="float16")
    with pytest.raises(RuntimeError):
        RadialEvaluator("sphere", device="cpu")
    ev = RadialEvaluator("sphere")
    n = [0.0, 0.0, 1.0]
    with pytest.raises(ValueError):
        ev.prepare([0.1], n, 1.0)                                  # no radii
    with pytest.raises(ValueError):
        ev.prepare([-2.0], n, 1.0, radii=1.0)                      # distance < -radius
    with pytest.raises(ValueError):
        ev.prepare([0.1], [0.0, 0.0, 2.0], 1.0, radii=1.0)         # not unit
    with pytest.raises(ValueError):
        ev.prepare([0.1], n, 0.0, radii=1.0)                       # support <= 0
    with pytest.raises(ValueError):
        ev.prepare([0.1], n, 1.0, radii=1e-5)                      # r/h below the domain
    with pytest.raises(ValueError):
        ev.prepare([0.1, 0.2], [[0, 0, 1.0]] * 3, 1.0, radii=1.0)  # shapes
    with pytest.raises(ValueError):
        RadialEvaluator("plane").prepare([0.1], n, 1.0, radii=1.0)
    with pytest.raises(ValueError):
        RadialEvaluator("plane", precision="float32").prepare([1e39], n, 1.0)


def test_abi_argument_errors():
    meta = (ctypes.c_int32 * 8)(0, 0, 0, 0, 1, 0, 0, 0)
    f = _lib.lib.wsb_radial_channels
    assert f(7, 1, 0, None, None, None, None, 4, meta, 2, None, None, None, None) == _lib.WSB_ERR_ARG
    assert f(0, 1, 0, None, None, None, None, 4, meta, 29, None, None, None, None) == _lib.WSB_ERR_ARG
    assert f(0, 5, 0, None, None, None, None, 4, meta, 2, None, None, None, None) == _lib.WSB_ERR_UNSUPPORTED
    assert f(0, 1, 1, None, None, None, None, 4, meta, 2, None, None, None, None) == _lib.WSB_ERR_UNSUPPORTED
    assert f(0, 1, 0, None, None, None, None, 4, meta, 2, None, None, None, None) == _lib.WSB_ERR_ARG   # NULL arrays
    bad = (ctypes.c_int32 * 4)(2, 0, 0, 1)
    assert f(0, 1, 0, None, None, None, None, 4, bad, 1, None, None, None, None) == _lib.WSB_ERR_ARG
    assert f(0, 1, 0, None, None, None, None, 0, meta, 2, None, None, None, None) == _lib.WSB_OK         # empty batch


def test_whole_support_constants_match_the_oracle():
    """exact constants vs the oracle's adaptive quadrature of monomial-form profiles (good to about 1e-11)."""
    from warpsphboundaries_b200 import kernels as K
    for name in K.RADIAL_KERNELS:
        full = np.array([float(x) for x in K._radial_full(name)])
        assert np.abs(full - OR.invariants(-1.5, name)).max() < 1e-10
        assert np.abs(full - OR.invariants(-1.0, name, radius=3.0)).max() < 1e-10
