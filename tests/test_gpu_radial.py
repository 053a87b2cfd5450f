"""Solid spheres and half-spaces (3-D) on the GPU through wsb_radial_channels, against the reference's 70-digit
fixtures and the oracle."""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import radial as OR

pytestmark = pytest.mark.gpu
G = json.loads((Path(__file__).parent / "golden" / "radial_golden.json").read_text())


def _f(xs):
    return np.array([float(x) for x in xs])


@pytest.mark.parametrize("precision,tol", [("float64", 1e-13), ("float32", 2e-5)])
def test_radial_fixture(precision, tol):
    from warpsphboundaries_b200.radial import RadialEvaluator
    worst = 0.0
    for kind in ("plane", "sphere"):
        for kernel in ("cubic", "w2", "w4", "w6"):
            cases = [c for c in G["radial"] if c["kind"] == kind and c["kernel"] == kernel]
            if precision == "float32":
                cases = [c for c in cases if c["radius"] is None or float(c["radius"]) >= 1e-2]
            if not cases:
                continue
            ev = RadialEvaluator(kind, kernel=kernel, precision=precision)
            d = _f([c["distance"] for c in cases])
            n = np.array([_f(c["normal"]) for c in cases])
            kw = {"radii": _f([c["radius"] for c in cases])} if kind == "sphere" else {}
            b = ev.prepare(d, n, 1.0, **kw)
            b.launch()
            inv = b.work.cpu().numpy()
            vals = b.numpy()
            for k, c in enumerate(cases):
                ri, rv = _f(c["invariants"]), _f(c["values"])
                sc = 1 + np.abs(ri).max()
                e = max(np.abs(inv[k] - ri).max(), np.abs(vals[k] - rv).max()) / sc
                worst = max(worst, e)
                assert e < tol, (kind, kernel, c["distance"], c["radius"], e)
            assert (b.status.cpu().numpy() == 0).all()
    print("worst scaled error", worst)


def test_sphere_fixture_requests_in_fixture_order():
    from warpsphboundaries_b200.radial import RadialEvaluator, Request
    for c in G["sphere"]:
        reqs = [Request(*json.loads(k)) for k in c["values"]]
        ev = RadialEvaluator("sphere", reqs, kernel=c["kernel"])
        got = ev.evaluate([float(c["distance"])], _f(c["normal"]), 1.0, radii=float(c["radius"]))[0]
        ref = _f(c["values"].values())
        assert np.abs(got - ref).max() < 1e-13 * (1 + np.abs(ref).max()), (c["label"], c["kernel"])


def test_physical_units_and_random_batch_against_oracle():
    """supports h != 1: invariants scale as (1, h, h^2, h^2, 1/h, 1, 1, 1/h^2, 1/h^2)."""
    from warpsphboundaries_b200.radial import RadialEvaluator
    rng = np.random.default_rng(5)
    m = 400
    h = rng.uniform(0.01, 0.05, m)
    R = np.exp(rng.uniform(np.log(0.2), np.log(50), m)) * h
    d = rng.uniform(-1.2, 1.2, m) * h
    d = np.maximum(d, -R)
    n = rng.normal(size=(m, 3))
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    for kernel in ("cubic", "w4"):
        ev = RadialEvaluator("sphere", kernel=kernel)
        b = ev.prepare(d, n, h, radii=R)
        b.launch()
        got = b.numpy()
        req_scale = np.array([r.scale for r in ev.requests])          # |alpha| - |derivative|
        for k in range(0, m, 7):
            # compare at unit support: the oracle's adaptive quadrature of monomial profiles is good to ~1e-11 there
            ref = OR.select(OR.invariants(d[k] / h[k], kernel, R[k] / h[k]), n[k])
            unit = got[k] / h[k] ** req_scale
            assert np.abs(unit - ref).max() < 1e-9 * (1 + np.abs(ref).max()), (kernel, k)


def test_invalid_rows_get_nan_and_status_through_the_abi():
    """the C ABI does not sync to validate: bad rows come back NaN with status 1, good rows are untouched."""
    import ctypes
    from warpsphboundaries_b200 import _lib
    dev = torch.device("cuda")
    d = torch.tensor([0.1, -3.0, 0.2, 0.0], dtype=torch.float64, device=dev)
    R = torch.tensor([1.0, 1.0, -1.0, 1.0], dtype=torch.float64, device=dev)
    n = torch.tensor([[0, 0, 1.0]] * 4, dtype=torch.float64, device=dev)
    h = torch.tensor([1.0, 1.0, 1.0, 0.0], dtype=torch.float64, device=dev)
    meta = np.array([[0, 0, 0, 0], [1, 2, 0, 0]], dtype=np.int32)
    out = torch.zeros(4, 2, dtype=torch.float64, device=dev)
    st = torch.full((4,), 7, dtype=torch.int32, device=dev)
    rc = _lib.lib.wsb_radial_channels(_lib.RADIAL_SPHERE, 1, _lib.PREC_FP64, _lib.ptr(d), _lib.ptr(R), _lib.ptr(n),
                                      _lib.ptr(h), 4, meta.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), 2,
                                      _lib.ptr(out), None, _lib.ptr(st), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert st.tolist() == [0, 1, 1, 1]
    o = out.cpu().numpy()
    assert np.isfinite(o[0]).all() and np.isnan(o[1:]).all()
    ref = OR.select(OR.invariants(0.1, "w2", 1.0), [0, 0, 1.0], [((0, 0, 0), ()), ((0, 0, 1), ())])
    assert np.abs(o[0] - ref).max() < 1e-13


def test_empty_batch_and_subset_requests():
    from warpsphboundaries_b200.radial import RadialEvaluator, Request
    ev = RadialEvaluator("plane", [Request((0, 0, 0), (0, 2))], kernel="w6")
    b = ev.prepare(np.zeros(0), np.zeros((0, 3)), 1.0)
    assert b.launch().shape == (0, 1)
    got = ev.evaluate([-0.3, 0.4], [[0.6, 0.0, 0.8]] * 2, 0.5)
    for k, dist in enumerate([-0.3, 0.4]):
        ref = OR.select(OR.invariants(dist / 0.5, "w6") * 0.5 ** np.array([0, 1, 2, 2, -1, 0, 0, -2, -2]),
                        [0.6, 0.0, 0.8], [((0, 0, 0), (0, 2))])
        assert abs(got[k, 0] - ref[0]) < 1e-10 * (1 + abs(ref[0]))      # the oracle is good to ~1e-11
