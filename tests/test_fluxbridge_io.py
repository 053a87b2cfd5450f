"""The fluxbridge fixture file (schema 1) as an interchange format: the reference's own file (a subset made by
tests/golden/make_golden.py) round-trips unchanged through load / dump, malformed cases are refused, and on the GPU
every request the device routes serve matches the stored 70-digit value within 1e-10 (1 + |v|)."""
import json
from pathlib import Path

import numpy as np
import pytest

from warpsphboundaries_b200 import fluxbridge_io as fx

SRC = Path(__file__).parent / "golden" / "fluxbridge_v1_subset.json"


def test_round_trip_is_unchanged(tmp_path):
    f = fx.load(SRC)
    assert f.dps == 70 and len(f.cases) == 44
    assert {c.dimension for c in f.cases} == {2, 3} and {c.measure for c in f.cases} == {"volume", "surface"}
    text = fx.dump(f, tmp_path / "out.json")
    assert json.loads(text) == json.loads(SRC.read_text())
    again = fx.load(tmp_path / "out.json")
    assert fx.to_dict(again) == fx.to_dict(f)


def test_served_requests_and_refusals():
    f = fx.load(SRC)
    tet = next(c for c in f.cases if c.dimension == 3 and c.measure == "volume" and not fx._on_tet_boundary(c))
    on = [c for c in f.cases if c.dimension == 3 and c.measure == "volume" and fx._on_tet_boundary(c)]
    assert len(on) == 8 and all(c.query in ([0, 0, 0], [1, 0, 0]) for c in on)          # a vertex, an edge midpoint
    assert not any(fx.served(on[0]))
    tri = next(c for c in f.cases if c.dimension == 2)
    assert sum(fx.served(tet)) == 28 and sum(fx.served(tri)) == 12
    surf = next(c for c in f.cases if c.measure == "surface")
    assert not any(fx.served(surf))
    bad = json.loads(SRC.read_text())
    bad["schema"] = 2
    with pytest.raises(ValueError):
        fx.load(bad)
    bad = json.loads(SRC.read_text())
    bad["cases"][0]["values"] = bad["cases"][0]["values"][:-1]
    with pytest.raises(ValueError):
        fx.load(bad)


@pytest.mark.gpu
def test_device_matches_the_stored_values():
    f = fx.load(SRC)
    worst, n = 0.0, 0
    for c in f.cases:
        if c.measure == "surface":
            with pytest.raises(NotImplementedError):
                fx.evaluate(c)
            continue
        got = fx.evaluate(c)
        ref = c.reference()
        ok = np.array(fx.served(c))
        assert np.isnan(got[~ok]).all()
        if not ok.any():
            continue
        err = np.abs(got[ok] - ref[ok]) / (1 + np.abs(ref[ok]))
        worst = max(worst, float(err.max()))
        n += int(ok.sum())
        assert err.max() < 1e-10, (c.dimension, c.kernel, c.query, float(err.max()))
    assert n > 400
    print(f"fluxbridge fixture: {n} values, worst {worst:.2e}")
