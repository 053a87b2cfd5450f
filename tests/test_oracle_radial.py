"""The radial oracle (solid spheres / half-spaces, 3-D) against the reference's 70-digit fixtures."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import radial as R

G = json.loads((Path(__file__).parent / "golden" / "radial_golden.json").read_text())


@pytest.mark.parametrize("case", G["radial"][::3], ids=[f"{c['kind']}-{c['kernel']}-{c['distance']}-{c['radius']}"
                                                        for c in G["radial"][::3]])
def test_invariants_and_channels(case):
    rad = None if case["radius"] in (None, "None") else float(case["radius"])
    inv = R.invariants(float(case["distance"]), case["kernel"], rad)
    ref = np.array([float(x) for x in case["invariants"]])
    assert np.abs(inv - ref).max() < 1e-9 * (1 + np.abs(ref).max())
    vals = R.select(ref, [float(x) for x in case["normal"]])
    assert np.abs(vals - np.array([float(x) for x in case["values"]])).max() < 1e-12 * (1 + np.abs(ref).max())


@pytest.mark.parametrize("case", G["sphere"], ids=[f"{c['label']}-{c['kernel']}-{c['distance']}-{c['radius']}"
                                                 for c in G["sphere"]])
def test_sphere_requests(case):
    """the sphere fixture lists the baseline requests in its own order: compare request by request."""
    inv = R.invariants(float(case["distance"]), case["kernel"], float(case["radius"]))
    reqs = [(tuple(a), tuple(d)) for a, d in map(json.loads, case["values"])]
    vals = R.select(inv, [float(x) for x in case["normal"]], reqs)
    ref = np.array([float(v) for v in case["values"].values()])
    assert sorted(reqs) == sorted(R.baseline())
    assert np.abs(vals - ref).max() < 1e-9 * (1 + np.abs(ref).max())
