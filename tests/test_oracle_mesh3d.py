"""The closed-surface oracle (float64 restatement of the reference's exact reduction) against the reference's own
mpmath values."""
import json
from pathlib import Path

import numpy as np
import pytest

from oracle import mesh3d as M3

G = json.loads((Path(__file__).parent / "golden" / "mesh3d_golden.json").read_text())


@pytest.mark.parametrize("case", G["cases"][::2], ids=[f"{c['mesh']}-{c['kernel']}-{c['h']}-{k}"
                                                      for k, c in enumerate(G["cases"][::2])])
def test_oracle_matches_reference(case):
    m = G["meshes"][case["mesh"]]
    got = M3.channels(m["vertices"], m["faces"], case["query"], case["h"], case["kernel"])
    ref = np.array([float(v) for v in case["values"]])
    scale = np.abs(ref).max()
    assert np.abs(got - ref).max() < 1e-8 * (1 + scale)
