"""Oracle values on seeded subsets of the full-size benchmark scenes, for the GPU parity tests at those sizes.

    python tests/golden/make_config_fixtures.py [c3]

c3  the 3-D scene (2^21 particles uniform in [-1, 1]^3, h = 0.03, the jittered icosphere of 20 480 faces): the 28
    baseline channels of 64 queries -- 48 particles of the scene within one support of the surface (by the exact
    point-triangle distance), 8 particles farther from it (constant rows), and 8 planted queries 1e-7 h off vertices,
    edge midpoints and face centres of the jittered surface -- for w2, w4 and w6, from oracle/mesh3d.py (the float64
    restatement of the reference's closed-surface reduction, pinned to its mpmath values).  The oracle costs ~35 s a
    query on this surface, which is why the values are computed here once (in worker processes) and committed.

Writes tests/golden/c3_subset.json.  Reads nothing outside this repository.
"""
import json
import multiprocessing as mp
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

C3_KERNELS = ("w2", "w4", "w6")


def _point_triangle_distance(p, A, B, C):
    """distance of p [3] to each triangle (A, B, C [F, 3]) by projection and edge clamping (selection only)."""
    n = np.cross(B - A, C - A)
    nn = np.linalg.norm(n, axis=1)
    nu = n / nn[:, None]
    d = ((p - A) * nu).sum(1)
    q = p - d[:, None] * nu
    inside = np.ones(len(A), bool)
    for U, W in ((A, B), (B, C), (C, A)):
        inside &= (np.cross(W - U, q - U) * n).sum(1) >= 0
    best = np.where(inside, np.abs(d), np.inf)
    for U, W in ((A, B), (B, C), (C, A)):
        e = W - U
        t = np.clip(((p - U) * e).sum(1) / (e * e).sum(1), 0.0, 1.0)
        best = np.minimum(best, np.linalg.norm(p - (U + t[:, None] * e), axis=1))
    return best.min()


def c3_queries():
    """(row ids into the c3 particle set, planted queries [8, 3], all queries [64, 3], h)."""
    from warpsphboundaries_b200 import workloads
    V, Fc, X, h = workloads.c3()
    A, B, C = V[Fc[:, 0]], V[Fc[:, 1]], V[Fc[:, 2]]
    rng = np.random.default_rng(2024)
    r = np.linalg.norm(X, axis=1)
    band = np.nonzero(np.abs(r - 0.6) < 0.6 * 0.05 + h)[0]
    near, far = [], []
    for i in rng.permutation(band):
        if len(near) == 48:
            break
        if _point_triangle_distance(X[i], A, B, C) < h:
            near.append(int(i))
    for i in rng.permutation(len(X)):
        if len(far) == 8:
            break
        if abs(r[i] - 0.6) > 0.6 * 0.05 + 2 * h:
            far.append(int(i))
    nrm = np.cross(B - A, C - A)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    k = rng.choice(len(Fc), 8, replace=False)
    planted = np.concatenate([
        V[Fc[k[:3], 0]] + 1e-7 * h * nrm[k[:3]],                                # just outside vertices
        (V[Fc[k[3:6], 0]] + V[Fc[k[3:6], 1]]) / 2 - 1e-7 * h * nrm[k[3:6]],     # just inside edge midpoints
        (A[k[6:]] + B[k[6:]] + C[k[6:]]) / 3 + 1e-7 * h * nrm[k[6:]],           # just outside face centres
    ])
    rows = near + far
    return rows, planted, np.concatenate([X[rows], planted]), h


def _c3_one(args):
    q, kernel = args
    from oracle import mesh3d as M3
    from warpsphboundaries_b200 import workloads
    V, Fc = workloads.icosphere(5, 0.6, 0.05, 21)
    return M3.channels(V, Fc, q, 0.03, kernel).tolist()


def make_c3(procs=None):
    rows, planted, Q, h = c3_queries()
    jobs = [(q, k) for k in C3_KERNELS for q in Q]
    with mp.get_context("spawn").Pool(procs or os.cpu_count() or 1) as pool:
        vals = pool.map(_c3_one, jobs, chunksize=1)
    out = {"source": "oracle/mesh3d.py channels (float64 restatement of the reference's closed-surface reduction)",
           "scene": "workloads.c3(): 2^21 particles in [-1,1]^3 (seed 0), icosphere 5 subdivisions, r 0.6, 5% jitter",
           "h": h, "rows": rows, "planted": planted.tolist(), "queries": Q.tolist(), "kernels": list(C3_KERNELS),
           "values": {k: vals[i * len(Q):(i + 1) * len(Q)] for i, k in enumerate(C3_KERNELS)}}
    (HERE / "c3_subset.json").write_text(json.dumps(out))
    print("c3_subset.json:", len(Q), "queries x", len(C3_KERNELS), "kernels")


if __name__ == "__main__":
    which = sys.argv[1:] or ["c3"]
    if "c3" in which:
        make_c3()
