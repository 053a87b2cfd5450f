"""GPU parity through the C ABI: neighbour sets bit-exact, channels within the stated tolerances of the oracle.

Tolerances (outputs in units of the support h, where every channel is O(1)):
  float64 routes (fused, plain)   <= 1e-10 absolute
  mixed route                     <= 1e-6 absolute (the target bound of the mixed-precision path)
  float route                     <= 2e-5 absolute (float32 chord sums: a few ulp of each profile's scale)
"""
import json
from fractions import Fraction as F
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import edge2d as O
from tests.helpers import DEV, gpu_outputs, make_scene, oracle_outputs, scaled_errors, small_c2
from warpsphboundaries_b200 import workloads
from warpsphboundaries_b200.fixedadj import fixed_topology

pytestmark = pytest.mark.gpu
KERNELS = ["cubic", "w2", "w4", "w6", "quartic", "quintic", "poly6", "cone", "lw2", "lw4"]
TOL64 = 1e-10
TOL_MIXED = 1e-6
TOL_FP32 = 2e-5


@pytest.fixture(scope="module")
def c1():
    loops, X, h = workloads.c1()
    return loops, X, h


@pytest.fixture(scope="module")
def c2s():
    return small_c2()


def test_fixed_topology_slots_bit_exact(c2s):
    """every row's neighbour edges (set AND order) and its indicator equal the oracle's, near-tangent rows included."""
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    lpos = torch.tensor(X, dtype=torch.float64, device=DEV)
    lsup = torch.full((len(X),), h, dtype=torch.float64, device=DEV)
    ft = fixed_topology(rep, lpos, lsup, torch.ones(len(X), dtype=torch.bool, device=DEV), h)
    e = ft.e.reshape(len(X), ft.K).cpu().numpy()
    V, E = workloads.edges_of(loops)
    cl = O.build_cell_list(V, E, h)
    ref = O.fixed_slots(V, E, cl, X, np.full(len(X), h))
    npairs = 0
    for r in range(len(X)):
        got = e[r][e[r] >= 0]
        assert np.array_equal(got, ref[r]), r
        assert np.all(e[r][len(got):] == -1)
        npairs += len(got)
    assert npairs > 1000
    ind_ref = O.indicator(V, E, 0, X, np.full(len(X), h))
    ind = ft.ind.cpu().numpy()
    exact = np.abs(ind_ref - np.round(ind_ref)) == 0
    assert np.array_equal(ind[exact], ind_ref[exact])
    assert np.abs(ind - ind_ref).max() < 1e-12


def test_static_cell_list_equals_oracle(c2s):
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    ns = rep.native(h, DEV)
    start, items = ns.cells()
    V, E = workloads.edges_of(loops)
    lo, cell, (nx, ny), rstart, ritems = O.build_cell_list(V, E, h)
    assert (ns.info.nx, ns.info.ny) == (nx, ny)
    assert np.array_equal(start, rstart) and np.array_equal(items, ritems)
    assert ns.K == int(np.diff(rstart).max())


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("route", ["fused", "plain"])
def test_fp64_routes_match_oracle_c2(c2s, kernel, route):
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    got = gpu_outputs(scene, X, h, kernel, h, route=route)
    ref = oracle_outputs(loops, X, h, kernel, h)
    err = scaled_errors(got, ref, h)
    assert max(err.values()) < TOL64, err


@pytest.mark.parametrize("kernel", ["cubic", "w2", "w4", "w6", "cone", "lw2", "lw4"])
def test_mixed_route_within_1e6(c2s, kernel):
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    got = gpu_outputs(scene, X, h, kernel, h, precision="mixed")
    ref = oracle_outputs(loops, X, h, kernel, h)
    err = scaled_errors(got, ref, h)
    assert max(err.values()) < TOL_MIXED, err


@pytest.mark.parametrize("kernel", ["cubic", "w2", "w4", "w6", "quartic", "quintic", "poly6", "cone", "lw2", "lw4"])
def test_fp32_route_within_tolerance(c2s, kernel):
    """the float route (Chebyshev profiles and graded Gauss-Legendre chord quadrature in float32, float64 clip, edge
    frame and row sums) against the oracle, near-tangent and on-vertex rows included."""
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    got = gpu_outputs(scene, X, h, kernel, h, precision="fp32")
    ref = oracle_outputs(loops, X, h, kernel, h)
    err = scaled_errors(got, ref, h)
    print(f"fp32 {kernel}: " + ", ".join(f"{k} {v:.1e}" for k, v in err.items()))
    assert max(err.values()) < TOL_FP32, err


@pytest.mark.parametrize("kernel", ["cubic", "w2", "w4", "w6"])
def test_c1_against_reference_numpy_fixture(kernel):
    """the 256-gon scene against the reference's np2d values (tests/golden/np2d_c1.npz)."""
    d = np.load(Path(__file__).parent / "golden" / "np2d_c1.npz")
    P, X, sub, h = d["polygon"], d["particles"], d["subset"], float(d["h"])
    scene, rep, body = make_scene([P])
    got = gpu_outputs(scene, X[sub], h, kernel, h)
    ch = d["ch_" + kernel]
    sc = np.array([1, 1 / h, 1 / h, h, h, 1, 1, 1, 1, 1 / h ** 2, 1 / h ** 2, 1 / h ** 2])
    mine = np.concatenate([got["lam"][:, None], got["m1"], got["G"], got["Cov"].reshape(-1, 4),
                           got["m2"].reshape(-1, 4)[:, [0, 1, 3]]], 1)
    assert np.abs((mine - ch) * sc).max() < 5e-11


@pytest.mark.parametrize("kernel", ["w4", "cubic"])
def test_rotated_translated_body(c2s, kernel):
    loops, X, h = c2s
    center, angle = (0.3, -0.2), 0.7
    # the loops are given in the body frame: world = R local + center
    scene, rep, body = make_scene(loops, center=center, angle=angle)
    got = gpu_outputs(scene, X, h, kernel, h)
    ref = oracle_outputs(loops, X, h, kernel, h, center=center, angle=angle)
    err = scaled_errors(got, ref, h)
    assert max(err.values()) < TOL64, err


def test_background_surface_tank():
    """a clockwise tank (solid outside, background 1): every particle sees the wall as solid outside the loop."""
    rng = np.random.default_rng(3)
    tank = workloads.star(rng, (0.5, 0.5), 0.4, 200, jitter=0.05)
    X = rng.uniform(0.05, 0.95, size=(3000, 2))
    h = 0.03
    scene, rep, body = make_scene([tank], background=1)
    V = rep.vertices.cpu().numpy()
    E = rep.edges.cpu().numpy().astype(np.int64)
    for kernel in ["w2", "cubic"]:
        got = gpu_outputs(scene, X, h, kernel, h)
        out12 = O.local_twelve(V, E, 1, X, np.full(len(X), h), kernel, h)
        ref = O.to_world(out12, 0.0)
        err = scaled_errors(got, ref, h)
        assert max(err.values()) < TOL64, err


def test_deterministic_repeat(c2s):
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    a = gpu_outputs(scene, X, h, "w4", h)
    b = gpu_outputs(scene, X, h, "w4", h)
    for k in a:
        assert np.array_equal(a[k], b[k])


GOLD = json.loads((Path(__file__).parent / "golden" / "edge2d_golden_subset.json").read_text())


def test_golden_elements_on_gpu():
    """every 40-digit golden element (polygon, point, support) through the fused route: value, moments and gradient
    within 1e-10 (1 + |ref|) in physical units."""
    worst = 0.0
    for case in GOLD["cases"]:
        P = np.array([[float(F(a)), float(F(b))] for a, b in case["polygon"]])
        x = np.array([[float(F(s)) for s in case["x"]]])
        h = float(F(case["h"]))
        loops = [P]
        scene, rep, body = make_scene(loops)
        for k in ["cubic", "w2", "w4", "w6"]:
            e = case["kernels"][k]
            got = gpu_outputs(scene, x, h, k, h)
            pairs = [(got["lam"][0], e["value"]), (got["m1"][0, 0], e["moments"]["1,0"]),
                     (got["m1"][0, 1], e["moments"]["0,1"]), (got["m2"][0, 0, 0], e["moments"]["2,0"]),
                     (got["m2"][0, 0, 1], e["moments"]["1,1"]), (got["m2"][0, 1, 1], e["moments"]["0,2"]),
                     (got["G"][0, 0], e["grad"][0]), (got["G"][0, 1], e["grad"][1])]
            for g, r in pairs:
                r = float(r)
                err = abs(g - r) / (1 + abs(r))
                worst = max(worst, err)
                assert err < 1e-10, (case["id"], k, g, r)
    assert worst < 1e-10


@pytest.mark.parametrize("kernels", [("w4",), ("cubic", "w2", "w4", "w6"), ("w2", "cone", "lw2")])
@pytest.mark.parametrize("assign", [True, False])
@pytest.mark.parametrize("offset", [0, 1, 2])
def test_staged_and_direct_evaluation_agree(c2s, kernels, assign, offset):
    """a workspace with the staging region (work rows' sums staged, every row expanded in one coalesced pass) and one
    without it (work rows' outputs stored directly) give the same bits, for one kernel and for packs; outputs that
    start 8 bytes off a 16-byte boundary (offset 1) take the expansion's scalar stores, 16 bytes off a 32-byte one
    (offset 2) its 16-byte stores, aligned ones its 32-byte stores."""
    import ctypes
    from warpsphboundaries_b200 import _lib
    from warpsphboundaries_b200.kernels import KERNEL_IDS
    from warpsphboundaries_b200.scene import _stream
    loops, X, h = c2s
    scene, rep, body = make_scene(loops, center=(0.02, -0.01), angle=0.3)
    ns = rep.native(h, DEV)
    n = len(X)
    pos = torch.tensor(X, dtype=torch.float64, device=DEV)
    sup = torch.full((n,), h, dtype=torch.float64, device=DEV)
    base = int(_lib.lib.wsb_aggregate_workspace_size(ns.handle, n))
    full = base + int(_lib.lib.wsb_aggregate_staging_size(ns.handle, n))
    kids = _lib.int32s([KERNEL_IDS[k] for k in kernels])
    obb = (ctypes.c_double * 4)(*body.obb())
    pose = body.pose_tensor(DEV)
    mode = _lib.OUT_ALL | (_lib.OUT_ASSIGN if assign else 0)
    res = []
    for nbytes in (base, full):
        ws = torch.empty(nbytes, dtype=torch.uint8, device=DEV)
        outs = [[torch.full((n * w + 1,), 0.25, dtype=torch.float64, device=DEV)[offset:offset + n * w]
                 for _ in kernels] for w in (1, 2, 4, 2, 4)]
        _lib.check(_lib.lib.wsb_aggregate_groups(ns.handle, len(kernels), kids, _lib.PREC_FP64, _lib.ptr(pos),
                                                 _lib.ptr(sup), None, n, _lib.ptr(pose), obb, 0, mode,
                                                 *[_lib.ptrs(o) for o in outs], _lib.ptr(ws), nbytes, _stream()))
        torch.cuda.synchronize()
        res.append(outs)
    for a, b in zip(res[0], res[1]):
        for x, y in zip(a, b):
            assert torch.equal(x, y)
