"""The oracle (oracle/edge2d.py) against the reference's golden vectors and its own numpy / torch paths."""
import json
from fractions import Fraction as F
from pathlib import Path

import numpy as np
import pytest

from oracle import edge2d as O
from warpsphboundaries_b200 import workloads

G = Path(__file__).parent / "golden"
GOLD = json.loads((G / "edge2d_golden_subset.json").read_text())
KERNELS = ["cubic", "w2", "w4", "w6"]


def _case(c):
    P = np.array([[float(F(a)), float(F(b))] for a, b in c["polygon"]])
    x = np.array([float(F(s)) for s in c["x"]])
    return P, x, float(F(c["h"]))


@pytest.mark.parametrize("case", GOLD["cases"], ids=[c["id"] for c in GOLD["cases"]])
def test_oracle_matches_40_digit_golden_vectors(case):
    """value, moments |alpha| <= 2, gradient and moment gradients of every golden element, all four kernels:
    absolute error <= 1e-11 (1 + |ref|) (float64 monomial closed form; the golden values are exact to 1e-35)."""
    P, x, h = _case(case)
    tags = set(case["tags"])
    for k in KERNELS:
        e = case["kernels"][k]
        r = O.polygon_moments(P, x, h, k)
        pairs = [(r[(0, 0)], e["value"])]
        for al in [(1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]:
            pairs.append((r[al], e["moments"][f"{al[0]},{al[1]}"]))
        pairs += [(r["G"][0], e["grad"][0]), (r["G"][1], e["grad"][1])]
        for al in [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]:
            g = O.moment_gradient(P, x, h, k, al)
            ref = e["moment_grad"][f"{al[0]},{al[1]}"]
            pairs += [(g[0], ref[0]), (g[1], ref[1])]
        for got, ref in pairs:
            ref = float(ref)
            assert abs(got - ref) <= 1e-11 * (1 + abs(ref)), (case["id"], k, got, ref, tags)


def test_golden_coverage():
    tags = {t for c in GOLD["cases"] for t in c["tags"]}
    assert {"x_on_edge", "x_at_vertex", "z_to_0", "tiny_chord", "small_element", "half_plane", "nonconvex",
            "clockwise", "h_scaled", "outside_support", "cubic_knot", "generic"} <= tags
    assert {c["where"] for c in GOLD["cases"]} == {"inside", "outside", "edge", "vertex"}


def test_oracle_matches_reference_numpy_path_on_c1():
    """the twelve channels of the 256-gon scene against the reference's np2d run on the same particles:
    scaled absolute error <= 5e-12 (G scaled by 1/h, m1 by h, m2 by h^2)."""
    d = np.load(G / "np2d_c1.npz")
    P, X, sub, h = d["polygon"], d["particles"], d["subset"], float(d["h"])
    n = len(P)
    E = np.stack([np.arange(n), (np.arange(n) + 1) % n], 1)
    scale = np.array([1, h, h, 1 / h, 1 / h, 1, 1, 1, 1, h * h, h * h, h * h])
    for k in KERNELS:
        out = O.local_twelve(P, E, 0, X[sub], np.full(len(sub), h), k, h)
        err = np.abs(out - d["ch_" + k]) / scale
        assert err.max() < 5e-12, (k, err.max(0))


def test_oracle_gradients_match_reference_torch_autograd():
    """d m_alpha / dx and d m_alpha / d vertex (|alpha| <= 2, w4) against torch autograd through the reference's
    torch2d on a star polygon: scaled error <= 1e-11."""
    g = np.load(G / "torch2d_grad.npz")
    P, X, h = g["polygon"], g["particles"], float(g["h"])
    for al in [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]:
        key = f"{al[0]}{al[1]}"
        sc = h ** (al[0] + al[1] - 1)
        for i in range(0, len(X), 3):
            assert np.abs(O.moment_gradient(P, X[i], h, "w4", al) - g["dx_" + key][i]).max() / sc < 1e-11
            assert np.abs(O.shape_gradient(P, X[i], h, "w4", al) - g["dv_" + key][i]).max() / sc < 1e-11


def test_plane_constants():
    for k, (m, p2) in {"w4": (1, F(7, 132)), "w2": (1, F(5, 72)), "w6": (1, F(3, 70)), "cubic": (1, F(31, 392))}.items():
        mass, plane2 = O.kernel_mass_and_plane(k)
        assert mass == m and plane2 == p2


WALL = json.loads((G / "edge2d_wall_kernels.json").read_text())


def test_wall_kernel_tables_equal_the_reference_registration():
    """cone, lw2, lw4: the normalisation and block coefficients the reference registers (edge/kernels.py, scene/
    viscosity.py) equal the exact tables of the library and of the oracle."""
    from warpsphboundaries_b200 import kernels as K
    for k in ("cone", "lw2", "lw4"):
        ref = WALL["kernels"][k]
        assert K.kernel(k).c2pi == F(ref["c2_pi"])
        ours = [(b.R, [F(x) for x in b.c]) for b in K.kernel(k).blocks]
        theirs = [(F(R), [F(x) for x in cs]) for R, cs in ref["blocks"]]
        assert len(ours) == len(theirs)
        for (r0, c0), (r1, c1) in zip(ours, theirs):
            assert r0 == r1
            n = max(len(c0), len(c1))
            assert c0 + [F(0)] * (n - len(c0)) == c1 + [F(0)] * (n - len(c1)), k
        orc = O.blocks(k)
        assert [(R, [P.get(i, F(0)) for i in range(len(cs))]) for (R, P), (_, cs) in zip(orc, theirs)] == theirs


@pytest.mark.parametrize("case", WALL["cases"], ids=[c["id"] for c in WALL["cases"]])
def test_oracle_matches_wall_kernel_golden_vectors(case):
    """the wall-operator kernels (cone, lw2, lw4) on every golden element: value, moments |alpha| <= 2, gradient and
    moment gradients against the reference's 40-digit evaluation, absolute error <= 1e-11 (1 + |ref|)."""
    geo = next(c for c in GOLD["cases"] if c["id"] == case["id"])
    P, x, h = _case(geo)
    for k, e in case["kernels"].items():
        r = O.polygon_moments(P, x, h, k)
        pairs = [(r[(0, 0)], e["value"])]
        for al in [(1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]:
            pairs.append((r[al], e["moments"][f"{al[0]},{al[1]}"]))
        pairs += [(r["G"][0], e["grad"][0]), (r["G"][1], e["grad"][1])]
        for al in [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]:
            g = O.moment_gradient(P, x, h, k, al)
            ref = e["moment_grad"][f"{al[0]},{al[1]}"]
            pairs += [(g[0], ref[0]), (g[1], ref[1])]
        for got, ref in pairs:
            ref = float(ref)
            assert abs(got - ref) <= 1e-11 * (1 + abs(ref)), (case["id"], k, got, ref)


def test_powered_kernel_normalisation_equals_the_reference_registration():
    """w2p5 / w4p5 (W^5 of Wendland C2 / C4, the tensile group): the reference's normalisation equals ours and the
    oracle's; its block is the expanded polynomial of C u^p B(u)^5."""
    from warpsphboundaries_b200 import kernels as K
    for k in ("w2p5", "w4p5"):
        ref = WALL["kernels"][k]
        assert K.quad_kernel(k)[0] == F(ref["c2_pi"]) == O.powered(k)[0]
        (R, cs), = ref["blocks"]
        r = F(3, 7)
        assert sum(F(c) * r ** n for n, c in enumerate(cs)) == K.pi_w_quad(k, r)


@pytest.mark.parametrize("case", WALL["cases"], ids=[c["id"] for c in WALL["cases"]])
def test_oracle_tensile_gradient_matches_golden(case):
    """the tensile kernels' gradient (adaptive quadrature along each chord) against the reference's 40-digit exact
    edge reduction on every golden element: absolute error <= 1e-11 (1 + |ref|)."""
    geo = next(c for c in GOLD["cases"] if c["id"] == case["id"])
    P, x, h = _case(geo)
    for k, ref in case["powered_grad"].items():
        got = O.powered_gradient(P, x, h, k)
        for a, b in zip(got, ref):
            b = float(b)
            assert abs(a - b) <= 1e-11 * (1 + abs(b)), (case["id"], k, a, b)


# ------------------------------------------------------------------------------------------------ detector inputs
CONE = json.loads((G / "cone_area_golden.json").read_text())


@pytest.mark.parametrize("case", range(len(CONE["cases"])))
def test_cone_area_oracle_matches_the_reference_closed_form(case):
    """oracle/cone_area.py against the reference's own vectorised closed form (scene/cone_area.py) on the golden
    points: the same per-edge formula in float64, so the tolerance is round-off, 1e-13 H^2."""
    from oracle import cone_area as C
    c = CONE["cases"][case]
    r = CONE["reps"][c["rep"]]
    got = C.cone_area(r["points"], r["axes"], c["half_angle"], c["H"], r["vertices"], r["edges"], r["background"])
    assert np.abs(got - np.array(c["value"])).max() <= 1e-13 * c["H"] ** 2
    assert (np.array(c["value"]) > 1e-3 * c["H"] ** 2).sum() > 10          # the points do see the solid


def test_cone_area_oracle_additivity_and_bounds():
    """two complementary wedges (axis a, half angle al; axis -a, half angle pi - al) tile the disk, so their areas
    sum to the full-disk area; 0 <= wedge area <= full area <= pi H^2 (round-off 1e-13 H^2)."""
    from oracle import cone_area as C
    H = 0.5
    for r in CONE["reps"]:
        p, a = np.array(r["points"]), np.array(r["axes"])
        full = C.cone_area(p, a, np.pi, H, r["vertices"], r["edges"], r["background"])
        for al in (0.3, 1.0, 2.5):
            w1 = C.cone_area(p, a, al, H, r["vertices"], r["edges"], r["background"])
            w2 = C.cone_area(p, -a, np.pi - al, H, r["vertices"], r["edges"], r["background"])
            assert np.abs(w1 + w2 - full).max() <= 1e-13
            assert w1.min() >= -1e-13 and (w1 - full).max() <= 1e-13
        assert full.max() <= np.pi * H * H + 1e-13


def test_dir_extreme_local_oracle_matches_the_polar_grid():
    """the closed-form direction extreme (oracle/cone_area.dir_extreme_local) against the reference test's polar
    grid oracle with even-odd membership (tests/scene/test_fused_wall.py:207-226): never below it, within its
    angular resolution (the reference's tolerance 1.5e-2), both near and far points present, a zero vector gives 0."""
    from oracle import cone_area as C
    rng = np.random.default_rng(5)
    H = 0.5
    for r in CONE["reps"]:
        V, E, bg = np.array(r["vertices"]), np.array(r["edges"]), r["background"]
        p = np.array(r["points"])[:40]
        v = rng.normal(size=(len(p), 2))
        v[3] = 0.0
        got = C.dir_extreme_local(p, v, H, V, E, bg)
        ref = C.dir_extreme_polar(p, v, H, V, E, bg, nr=150, nphi=1440)
        assert (got >= ref - 1e-9).all(), float((ref - got).max())
        assert np.abs(got - ref).max() <= 1.5e-2
        assert got[3] == 0.0
        assert (got > 0.5).sum() > 3


def test_binned_indicator_equals_the_whole_loop_indicator():
    """the oracle's restatement of the reference's fast indicator (cell cache + y-bin ray cast, scene.py:281-396) gives
    the same value as the whole-loop form, bit for bit, on seeded rows of the large 2-D scene -- including rows exactly
    on vertices and on edge midpoints (interior-angle fractions) and rows in edge-free cells (the cell cache)."""
    loops, X, h = workloads.c2(n_particles=1 << 16)
    V, E = workloads.edges_of(loops)
    rng = np.random.default_rng(3)
    sub = X[rng.choice(len(X), 3000, replace=False)]
    sub[:100] = V[rng.choice(len(V), 100, replace=False)]
    k = rng.choice(len(E), 100, replace=False)
    sub[100:200] = (V[E[k, 0]] + V[E[k, 1]]) / 2
    sup = np.full(len(sub), h)
    cl = O.build_cell_list(V, E, h)
    a = O.indicator(V, E, 0, sub, sup)
    b = O.indicator_binned(V, E, 0, sub, sup, cl)
    assert np.array_equal(a, b)
    assert np.any(a[:200] % 1.0 != 0.0)                       # boundary rows took the angle sum


def test_oracle_matches_reference_torch2d_on_the_gradient_scene():
    """on 256 near-wall rows of the full gradient scene (2^18 particles, 16 stars of 128 vertices, h = 0.02, w4) the
    oracle's six moments equal the reference's torch2d values (tests/golden/torch2d_c4.npz) within 1e-12 in units of
    h^|alpha|."""
    g = np.load(Path(__file__).parent / "golden" / "torch2d_c4.npz")
    loops, X, h = workloads.c4()
    assert np.array_equal(X[g["rows"]], g["particles"])
    V, E = workloads.edges_of(loops)
    Xs = g["particles"]
    out = O.local_twelve(V, E, 0, Xs, np.full(len(Xs), h), "w4", h)
    for key, c in {"00": 0, "10": 1, "01": 2, "20": 9, "11": 10, "02": 11}.items():
        sc = h ** (int(key[0]) + int(key[1]))
        assert np.abs(out[:, c] - g["m_" + key]).max() / sc < 1e-12, key
