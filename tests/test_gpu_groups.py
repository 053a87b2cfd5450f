"""Several kernel groups in one aggregate (wsb_aggregate_groups / FusedWall with a tuple of groups).

The kernel sets {cubic, w2, w4, w6}, {w2, w4, w6} and the delta+ sets {w2 | w4, cone[, lw2 | lw4]} run as one pass over
the neighbour pairs that shares each pair's chord, special functions and monomial integrals between kernel blocks of
equal radius (the first such set contained in the groups; the other groups one pass each); every other set runs one
pass per group.  Either way group g must equal the single-kernel aggregate of its kernel: the pack forms the same
quantities by the same operations, so the tolerance is a few ulp of the channel scale (1e-13), far below the 1e-10
of the oracle comparisons.  The near-tangent scene of the parity tests is used, in both precision routes, with the
groups in pack order and shuffled, plus a set that no pack covers, the oracle for the float64 pack, and FusedWall.
"""
import numpy as np
import pytest
import torch

from helpers import DEV, make_scene, oracle_outputs, scaled_errors, small_c2
from warpsphboundaries_b200 import _lib
from warpsphboundaries_b200.kernels import KERNEL_IDS
from warpsphboundaries_b200.provider import FusedGroup, FusedWall
from warpsphboundaries_b200.scene import _stream
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu

TOL_SAME = 1e-13
TOL64 = 1e-10
NAMES = ("lam", "G", "Cov", "m1", "m2")


@pytest.fixture(scope="module")
def c2s():
    return small_c2()


def _buffers(n):
    return {"lam": torch.full((n,), np.nan, dtype=torch.float64, device=DEV),
            "G": torch.full((n, 2), np.nan, dtype=torch.float64, device=DEV),
            "Cov": torch.full((n, 4), np.nan, dtype=torch.float64, device=DEV),
            "m1": torch.full((n, 2), np.nan, dtype=torch.float64, device=DEV),
            "m2": torch.full((n, 4), np.nan, dtype=torch.float64, device=DEV)}


def _grouped_and_single(c2s, kernels, precision):
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    ns = rep.native(h, DEV)
    n = len(X)
    pos = torch.tensor(X, dtype=torch.float64, device=DEV)
    sup = torch.full((n,), h, dtype=torch.float64, device=DEV)
    pose = body.pose_tensor(DEV)
    obb = (_lib.ctypes.c_double * 4)(*body.obb())
    ws, need = ns.workspace(n)
    prec = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}[precision]
    mode = _lib.OUT_ALL | _lib.OUT_ASSIGN
    grouped = [_buffers(n) for _ in kernels]
    _lib.check(_lib.lib.wsb_aggregate_groups(ns.handle, len(kernels), _lib.int32s([KERNEL_IDS[k] for k in kernels]),
                                             prec, _lib.ptr(pos), _lib.ptr(sup), None, n, _lib.ptr(pose), obb, 0, mode,
                                             *[_lib.ptrs([g[name] for g in grouped]) for name in NAMES],
                                             _lib.ptr(ws), need, _stream()), "wsb_aggregate_groups")
    single = []
    for k in kernels:
        o = _buffers(n)
        _lib.check(_lib.lib.wsb_aggregate(ns.handle, KERNEL_IDS[k], prec, _lib.ptr(pos), _lib.ptr(sup), None, n,
                                          _lib.ptr(pose), obb, 0, mode, *[_lib.ptr(o[name]) for name in NAMES],
                                          _lib.ptr(ws), need, None, _stream()), "wsb_aggregate")
        single.append(o)
    torch.cuda.synchronize()
    as_np = lambda o: {"lam": o["lam"].cpu().numpy(), "G": o["G"].cpu().numpy(),
                       "Cov": o["Cov"].cpu().numpy().reshape(-1, 2, 2), "m1": o["m1"].cpu().numpy(),
                       "m2": o["m2"].cpu().numpy().reshape(-1, 2, 2)}
    return [as_np(o) for o in grouped], [as_np(o) for o in single], h


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kernels", [("cubic", "w2", "w4", "w6"), ("w6", "cubic", "w4", "w2"), ("w2", "w4", "w6"),
                                     ("w4", "w6", "w2"), ("w2", "cone", "lw2"), ("lw4", "w4", "cone"), ("cone", "w2"),
                                     ("w4", "cone", "w6"), ("cubic", "w2", "w4", "w6", "cone")])
def test_packed_groups_equal_single_kernels(c2s, kernels, precision):
    grouped, single, h = _grouped_and_single(c2s, kernels, precision)
    for k, g, s in zip(kernels, grouped, single):
        for name in NAMES:
            assert np.isfinite(g[name]).all(), (k, name)
        err = scaled_errors(g, s, h)
        assert max(err.values()) < TOL_SAME, (k, err)


@pytest.mark.parametrize("kernels", [("w4", "quartic"), ("cubic", "w2", "w4", "w4"), ("poly6",)])
def test_unpacked_group_sets_equal_single_kernels(c2s, kernels):
    grouped, single, h = _grouped_and_single(c2s, kernels, "fp64")
    for k, g, s in zip(kernels, grouped, single):
        err = scaled_errors(g, s, h)
        assert max(err.values()) == 0.0, (k, err)


def test_packed_groups_match_oracle(c2s):
    loops, X, h = c2s
    kernels = ("cubic", "w2", "w4", "w6")
    grouped, _, h = _grouped_and_single(c2s, kernels, "fp64")
    for k, g in zip(kernels, grouped):
        ref = oracle_outputs(loops, X, h, k, h)
        err = scaled_errors(g, ref, h)
        assert max(err.values()) < TOL64, (k, err)


def test_fused_wall_with_four_groups(c2s):
    """FusedWall with four groups (one wsb_aggregate_groups call per surface) equals four one-group FusedWalls."""
    loops, X, h = c2s
    scene, rep, body = make_scene(loops, center=(0.02, -0.01), angle=0.3)
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    kernels = ("w2", "cubic", "w6", "w4")
    fw = FusedWall(scene, ps, h, tuple(FusedGroup(k) for k in kernels), precision="mixed")
    for gi, k in enumerate(kernels):
        one = FusedWall(scene, ps, h, (FusedGroup(k),), precision="mixed")
        a = {name: fw.res[gi][name][0].cpu().numpy() for name in NAMES}
        b = {name: one.res[0][name][0].cpu().numpy() for name in NAMES}
        assert max(scaled_errors(a, b, h).values()) < TOL_SAME, k


def test_group_count_and_kernel_ids_are_checked(c2s):
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    ns = rep.native(h, DEV)
    n = 16
    pos = torch.zeros((n, 2), dtype=torch.float64, device=DEV)
    sup = torch.full((n,), h, dtype=torch.float64, device=DEV)
    ws, need = ns.workspace(n)
    obb = (_lib.ctypes.c_double * 4)(*body.obb())
    outs = [_lib.ptrs([None] * 9) for _ in NAMES]
    for count, ids, code in ((0, [], _lib.WSB_ERR_ARG), (9, [2] * 9, _lib.WSB_ERR_ARG),
                             (2, [2, 42], _lib.WSB_ERR_UNSUPPORTED)):
        rc = _lib.lib.wsb_aggregate_groups(ns.handle, count, _lib.int32s(ids or [0]), _lib.PREC_FP64, _lib.ptr(pos),
                                           _lib.ptr(sup), None, n, _lib.ptr(body.pose_tensor(DEV)), obb, 0,
                                           _lib.OUT_ALL, *outs, _lib.ptr(ws), need, _stream())
        assert rc == code, (count, ids, rc)


def _single_into(c2s, kernel, views, mode):
    loops, X, h = c2s
    scene, rep, body = make_scene(loops)
    ns = rep.native(h, DEV)
    n = len(X)
    pos = torch.tensor(X, dtype=torch.float64, device=DEV)
    sup = torch.full((n,), h, dtype=torch.float64, device=DEV)
    ws, need = ns.workspace(n)
    obb = (_lib.ctypes.c_double * 4)(*body.obb())
    _lib.check(_lib.lib.wsb_aggregate(ns.handle, KERNEL_IDS[kernel], _lib.PREC_MIXED, _lib.ptr(pos), _lib.ptr(sup),
                                      None, n, _lib.ptr(body.pose_tensor(DEV)), obb, 0, mode,
                                      *[_lib.ptr(views[name]) for name in NAMES], _lib.ptr(ws), need, None,
                                      _stream()), "wsb_aggregate")
    torch.cuda.synchronize()


@pytest.mark.parametrize("kernel", ["cubic", "w4"])
def test_misaligned_outputs_and_the_add_mode(c2s, kernel):
    """outputs that are not 16 / 32-byte aligned (views one element into a buffer) get the same values as aligned
    ones, in both the assign and the add mode (the add mode on top of the first result doubles it exactly)."""
    n = len(c2s[1])
    widths = {"lam": 1, "G": 2, "Cov": 4, "m1": 2, "m2": 4}
    aligned = {k: torch.zeros(n * w, dtype=torch.float64, device=DEV) for k, w in widths.items()}
    raw = {k: torch.zeros(n * w + 1, dtype=torch.float64, device=DEV) for k, w in widths.items()}
    shifted = {k: raw[k][1:] for k in widths}
    assert shifted["G"].data_ptr() % 16 != 0
    for views in (aligned, shifted):
        _single_into(c2s, kernel, views, _lib.OUT_ALL | _lib.OUT_ASSIGN)
    for k in widths:
        assert torch.equal(aligned[k], shifted[k]), k
    first = {k: aligned[k].clone() for k in widths}
    for views in (aligned, shifted):
        _single_into(c2s, kernel, views, _lib.OUT_ALL)              # add a second time on top
    for k in widths:
        assert torch.equal(aligned[k], shifted[k]), k
        assert torch.equal(aligned[k], first[k] + first[k]), k


def test_wall_operator_groups_cover_vector_and_laplacian(c2s):
    """FusedWall with the delta+ groups it serves -- the smoothing kernel, lw2 (W'/r of w2) and cone: the 'lap' output
    (2 lam - tr Cov of the lw2 group, the wall Laplacian before the scheme's factor) and the cover vector (G of the cone
    group) against the oracle, and every group equal to its one-group FusedWall."""
    from helpers import oracle_outputs
    from warpsphboundaries_b200.provider import WallOutput
    loops, X, h = c2s
    scene, rep, body = make_scene(loops, center=(0.01, 0.02), angle=-0.4)
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    groups = (FusedGroup("w2"), FusedGroup("lw2"), FusedGroup("cone", (3, 4)))
    fw = FusedWall(scene, ps, h, groups)
    out = fw.evaluate([WallOutput("lap", 1, "lap"), WallOutput("cover", 2, "g0")])
    ref_l = oracle_outputs(loops, X, h, "lw2", h, center=(0.01, 0.02), angle=-0.4)
    ref_c = oracle_outputs(loops, X, h, "cone", h, center=(0.01, 0.02), angle=-0.4)
    lap_ref = 2.0 * ref_l["lam"] - (ref_l["Cov"][:, 0, 0] + ref_l["Cov"][:, 1, 1])
    assert np.abs(out["lap"][0].cpu().numpy() - lap_ref).max() < 1e-10
    assert np.abs((out["cover"][0].cpu().numpy() - ref_c["G"]) * h).max() < 1e-10
    for gi, g in enumerate(groups):
        one = FusedWall(scene, ps, h, (g,))
        for name in NAMES:
            assert torch.equal(fw.res[gi][name], one.res[0][name]), (g.kernel, name)


@pytest.mark.parametrize("kernel", ["w2p5", "w4p5"])
def test_tensile_group_gradient_matches_oracle(c2s, kernel):
    """the tensile group (W^5 of Wendland C2 / C4, chord quadrature): its G against the oracle's adaptive quadrature
    (pinned to the reference's 40-digit values), 1e-10 in units of 1/h; its other outputs are NaN, not numbers."""
    from oracle import edge2d as O
    loops, X, h = c2s
    X = X[:1500]
    scene, rep, body = make_scene(loops)
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    fw = FusedWall(scene, ps, h, (FusedGroup(kernel, (3, 4)),))
    from helpers import workloads
    V, E = workloads.edges_of(loops)
    ref = O.powered_gradient_local(V, E, X, h, kernel)
    got = fw.res[0]["G"][0].cpu().numpy()
    assert np.abs((got - ref) * h).max() < 1e-10
    assert np.abs(ref).max() > 1.0
    assert torch.isnan(fw.res[0]["lam"]).all()
    with pytest.raises(ValueError):
        from warpsphboundaries_b200.provider import WallOutput
        fw.evaluate([WallOutput("x", 0, "lam")])


def test_delta_plus_layout_aggregate(c2s):
    """AnalyticBoundary.aggregate without `lean`: the delta+ layout (w2, cone, lw2, w2p5) -- lam, G, Cov of the scheme
    kernel, the cover vector, the wall Laplacian and the tensile vector -- against the oracle."""
    from oracle import edge2d as O
    from helpers import oracle_outputs, workloads
    from warpsphboundaries_b200.provider import AnalyticBoundary
    from warpsphboundaries_b200.shim import KernelFunctions
    loops, X, h = c2s
    X = X[:1500]
    scene, rep, body = make_scene(loops)
    ps = ParticleState(torch.tensor(X, dtype=torch.float64, device=DEV),
                       torch.full((len(X),), h, dtype=torch.float64, device=DEV))
    fw = AnalyticBoundary(scene).aggregate(ps, h, kernel=KernelFunctions.Wendland2, laplacian=True)
    assert set(fw.out) == {"lam", "G", "Cov", "cover", "lap", "tens"}
    w = oracle_outputs(loops, X, h, "w2", h)
    assert np.abs(fw.out["lam"][0].cpu().numpy() - w["lam"]).max() < 1e-10
    c = oracle_outputs(loops, X, h, "cone", h)
    assert np.abs((fw.out["cover"][0].cpu().numpy() - c["G"]) * h).max() < 1e-10
    lw = oracle_outputs(loops, X, h, "lw2", h)
    lap = 2.0 * lw["lam"] - (lw["Cov"][:, 0, 0] + lw["Cov"][:, 1, 1])
    assert np.abs(fw.out["lap"][0].cpu().numpy() - lap).max() < 1e-10
    V, E = workloads.edges_of(loops)
    t = O.powered_gradient_local(V, E, X, h, "w2p5")
    assert np.abs((fw.out["tens"][0].cpu().numpy() - t) * h).max() < 1e-10
