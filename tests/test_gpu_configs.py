"""GPU parity on the benchmark scenes at their stated sizes, through the public API and the C ABI.

c2  2^20 particles in [0, 4]^2, 64 star polygons (one multi-loop surface), h = 0.02: the device evaluates every row
    for cubic, w2, w4 and w6 in one FusedWall (the bench's step), on the float64, mixed and float routes; a seeded
    10 000-row subset -- every near-tangent and endpoint-on-circle particle, 6 000 rows with neighbour pairs, the rest
    uniform -- is compared with the oracle channel by channel, and its neighbour slots bit for bit.
c3  2^21 particles in [-1, 1]^3 plus 8 planted queries 1e-7 h off vertices, edge midpoints and face centres, the
    jittered 20 480-face icosphere, h = 0.03, w2 / w4 / w6: 64 rows against oracle values computed once by
    tests/golden/make_config_fixtures.py (the 3-D oracle costs ~35 s a query on this surface).
c4  2^18 particles, 16 star polygons of 128 vertices, h = 0.02, w4: forward and adjoint over all rows; 256 near-wall
    rows against the reference's own torch2d values and autograd gradients (tests/golden/torch2d_c4.npz, made by
    tests/golden/make_golden.py) and central differences of the full-size forward.

Relative error per channel: |got - ref| / max(|ref|, FLOOR) with every channel in its natural unit of h (lam and g1
as they are, m1 / h, m2 / h^2, G * h; 3-D: y^alpha moments / h^|alpha|, gradient moments / h^(|alpha| - 1), Hessian
* h^2), where each channel is O(1) at a wall; FLOOR = 1e-3.
"""
import json
from pathlib import Path

import numpy as np
import pytest
import torch

from oracle import edge2d as O
from warpsphboundaries_b200 import workloads
from warpsphboundaries_b200.autograd import aggregate_moments
from warpsphboundaries_b200.fixedadj import fixed_topology
from warpsphboundaries_b200.provider import FusedGroup, FusedWall
from warpsphboundaries_b200.scene import Body, Scene, SurfaceRep
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu
DEV = "cuda"
GOLD = Path(__file__).parent / "golden"
FLOOR = 1e-3
C2_KERNELS = ["cubic", "w2", "w4", "w6"]
CH12 = ["lam", "m10", "m01", "m20", "m11", "m02", "Gx", "Gy", "g1xx", "g1xy", "g1yx", "g1yy"]


def rel_err(got, ref):
    """per column: max over rows of |got - ref| / max(|ref|, FLOOR), and the max absolute error."""
    d = np.abs(got - ref)
    return (d / np.maximum(np.abs(ref), FLOOR)).max(0), d.max(0)


def report(title, names, rel, ab):
    print(f"\n{title}")
    for n, r, a in zip(names, rel, ab):
        print(f"  {n:>6}  rel {r:.2e}  abs {a:.2e}")


def twelve_from_world(res, h):
    """[n, 12] in report order, natural units (identity pose: world = body frame)."""
    lam, m1, G, cov, m2 = (np.asarray(res[k]) for k in ("lam", "m1", "G", "Cov", "m2"))
    return np.stack([lam, m1[:, 0] / h, m1[:, 1] / h, m2[:, 0, 0] / h ** 2, m2[:, 0, 1] / h ** 2, m2[:, 1, 1] / h ** 2,
                     G[:, 0] * h, G[:, 1] * h, cov[:, 0, 0], cov[:, 0, 1], cov[:, 1, 0], cov[:, 1, 1]], 1)


def twelve_from_local(out12, h):
    """the oracle's [n, 12] local channels (physical units) in report order, natural units."""
    o = out12
    return np.stack([o[:, 0], o[:, 1] / h, o[:, 2] / h, o[:, 9] / h ** 2, o[:, 10] / h ** 2, o[:, 11] / h ** 2,
                     o[:, 3] * h, o[:, 4] * h, o[:, 5], o[:, 6], o[:, 7], o[:, 8]], 1)


# ------------------------------------------------------------------------------------------------------------- c2
@pytest.fixture(scope="module")
def c2_run():
    loops, X, h, special = workloads.c2(return_special=True)
    N = len(X)
    rep = SurfaceRep.loops(loops)
    scene = Scene([Body(reps=[rep])], DEV)
    pos = torch.tensor(X, dtype=torch.float64, device=DEV)
    sup = torch.full((N,), h, dtype=torch.float64, device=DEV)
    ps = ParticleState(pos, sup)
    groups = tuple(FusedGroup(k) for k in C2_KERNELS)
    got = {}
    for prec in ("fp64", "mixed", "fp32"):
        fw = FusedWall(scene, ps, h, groups, precision=prec)
        got[prec] = [{k: v[0] for k, v in r.items()} for r in fw.res]
    ft = fixed_topology(rep, pos, sup, torch.ones(N, dtype=torch.bool, device=DEV), h)
    K = ft.K
    e = ft.e.reshape(N, K)
    npairs = (e >= 0).sum(1).cpu().numpy()
    rng = np.random.default_rng(10)
    spec = np.concatenate([special["tangent"], special["vertex"]])
    with_pairs = np.setdiff1d(np.nonzero(npairs > 0)[0], spec)
    rows = np.concatenate([spec, rng.choice(with_pairs, 6000, replace=False)])
    rest = np.setdiff1d(np.arange(N), rows)
    rows = np.concatenate([rows, rng.choice(rest, 10000 - len(rows), replace=False)])
    rt = torch.tensor(rows, device=DEV)
    sub = {prec: [{k: v[rt].cpu().numpy() for k, v in r.items()} for r in got[prec]] for prec in got}
    slots = e[rt].cpu().numpy()
    V, E = workloads.edges_of(loops)
    Xs = X[rows]
    hs = np.full(len(rows), h)
    cl = O.build_cell_list(V, E, h)
    ind = O.indicator_binned(V, E, 0, Xs, hs, cl)
    ref = {k: O.local_twelve(V, E, 0, Xs, hs, k, h, ind=ind, cl=cl) for k in C2_KERNELS}
    ref_slots = O.fixed_slots(V, E, cl, Xs, hs)
    return dict(loops=loops, h=h, rows=rows, special=spec, sub=sub, ref=ref, slots=slots, ref_slots=ref_slots,
                ind=ind, gpu_ind=ft.ind[rt].cpu().numpy(), npairs=npairs, X=X)


def test_c2_neighbour_slots_bit_exact_at_full_size(c2_run):
    """the 10 000 subset rows' neighbour edges (set and order) and indicators from the 2^20-row launch equal the
    oracle's; the near-tangent rows (distance h (1 - eps) to an edge line, eps down to 1e-9) included."""
    r = c2_run
    n = 0
    for k in range(len(r["rows"])):
        got = r["slots"][k][r["slots"][k] >= 0]
        assert np.array_equal(got, r["ref_slots"][k]), (k, r["rows"][k])
        assert np.all(r["slots"][k][len(got):] == -1)
        n += len(got)
    assert n > 10000
    exact = r["ind"] == np.round(r["ind"])
    assert np.array_equal(r["gpu_ind"][exact], r["ind"][exact])
    assert np.abs(r["gpu_ind"] - r["ind"]).max() < 1e-12
    assert len(r["special"]) > 200 and (r["npairs"][r["special"]] > 0).mean() > 0.9


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-8), ("mixed", 1e-4), ("fp32", 1e-3)])
def test_c2_twelve_channels_relative_error_at_full_size(c2_run, prec, tol):
    """lambda and the twelve moments of cubic, w2, w4 and w6 on the 10 000 subset rows of the 2^20-row launch against
    the float64 oracle: the per-channel relative error (floor 1e-3 in natural units) within `tol` for every channel
    and kernel, also on the near-tangent and endpoint-on-circle rows alone.  Tolerances: float64 1e-8 (absolute
    differences stay below 1e-12; at the floor that is the oracle's own float64 cancellation in its monomial term
    plan, up to ~4e3 for w6); mixed 1e-4 (the float chord angle: ~1e-7 absolute, so the mixed route does not reach
    1e-6 relative at the floor); float route 1e-3 (float32 chord sums, ~1e-6 absolute)."""
    r = c2_run
    h = r["h"]
    worst = 0.0
    spec = np.isin(r["rows"], r["special"])
    for gi, k in enumerate(C2_KERNELS):
        got = twelve_from_world(r["sub"][prec][gi], h)
        ref = twelve_from_local(r["ref"][k], h)
        rel, ab = rel_err(got, ref)
        rel_s, _ = rel_err(got[spec], ref[spec])
        report(f"c2 {prec} {k}: worst per channel over {len(got)} rows (special rows alone: max {rel_s.max():.2e})",
               CH12, rel, ab)
        assert rel.max() <= tol, (k, dict(zip(CH12, rel)))
        worst = max(worst, rel.max())
    print(f"c2 {prec}: worst relative error {worst:.2e}")


# ------------------------------------------------------------------------------------------------------------- c3
C3_SCALE_POW = [0, 1, 1, 1, 2, 2, 2, 2, 2, 2] + [-1] * 3 + [0] * 9 + [-2] * 6   # h power of each of the 28 channels


def test_c3_closed_surface_at_full_size():
    """the 28 baseline channels of the 2^21-particle 3-D scene (and 8 planted queries 1e-7 h off vertices, edges and
    face centres), launched in one call per kernel over all rows; 64 rows against the oracle values."""
    from warpsphboundaries_b200.mesh3d import ClosedMesh
    fx = json.loads((GOLD / "c3_subset.json").read_text())
    V, Fc, X, h = workloads.c3()
    assert h == fx["h"]
    Q = np.concatenate([X, np.asarray(fx["planted"])])
    rows = np.concatenate([np.asarray(fx["rows"]), len(X) + np.arange(len(fx["planted"]))])
    assert np.array_equal(Q[rows], np.asarray(fx["queries"]))
    m = ClosedMesh(V, Fc, h, DEV)
    pos = torch.tensor(Q, dtype=torch.float64, device=DEV)
    sup = torch.full((len(Q),), h, dtype=torch.float64, device=DEV)
    rt = torch.tensor(rows, device=DEV)
    scale = h ** np.asarray(C3_SCALE_POW, float)
    names = [f"c{j}" for j in range(28)]
    for k in fx["kernels"]:
        out = m.channels(pos, sup, k)
        got = out[rt].cpu().numpy() / scale
        ref = np.asarray(fx["values"][k]) / scale
        rel, ab = rel_err(got, ref)
        report(f"c3 {k}: worst per channel over {len(rows)} rows", names, rel, ab)
        # the oracle sums the full-face solid angles and edge primitives of all 20 480 faces in float64: differences
        # up to ~1e-10 absolute (1e-8 relative at the floor) are within its accumulated rounding
        assert rel.max() <= 5e-8 and ab.max() <= 5e-10, (k, rel.max(), int(np.argmax(rel)), ab.max())
        del out


# ------------------------------------------------------------------------------------------------------------- c4
C4_ALPHAS = [(0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2)]


def _moment(out, al):
    if al == (0, 0):
        return out["lam"]
    if sum(al) == 1:
        return out["m1"][:, 0 if al == (1, 0) else 1]
    return {(2, 0): out["m2"][:, 0, 0], (1, 1): out["m2"][:, 0, 1], (0, 2): out["m2"][:, 1, 1]}[al]


def test_c4_gradients_at_full_size():
    """forward and adjoint over all 2^18 rows of the gradient scene: for every moment alpha (|alpha| <= 2) the values,
    d m_alpha / dx of 256 near-wall rows and d sum_rows m_alpha / d vertex against the reference's torch2d autograd
    (1e-10 in units of h^(|alpha| - 1)), and d lam / dx, d m1 / dx and d lam / d vertex against central differences
    of the full-size forward (step 1e-6, float64)."""
    g = np.load(GOLD / "torch2d_c4.npz")
    loops, X, h = workloads.c4()
    rows = g["rows"]
    assert np.array_equal(X[rows], g["particles"])
    rep = SurfaceRep.loops(loops)
    body = Body(reps=[rep])
    N = len(X)
    sup = torch.full((N,), h, dtype=torch.float64, device=DEV)
    rt = torch.tensor(rows, device=DEV)
    for al in C4_ALPHAS:
        key = f"{al[0]}{al[1]}"
        pos = torch.tensor(X, dtype=torch.float64, device=DEV, requires_grad=True)
        rep.vertices.requires_grad_(True)
        out = aggregate_moments(body, rep, pos, sup, "w4", h)
        m = _moment(out, al)
        gx, gv = torch.autograd.grad(m[rt].sum(), [pos, rep.vertices])
        rep.vertices.requires_grad_(False)
        sc = h ** (al[0] + al[1] - 1)
        em = np.abs(m[rt].detach().cpu().numpy() - g["m_" + key]).max() / (sc * h)
        ex = np.abs(gx[rt].cpu().numpy() - g["dx_" + key]).max() / sc
        ev = np.abs(gv.cpu().numpy() - g["dv_" + key].reshape(-1, 2)).max() / sc
        print(f"c4 alpha {al}: value {em:.2e}, d/dx {ex:.2e}, d/dvertex {ev:.2e} (units of h^(|alpha|-1))")
        assert em < 1e-10 and ex < 1e-10 and ev < 1e-10, (al, em, ex, ev)
        others = torch.ones(N, dtype=torch.bool, device=DEV)
        others[rt] = False
        assert float(gx[others].abs().max()) == 0.0                         # rows outside the loss: no gradient
    # central differences of the full-size forward
    rng = np.random.default_rng(12)
    wl = torch.zeros(N, dtype=torch.float64, device=DEV)
    w1 = torch.zeros((N, 2), dtype=torch.float64, device=DEV)
    wl[rt] = torch.tensor(rng.normal(size=len(rows)), device=DEV)
    w1[rt] = torch.tensor(rng.normal(size=(len(rows), 2)), device=DEV)

    def loss(Xa, verts=None):
        r, b = (rep, body) if verts is None else (SurfaceRep(verts, rep.edges.cpu().numpy(), conditioned=False), None)
        b = body if verts is None else Body(reps=[r])
        o = aggregate_moments(b, r, torch.as_tensor(Xa, dtype=torch.float64, device=DEV), sup, "w4", h)
        return float((o["lam"] * wl).sum() + (o["m1"] * w1).sum())

    pos = torch.tensor(X, dtype=torch.float64, device=DEV, requires_grad=True)
    rep.vertices.requires_grad_(True)
    o = aggregate_moments(body, rep, pos, sup, "w4", h)
    gx, gv = torch.autograd.grad((o["lam"] * wl).sum() + (o["m1"] * w1).sum(), [pos, rep.vertices])
    rep.vertices.requires_grad_(False)
    gx, gv = gx.cpu().numpy(), gv.cpu().numpy()
    step = 1e-6
    sx, sv = np.abs(gx).max(), np.abs(gv).max()
    for i in rows[::32]:
        for c in range(2):
            Xp, Xm = X.copy(), X.copy()
            Xp[i, c] += step
            Xm[i, c] -= step
            fd = (loss(Xp) - loss(Xm)) / (2 * step)
            assert abs(fd - gx[i, c]) < 1e-6 * sx, (i, c, fd, gx[i, c])
    V0 = rep.vertices.detach().cpu().numpy()
    hot = np.argsort(-np.abs(gv).max(1))[:8]
    for k in hot:
        for c in range(2):
            Vp, Vm = V0.copy(), V0.copy()
            Vp[k, c] += step
            Vm[k, c] -= step
            fd = (loss(X, Vp) - loss(X, Vm)) / (2 * step)
            assert abs(fd - gv[k, c]) < 1e-6 * sv, (k, c, fd, gv[k, c])


def test_c2_row_sums_agree_with_correctly_rounded_sums(c2_run):
    """the device sums each row's pair channels in a fixed order without compensation (the reference sums with Kahan /
    Neumaier compensation, fluxbridge/evaluate.py:177-187, wp_func.py:335-356).  On the 400 subset rows with the
    most neighbour pairs, the fused float64 pass's channels stay within 4e-15 (natural units) of the correctly
    rounded sum (math.fsum) of the same closed form's per-pair channels (wsb_pair_channels) plus the indicator term:
    the uncompensated sum of these bounded terms loses nothing a compensated one would keep."""
    import ctypes
    import math
    from oracle import edge2d as O2
    from warpsphboundaries_b200 import _lib
    from warpsphboundaries_b200.kernels import KERNEL_IDS
    from warpsphboundaries_b200.scene import _stream
    r = c2_run
    h = r["h"]
    counts = np.array([len(s) for s in r["ref_slots"]])
    top = np.argsort(-counts)[:400]
    assert counts[top].min() >= 8
    rep = SurfaceRep.loops(r["loops"])
    lpos = torch.tensor(r["X"][r["rows"][top]], dtype=torch.float64, device=DEV)
    lsup = torch.full((len(top),), h, dtype=torch.float64, device=DEV)
    topo = rep.topology(lpos, lsup)
    qi = topo.qi.to(torch.int32).contiguous()
    e = topo.e.to(torch.int32).contiguous()
    P = len(qi)
    ns = rep.native(h, DEV)
    worst = 0.0
    for gi, k in enumerate(C2_KERNELS):
        c = torch.empty((P, 12), dtype=torch.float64, device=DEV)
        st = torch.zeros(1, dtype=torch.int32, device=DEV)
        _lib.check(_lib.lib.wsb_pair_channels(ns.handle, KERNEL_IDS[k], _lib.PREC_FP64, _lib.ptr(qi), _lib.ptr(e), P,
                                              _lib.ptr(lpos), _lib.ptr(lsup), len(top), _lib.ptr(c), _lib.ptr(st),
                                              _stream()))
        cc = c.cpu().numpy()
        q = qi.cpu().numpy()
        plane = np.array(O2.plane_channels(k))
        phys = np.array([1, h, h, 1 / h, 1 / h, 1, 1, 1, 1, h * h, h * h, h * h])
        exact = np.zeros((len(top), 12))
        for t in range(len(top)):
            sel = cc[q == t]
            w = r["ind"][top[t]]
            exact[t] = [math.fsum(list(sel[:, j]) + [w * plane[j]]) * phys[j] for j in range(12)]
        got = twelve_from_world(r["sub"]["fp64"][gi], h)[top]
        d = np.abs(got - twelve_from_local(exact, h)).max()
        worst = max(worst, d)
        assert d < 4e-15, (k, d)
    print(f"c2 fp64 vs correctly rounded row sums (400 rows with the most pairs): {worst:.1e}")
