"""The scene handle and the serving loop through the C ABI alone (wsb_scene_*, wsb_server_*, wsb_serve_*): a two-body
scene built from wsb_surface handles equals FusedWall on the same bodies, and a mixed stream of requests (two
kernels, two precisions, with and without the adjoint, some larger than one batch and run in chunks) gives every
request the result it gets alone, bit for bit."""
import ctypes

import numpy as np
import pytest
import torch

from tests.helpers import small_c2
from warpsphboundaries_b200 import _lib, workloads
from warpsphboundaries_b200.kernels import KERNEL_IDS
from warpsphboundaries_b200.provider import FusedGroup, FusedWall
from warpsphboundaries_b200.scene import Body, Scene, SurfaceRep
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu
L = _lib.lib
DEV = torch.device("cuda:0")
WIDTH = {"lam": 1, "G": 2, "Cov": 4, "m1": 2, "m2": 4}


def _surface(loops, h):
    V, E = workloads.edges_of(loops)
    V = np.ascontiguousarray(V, dtype=np.float64)
    E = np.ascontiguousarray(E, dtype=np.int32)
    s = ctypes.c_void_p()
    _lib.check(L.wsb_surface_create(_lib.dptr(V), len(V), E.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(E), 0,
                                    h, 0, ctypes.byref(s)))
    return s


@pytest.fixture(scope="module")
def two_bodies():
    loops, X, h = small_c2(n_particles=6000, n_polys=5, seed=21)
    s0, s1, s2 = _surface(loops[:2], h), _surface(loops[2:4], h), _surface(loops[4:], h)
    sc = ctypes.c_void_p()
    _lib.check(L.wsb_scene_create(0, ctypes.byref(sc)))
    ang = 0.4
    poses = [np.array([0.0, 0.0, 1.0, 0.0]), np.array([0.1, -0.05, np.cos(ang), np.sin(ang)])]
    b = ctypes.c_int()
    _lib.check(L.wsb_scene_add_body(sc, _lib.dptr(poses[0]), ctypes.byref(b)))
    _lib.check(L.wsb_scene_add_surface(sc, 0, s0))
    _lib.check(L.wsb_scene_add_surface(sc, 0, s1))
    _lib.check(L.wsb_scene_add_body(sc, _lib.dptr(poses[1]), ctypes.byref(b)))
    _lib.check(L.wsb_scene_add_surface(sc, 1, s2))
    yield dict(scene=sc, surfaces=(s0, s1, s2), loops=loops, X=X, h=h, angle=ang, center=(0.1, -0.05))
    L.wsb_scene_destroy(sc)
    for s in (s0, s1, s2):
        L.wsb_surface_destroy(s)


def _outs(B, n):
    return {k: torch.full((B * n * w,), float("nan"), dtype=torch.float64, device=DEV) for k, w in WIDTH.items()}


def test_scene_aggregate_equals_fused_wall(two_bodies):
    t = two_bodies
    X, h = t["X"], t["h"]
    n = len(X)
    pos = torch.tensor(X, dtype=torch.float64, device=DEV)
    sup = torch.full((n,), h, dtype=torch.float64, device=DEV)
    nb, ns = ctypes.c_int(), ctypes.c_int()
    _lib.check(L.wsb_scene_info(t["scene"], ctypes.byref(nb), ctypes.byref(ns)))
    assert (nb.value, ns.value) == (2, 3)
    ld = n + 17                                         # a row stride larger than n
    o = {k: torch.zeros(2 * ld * w, dtype=torch.float64, device=DEV) for k, w in WIDTH.items()}
    ws = torch.empty(int(L.wsb_scene_workspace_size(t["scene"], n)), dtype=torch.uint8, device=DEV)
    kid = _lib.int32s([KERNEL_IDS["w4"]])
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(L.wsb_scene_aggregate(t["scene"], 1, kid, _lib.PREC_FP64, _lib.ptr(pos), _lib.ptr(sup), None, n, ld,
                                     *[_lib.ptrs([o[k]]) for k in WIDTH], _lib.ptr(ws), ws.numel(), st))
    loops = t["loops"]
    body0 = Body(reps=[SurfaceRep.loops(loops[:2]), SurfaceRep.loops(loops[2:4])])
    body1 = Body(center=t["center"], angle=t["angle"], reps=[SurfaceRep.loops(loops[4:])])
    fw = FusedWall(Scene([body0, body1], DEV), ParticleState(pos, sup), h, (FusedGroup("w4"),))
    for k, w in WIDTH.items():
        got = o[k].reshape(2, ld, w)[:, :n]
        ref = fw.res[0][k].reshape(2, n, w)
        assert torch.equal(got, ref), k


def test_mixed_stream_equals_each_request_alone(two_bodies):
    t = two_bodies
    h = t["h"]
    rng = np.random.default_rng(5)
    Xall = np.concatenate([t["X"], rng.uniform(-0.1, 1.1, (20000, 2))])
    sizes = [700, 3000, 5000, 12000, 150, 4096, 9000, 1, 2500, 800]      # max_batch_rows 4096: some run in chunks
    kinds = [("w4", _lib.PREC_FP64, 0), ("w2", _lib.PREC_MIXED, 0), ("w4", _lib.PREC_FP64, 1), ("w4", _lib.PREC_FP64, 0),
             ("w2", _lib.PREC_MIXED, 0), ("w4", _lib.PREC_FP64, 1), ("w2", _lib.PREC_FP64, 0), ("w4", _lib.PREC_FP64, 0),
             ("w4", _lib.PREC_FP64, 0), ("w2", _lib.PREC_MIXED, 0)]
    reqs = []
    for n, (k, prec, grad) in zip(sizes, kinds):
        idx = rng.choice(len(Xall), n, replace=False)
        pos = torch.tensor(Xall[idx], dtype=torch.float64, device=DEV)
        sup = torch.full((n,), h, dtype=torch.float64, device=DEV) * torch.tensor(rng.uniform(0.8, 1.0, n), device=DEV)
        reqs.append(dict(n=n, kernel=KERNEL_IDS[k], prec=prec, grad=grad, pos=pos, sup=sup))

    def run(server_args, subset):
        srv = ctypes.c_void_p()
        _lib.check(L.wsb_server_create(0, *server_args, ctypes.byref(srv)))
        st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        results, ids = [], []
        for r in subset:
            o = _outs(2, r["n"])
            d = torch.full((r["n"] * 2,), float("nan"), dtype=torch.float64, device=DEV) if r["grad"] else None
            rid = ctypes.c_int64()
            _lib.check(L.wsb_serve_submit(srv, t["scene"], r["kernel"], r["prec"], r["grad"], _lib.ptr(r["pos"]),
                                          _lib.ptr(r["sup"]), r["n"], *[_lib.ptr(o[k]) for k in WIDTH], _lib.ptr(d),
                                          st, ctypes.byref(rid)))
            done = ctypes.c_int()
            _lib.check(L.wsb_serve_poll(srv, 0, ctypes.byref(done)))
            results.append((o, d))
            ids.append(rid.value)
        for rid in ids:
            _lib.check(L.wsb_serve_wait(srv, rid))
            done = ctypes.c_int()
            _lib.check(L.wsb_serve_poll(srv, rid, ctypes.byref(done)))
            assert done.value == 1
            _lib.check(L.wsb_serve_release(srv, rid))
        cnt, p50, p99, res = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double(), ctypes.c_size_t()
        _lib.check(L.wsb_server_stats(srv, ctypes.byref(cnt), ctypes.byref(p50), ctypes.byref(p99), ctypes.byref(res)))
        assert cnt.value == len(subset) and 0.0 <= p50.value <= p99.value
        assert res.value <= server_args[2]
        _lib.check(L.wsb_server_destroy(srv))
        return results

    mixed = run((3, 4096, 1 << 30), reqs)
    for r, (o, d) in zip(reqs, mixed):
        (o1, d1), = run((1, 4096, 1 << 30), [r])
        for k in WIDTH:
            assert not torch.isnan(o[k]).any(), k
            assert torch.equal(o[k], o1[k]), (r["n"], k)
        if r["grad"]:
            assert torch.equal(d, d1)
            assert not torch.isnan(d).any()


def test_budget_and_argument_errors(two_bodies):
    t = two_bodies
    srv = ctypes.c_void_p()
    _lib.check(L.wsb_server_create(0, 2, 4096, 1024, ctypes.byref(srv)))      # 1 KiB: no slot fits
    pos = torch.zeros((10, 2), dtype=torch.float64, device=DEV)
    sup = torch.full((10,), t["h"], dtype=torch.float64, device=DEV)
    rid = ctypes.c_int64()
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.wsb_serve_submit(srv, t["scene"], 2, 0, 0, _lib.ptr(pos), _lib.ptr(sup), 10, None, None, None, None, None,
                            None, st, ctypes.byref(rid))
    assert rc == _lib.WSB_ERR_SIZE
    rc = L.wsb_serve_submit(srv, t["scene"], 2, 0, 1, _lib.ptr(pos), _lib.ptr(sup), 10, None, None, None, None, None,
                            None, st, ctypes.byref(rid))
    assert rc == _lib.WSB_ERR_ARG                                           # grad without d_pos
    assert L.wsb_serve_release(srv, 12345) == _lib.WSB_ERR_ARG
    _lib.check(L.wsb_server_destroy(srv))
