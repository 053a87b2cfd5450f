"""The allocation-free aggregate entry point (wsb_aggregate_noalloc).

Hosts that link libwsb through its C ABI but cannot allocate device memory for it (their own allocator has reserved
the GPU's memory, or their time-step loop must not call cudaMalloc / cudaFree, which synchronise the device) call
this variant: it runs on a scratch array built into the library.  This test calls it twice in a row through the C ABI
and checks both results against the workspace entry point wsb_aggregate, within the float64 tolerance the other
parity tests use, and that an oversized request is refused with WSB_ERR_SIZE instead of running.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL64 = 1e-10


def _outputs(n, dev):
    return [torch.zeros(n, dtype=torch.float64, device=dev), torch.zeros((n, 2), dtype=torch.float64, device=dev),
            torch.zeros((n, 4), dtype=torch.float64, device=dev), torch.zeros((n, 2), dtype=torch.float64, device=dev),
            torch.zeros((n, 4), dtype=torch.float64, device=dev)]


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    from warpsphboundaries_b200 import _lib, workloads
    from warpsphboundaries_b200.kernels import KERNEL_IDS
    from warpsphboundaries_b200.scene import Body, SurfaceRep, _stream

    dev = torch.device("cuda", 0)
    loops = workloads.stars(5, (32, 200), seed=9, box=1.0, rmin=0.05, rmax=0.3)
    rng = np.random.default_rng(4)
    X = rng.uniform(-0.1, 1.1, size=(20000, 2))
    h = 0.02
    rep = SurfaceRep.loops(loops)
    body = Body(center=(0.1, -0.05), angle=0.4, reps=[rep])
    ns = rep.native(h, dev)
    pos = torch.tensor(X, dtype=torch.float64, device=dev)
    sup = torch.full((len(X),), h, dtype=torch.float64, device=dev)
    pose = body.pose_tensor(dev)
    obb = (ctypes.c_double * 4)(*body.obb())
    n = len(X)
    for kernel, prec in (("w4", _lib.PREC_FP64), ("cubic", _lib.PREC_MIXED)):
        kid = KERNEL_IDS[kernel]
        ref = _outputs(n, dev)
        ws, need = ns.workspace(n)
        _lib.check(_lib.lib.wsb_aggregate(ns.handle, kid, prec, _lib.ptr(pos), _lib.ptr(sup), None, n, _lib.ptr(pose),
                                          obb, 0, _lib.OUT_ALL, *[_lib.ptr(t) for t in ref], _lib.ptr(ws), need, None,
                                          _stream()), "wsb_aggregate")
        for call in range(2):
            got = _outputs(n, dev)
            _lib.check(_lib.lib.wsb_aggregate_noalloc(ns.handle, kid, prec, _lib.ptr(pos), _lib.ptr(sup), None, n,
                                                      _lib.ptr(pose), obb, 0, _lib.OUT_ALL,
                                                      *[_lib.ptr(t) for t in got], None, _stream()),
                       "wsb_aggregate_noalloc")
            torch.cuda.synchronize()
            scale = [1.0, h, 1.0, 1.0 / h, 1.0 / (h * h)]          # lam, G, Cov, m1, m2 in units of h
            for a, b, sc in zip(got, ref, scale):
                err = float(((a - b).abs() * sc).max())
                assert err < TOL64, (kernel, call, err)


def test_noalloc_refuses_requests_beyond_its_scratch():
    from warpsphboundaries_b200 import _lib, workloads
    from warpsphboundaries_b200.scene import Body, SurfaceRep

    dev = torch.device("cuda", 0)
    rep = SurfaceRep.loops(workloads.stars(2, (32, 64), seed=1, box=1.0))
    body = Body(reps=[rep])
    ns = rep.native(0.02, dev)
    pos = torch.zeros((4, 2), dtype=torch.float64, device=dev)
    sup = torch.full((4,), 0.02, dtype=torch.float64, device=dev)
    out = _outputs(4, dev)
    obb = (ctypes.c_double * 4)(*body.obb())
    # the row count is checked against the scratch size before anything is launched
    rc = _lib.lib.wsb_aggregate_noalloc(ns.handle, 2, _lib.PREC_FP64, _lib.ptr(pos), _lib.ptr(sup), None, 1 << 24,
                                        _lib.ptr(body.pose_tensor(dev)), obb, 0, _lib.OUT_ALL,
                                        *[_lib.ptr(t) for t in out], None, None)
    assert rc == _lib.WSB_ERR_SIZE
    assert "scratch" in _lib.last_error()


def test_noalloc_serves_its_documented_capacity():
    """131072 rows over a grid of at most 256 x 256 cells fit the built-in scratch, and the call runs."""
    from warpsphboundaries_b200 import _lib, workloads
    from warpsphboundaries_b200.scene import Body, SurfaceRep, _stream

    dev = torch.device("cuda", 0)
    loops = workloads.stars(3, (32, 64), seed=2, box=1.0)
    V = np.concatenate(loops)
    h = float((V.max(0) - V.min(0)).max()) / 250.0          # the grid spans the extent + 2 h in cells of h
    rep = SurfaceRep.loops(loops)
    body = Body(reps=[rep])
    ns = rep.native(h, dev)
    assert ns.info.nx <= 256 and ns.info.ny <= 256
    n = 131072
    assert _lib.lib.wsb_aggregate_workspace_size(ns.handle, n) <= 16 << 20
    pos = torch.rand((n, 2), dtype=torch.float64, device=dev)
    sup = torch.full((n,), h, dtype=torch.float64, device=dev)
    out = _outputs(n, dev)
    obb = (ctypes.c_double * 4)(*body.obb())
    _lib.check(_lib.lib.wsb_aggregate_noalloc(ns.handle, 2, _lib.PREC_FP64, _lib.ptr(pos), _lib.ptr(sup), None, n,
                                              _lib.ptr(body.pose_tensor(dev)), obb, 0, _lib.OUT_ALL,
                                              *[_lib.ptr(t) for t in out], None, _stream()), "wsb_aggregate_noalloc")
    torch.cuda.synchronize()
    assert torch.isfinite(out[0]).all()
