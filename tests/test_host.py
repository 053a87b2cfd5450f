"""Host-side logic that needs no GPU: orientation, shims, error paths, workload generators."""
import numpy as np
import pytest
import torch

from warpsphboundaries_b200 import shim, workloads
from warpsphboundaries_b200.scene import Body, Pose, SurfaceRep


def test_polygon_orientation_ccw_inside_cw_outside():
    sq = [(0, 0), (0, 1), (1, 1), (1, 0)]                     # clockwise input
    r = SurfaceRep.polygon(sq)
    V = r.vertices.numpy()
    a = np.sum(V[:, 0] * np.roll(V[:, 1], -1) - np.roll(V[:, 0], -1) * V[:, 1])
    assert a > 0 and r.background == 0
    o = SurfaceRep.polygon(sq, solid="outside")
    V = o.vertices.numpy()
    assert np.sum(V[:, 0] * np.roll(V[:, 1], -1) - np.roll(V[:, 0], -1) * V[:, 1]) < 0 and o.background == 1


def test_loops_rep_concatenates_ccw():
    loops = workloads.stars(3, (16, 16), seed=3)
    r = SurfaceRep.loops(loops)
    assert r.vertices.shape == (48, 2) and r.edges.shape == (48, 2)
    assert int(r.edges[15, 1]) == 0 and int(r.edges[16, 0]) == 16


def test_pose_to_local_matches_formula():
    p = torch.tensor([[1.0, 2.0], [-0.5, 0.25]], dtype=torch.float64)
    pose = Pose(torch.tensor([0.3, -0.1], dtype=torch.float64), 0.7)
    loc = pose.toLocal(p)
    back = pose.toWorld(loc)
    assert torch.allclose(back, p, atol=1e-15)


def test_kernel_names_and_unsupported():
    assert shim.kernelName(shim.KernelFunctions.Wendland4) == "w4"
    assert shim.kernelName(shim.KernelFunctions.CubicSpline) == "cubic"
    with pytest.raises(NotImplementedError):
        shim.kernelName(shim.KernelFunctions.Gaussian)
    with pytest.raises(KeyError):
        shim.kernelName("nope")


def test_query_allowed_directions():
    ps = shim.ParticleState(torch.zeros(4, 2), torch.ones(4), kinds=torch.tensor([0, 1, 2, 0]))
    a = shim.queryAllowed(ps, shim.OperationDirection.BoundaryToFluid, "cpu")
    assert a.tolist() == [True, False, False, True]
    a = shim.queryAllowed(ps, shim.OperationDirection.FluidToFluid, "cpu")
    assert a.tolist() == [False] * 4


def test_body_kinematics_formulas_on_cpu_tensors():
    b = Body(center=(0.5, 0.0), angle=0.2, linearVelocity=(1.0, 0.0), angularVelocity=2.0, reps=[])
    x = torch.tensor([[0.5, 1.0]], dtype=torch.float64)
    assert torch.allclose(b.velocityAt(x), torch.tensor([[-1.0, 0.0]], dtype=torch.float64))


def test_workload_shapes():
    loops, X, h = workloads.c2(n_particles=4096)
    assert len(loops) == 64 and X.shape == (4096, 2) and h == 0.02
    assert all(32 <= len(L) <= 512 for L in loops)
    loops, X, h = workloads.c1()
    assert X.shape == (4096, 2) and len(loops[0]) == 256


def test_box_rep_is_the_outline_polygon():
    """BoxRep (scene.py:459-506): an obstacle is the counter-clockwise outline, a tank the clockwise outline with
    background 1; bounds, argument checks and the box's signed distance (positive in the fluid, normal into it)."""
    import torch
    from warpsphboundaries_b200.scene import BoxRep
    ob = BoxRep((0.1, -0.2), (2.3, 1.1))
    tk = BoxRep((0.1, -0.2), (2.3, 1.1), "outside")
    for rep, sign, bg in ((ob, 1.0, 0), (tk, -1.0, 1)):
        V = rep.vertices.numpy()
        area2 = float(np.sum(V[:, 0] * np.roll(V[:, 1], -1) - np.roll(V[:, 0], -1) * V[:, 1]))
        assert np.isclose(area2, sign * 2 * 2.2 * 1.3) and rep.background == bg
        lo, hi = rep.bounds()
        assert lo.tolist() == [0.1, -0.2] and hi.tolist() == [2.3, 1.1]
        assert rep.surface() is rep and rep.kind == "box"
    lp = torch.tensor([[0.0, 0.0], [1.0, 0.5], [3.0, 2.0], [1.2, 1.0]], dtype=torch.float64)
    d, n = ob.signed(lp)
    assert np.allclose(d.numpy(), [0.1, -0.6, np.hypot(0.7, 0.9), -0.1])
    assert np.allclose(n.numpy(), [[-1, 0], [0, 1], [0.7 / np.hypot(0.7, 0.9), 0.9 / np.hypot(0.7, 0.9)], [0, 1]])
    dt, nt = tk.signed(lp)
    assert np.allclose(dt.numpy(), -d.numpy()) and np.allclose(nt.numpy()[[0, 1, 3]], -n.numpy()[[0, 1, 3]])
    for bad in (((0, 0), (0, 1)), ((1, 0), (0, 1))):
        with pytest.raises(ValueError):
            BoxRep(*bad)
    with pytest.raises(ValueError):
        BoxRep((0, 0), (1, 1), "middle")


def _sdf_fixture():
    import json
    import sys
    from pathlib import Path
    here = Path(__file__).parent / "golden"
    sys.path.insert(0, str(here))
    import make_golden
    return make_golden.sdf_grids(), json.loads((here / "sdf_contour_golden.json").read_text())["cases"]


def test_marching_squares_equals_the_reference_contours():
    """the zero contour of sampled distances (scene.py:762-805): vertices, edges and background bit-identical to the
    reference's marching squares on a disk, a tank, two merging disks, a ring and both saddle resolutions."""
    from warpsphboundaries_b200.scene import _marching_squares
    grids, cases = _sdf_fixture()
    for (name, d, origin, sp), c in zip(grids, cases):
        rep = _marching_squares(d, origin, sp)
        assert np.array_equal(rep.vertices.numpy(), np.array(c["vertices"])), name
        assert np.array_equal(rep.edges.numpy(), np.array(c["edges"])), name
        assert rep.background == c["background"], name


def test_contours_are_oriented_and_closed():
    """the winding number of the contour (oracle angle sum) equals d < 0 at random points farther than one grid
    spacing from the zero level set: the loops are closed and carry the solid on their left."""
    from oracle.cone_area import winding
    from warpsphboundaries_b200.scene import _marching_squares
    grids, _ = _sdf_fixture()
    rng = np.random.default_rng(1)
    for name, d, origin, sp in grids[:4]:
        rep = _marching_squares(d, origin, sp)
        xs = origin[0] + sp * np.arange(d.shape[0])
        from scipy.interpolate import RegularGridInterpolator
        f = RegularGridInterpolator((xs, xs), d)
        P = rng.uniform(xs[0], xs[-1], (2000, 2))
        dv = f(P)
        far = np.abs(dv) > sp
        w = winding(P[far], rep.vertices.numpy(), rep.edges.numpy()) + rep.background
        assert np.array_equal(w > 0.5, dv[far] < 0), name


def test_contour_rejects_bad_grids():
    from warpsphboundaries_b200.scene import SdfRep, _marching_squares
    d = np.ones((5, 5))
    with pytest.raises(ValueError):
        _marching_squares(d, (0, 0), 0.1)                  # no zero level set
    d[0, 2] = -1.0
    with pytest.raises(ValueError):
        _marching_squares(d, (0, 0), 0.1)                  # a mixed border
    with pytest.raises(ValueError):
        SdfRep(np.ones((3, 3)), (0, 0), 0.0)


def test_implicit_lowering_host_logic():
    """ImplicitRep (scene.py:558-596): a cavity disk lowers to its area-preserving polygon with
    max(24, ceil(2 pi R / (h / 16))) edges, cached; a solid disk to a one-disk DiskArrayRep; a half plane has no
    exact form."""
    from warpsphboundaries_b200.implicit import DiskBody, HalfPlaneBody, TierPolicy
    from warpsphboundaries_b200.scene import ImplicitRep
    cav = ImplicitRep(DiskBody((0.2, -0.1), 0.9, solid="outside"))
    s = cav.lowered(0.1, "cpu")
    n = max(24, int(np.ceil(2 * np.pi * 0.9 / (0.1 / 16))))
    assert len(s.edges) == n and s.background == 1 and cav.lowered(0.1, "cpu") is s
    V = s.vertices.numpy()
    area = 0.5 * abs(np.sum(V[:, 0] * np.roll(V[:, 1], -1) - np.roll(V[:, 0], -1) * V[:, 1]))
    assert abs(area - np.pi * 0.81) < 1e-12                 # area preserving
    assert len(ImplicitRep(DiskBody((0, 0), 0.01, "outside")).lowered(0.1, "cpu").edges) == 24
    assert len(ImplicitRep(DiskBody((0, 0), 0.9, "outside"), TierPolicy(maxPolygonEdgeOverH=0.5)).lowered(
        0.1, "cpu").edges) == int(np.ceil(2 * np.pi * 0.9 / 0.05))
    from warpsphboundaries_b200.scene import DiskArrayRep
    solid = ImplicitRep(DiskBody((0.3, 0.1), 0.5)).lowered(0.1, "cpu")
    assert isinstance(solid, DiskArrayRep) and solid.centres.tolist() == [[0.3, 0.1]] and solid.radii.tolist() == [0.5]
    with pytest.raises(NotImplementedError):
        ImplicitRep(HalfPlaneBody((0, 0), (0, 1))).lowered(0.1, "cpu")
    b = Body(reps=[cav])
    assert b.unbounded() and b.fusable()
    assert Body(reps=[ImplicitRep(DiskBody((0, 0), 0.5))]).fusable()
    assert not Body(reps=[ImplicitRep(HalfPlaneBody((0, 0), (0, 1)))]).fusable()
    d, nrm, kap = DiskBody((0.0, 0.0), 1.0).signed(torch.tensor([[2.0, 0.0]], dtype=torch.float64))
    assert float(d[0]) == 1.0 and nrm.tolist() == [[1.0, 0.0]] and kap == 1.0
    d, nrm, _ = HalfPlaneBody((0.0, 1.0), (0.0, 1.0)).signed(torch.tensor([[3.0, 0.5]], dtype=torch.float64))
    assert float(d[0]) == -0.5 and nrm.tolist() == [[0.0, 1.0]]


def test_disk_array_host_logic():
    """DiskArrayRep (scene.py:808-905): bounds, argument checks and the signed distance to the nearest circle."""
    from warpsphboundaries_b200.scene import DiskArrayRep
    d = DiskArrayRep([[0.0, 0.0], [3.0, 1.0]], [1.0, 0.5])
    lo, hi = d.bounds()
    assert lo.tolist() == [-1.0, -1.0] and hi.tolist() == [3.5, 1.5]
    sd, n = d.signed(torch.tensor([[2.0, 0.0], [0.5, 0.0], [3.0, 2.0]], dtype=torch.float64))
    assert np.allclose(sd.numpy(), [np.hypot(1, 1) - 0.5, -0.5, 0.5]) and np.allclose(n.numpy()[1:], [[1, 0], [0, 1]])
    with pytest.raises(ValueError):
        DiskArrayRep([[0.0, 0.0]], [1.0, 2.0])
    with pytest.raises(ValueError):
        DiskArrayRep([[0.0, 0.0]], [0.0])


def test_pair_weights_host_checks():
    """fem.pair_weights (warpbc.py:486-510 signature) refuses unknown kernels and CPU devices before any launch, and
    the C entry point refuses NULL arrays and unknown kernel ids without a device."""
    from warpsphboundaries_b200 import _lib
    from warpsphboundaries_b200.fem import pair_weights
    V = np.array([[0.0, 0.0], [1.0, 0.0], [0.0, 1.0]])
    E = np.array([[0, 1, 2]])
    with pytest.raises(NotImplementedError):
        pair_weights([0], [0], [[0.2, 0.2]], [0.5], V, E, "w2p5", device="cuda")
    with pytest.raises(RuntimeError):
        pair_weights([0], [0], [[0.2, 0.2]], [0.5], V, E, "w2", device="cpu")
    L = _lib.lib
    nul = (None, None, 4, None, None, 1, None, 3, None, 1, None, None, None, None)
    assert L.wsb_pair_weights(1, *nul) == _lib.WSB_ERR_ARG
    assert L.wsb_pair_weights(10, *nul) == _lib.WSB_ERR_UNSUPPORTED
    assert L.wsb_pair_weights(1, None, None, 4, None, None, -1, None, 3, None, 1, None, None, None, None) == \
        _lib.WSB_ERR_ARG
    assert L.wsb_pair_weights(1, None, None, 0, None, None, 1, None, 3, None, 1, None, None, None, None) == _lib.WSB_OK


def test_scene_and_server_argument_checks():
    """the scene and server entry points refuse NULL handles and out-of-range arguments before touching a device."""
    import ctypes
    from warpsphboundaries_b200 import _lib
    L = _lib.lib
    assert L.wsb_scene_create(0, None) == _lib.WSB_ERR_ARG
    assert L.wsb_scene_add_body(None, None, None) == _lib.WSB_ERR_ARG
    assert L.wsb_scene_add_surface(None, 0, None) == _lib.WSB_ERR_ARG
    assert L.wsb_scene_info(None, None, None) == _lib.WSB_ERR_ARG
    assert L.wsb_scene_workspace_size(None, 10) == 0
    assert L.wsb_scene_destroy(None) == _lib.WSB_OK
    out = ctypes.c_void_p()
    assert L.wsb_server_create(0, 0, 1024, 1 << 20, ctypes.byref(out)) == _lib.WSB_ERR_ARG      # no streams
    assert L.wsb_server_create(0, 2, 0, 1 << 20, ctypes.byref(out)) == _lib.WSB_ERR_ARG         # no rows
    assert L.wsb_server_create(0, 2, 1024, 1 << 20, None) == _lib.WSB_ERR_ARG
    assert L.wsb_serve_poll(None, 0, None) == _lib.WSB_ERR_ARG
    assert L.wsb_serve_wait(None, 1) == _lib.WSB_ERR_ARG
    assert L.wsb_serve_release(None, 1) == _lib.WSB_ERR_ARG
    assert L.wsb_server_stats(None, None, None, None, None) == _lib.WSB_ERR_ARG
    assert L.wsb_server_destroy(None) == _lib.WSB_OK
