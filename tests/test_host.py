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
