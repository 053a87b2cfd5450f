"""B200-native exact SPH boundary integrals (2-D polygonal walls): a drop-in for the boundary-integral hot path of
warpSPHBoundaries' `AnalyticBoundary` / `BoundaryProvider`, computed by hand-written sm_100a CUDA kernels in
libwsb.so (include/wsb.h).  There is no CPU fallback: the compute entry points raise if the library is missing.
"""
from .kernels import KERNEL_IDS, kernel, plane_channels
from .shim import (GradientScheme, KernelFunctions, OperationDirection, OperationProperties, ParticleState,
                   WarpOperation, kernelName, queryAllowed)


def __getattr__(name):
    # the GPU-facing modules load libwsb.so on first use, so the exact algebra and the shims import without it
    if name in ("Scene", "Body", "Pose", "SurfaceRep", "BoxRep", "BodyKinematics", "RepMoments", "SurfaceTopology"):
        from . import scene
        return getattr(scene, name)
    if name in ("AnalyticBoundary", "BoundaryProvider", "FusedWall", "WallAggregate", "WallOutput", "FusedGroup"):
        from . import provider
        return getattr(provider, name)
    if name in ("fixed_adjacency", "fixed_topology", "FixedTopology", "indicator_device"):
        from . import fixedadj
        return getattr(fixedadj, name)
    if name in ("BoundaryMoments", "aggregate_moments"):
        from . import autograd
        return getattr(autograd, name)
    raise AttributeError(name)
