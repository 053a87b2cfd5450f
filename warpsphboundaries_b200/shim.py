"""Stand-ins for the warpSPHCore types the provider interface is written against.

The reference's provider (src/warpSPHBoundaries/scene/provider.py:23) imports
`KernelFunctions`, `OperationProperties`, `OperationDirection`, `WarpOperation`
and `GradientScheme` from warpSPHCore and reads `positions`, `supports`,
`kinds` of a `ParticleState`.  warpSPHCore is a separate package; these
classes carry the same names and attributes so a caller's code reads the same.
If warpSPHCore is importable its own enums are accepted too (by member name).
"""
from dataclasses import dataclass
from enum import Enum
from typing import Optional

import torch


class KernelFunctions(Enum):
    CubicSpline = "cubic"
    QuarticSpline = "quartic"
    QuinticSpline = "quintic"
    Wendland2 = "w2"
    Wendland4 = "w4"
    Wendland6 = "w6"
    Poly6 = "poly6"
    B7 = "b7"
    B8 = "b8"
    Gaussian = "gaussian"
    HOCT4 = "hoct4"


class OperationDirection(Enum):
    FluidToFluid = 0
    FluidToBoundary = 1
    BoundaryToFluid = 2
    BoundaryToBoundary = 3
    AllToFluid = 4
    AllToBoundary = 5
    AllToAll = 6
    TrueAllToToAll = 7


class WarpOperation(Enum):
    Density = 0
    Interpolate = 1
    Gradient = 2
    Divergence = 3
    Curl = 4
    Laplacian = 5


class GradientScheme(Enum):
    Naive = 0
    Symmetric = 1
    Difference = 2


@dataclass
class OperationProperties:
    kernel: object = KernelFunctions.Wendland2
    operation: WarpOperation = WarpOperation.Density
    gradientMode: GradientScheme = GradientScheme.Naive
    operationMode: OperationDirection = OperationDirection.BoundaryToFluid


@dataclass
class ParticleState:
    """the attributes of warpSPHCore's ParticleState the boundary reads: positions [N, 2], supports [N] (kernel support
    radius h per particle), optional kinds [N] (0 fluid, 1 boundary, 2 ghost), masses, densities."""
    positions: torch.Tensor
    supports: torch.Tensor
    masses: Optional[torch.Tensor] = None
    kinds: Optional[torch.Tensor] = None
    densities: Optional[torch.Tensor] = None


# the kernels with an exact boundary integral (boundaryOps.py:30-44); B7 / B8 are not among this build's kernel tables
_EXACT = {"CubicSpline": "cubic", "QuarticSpline": "quartic", "QuinticSpline": "quintic", "Wendland2": "w2",
          "Wendland4": "w4", "Wendland6": "w6", "Poly6": "poly6"}


def kernelName(kernel) -> str:
    """registered kernel name of a KernelFunctions member (or a name); raises NotImplementedError for kernels
    without an exact piecewise-polynomial boundary integral (boundaryOps.py:35-44)."""
    from .kernels import KERNEL_IDS
    if isinstance(kernel, str):
        if kernel in KERNEL_IDS:
            return kernel
        raise KeyError(f"unknown kernel {kernel!r}; expected one of {sorted(KERNEL_IDS)}")
    name = getattr(kernel, "name", None)
    if name in _EXACT:
        return _EXACT[name]
    raise NotImplementedError(f"{kernel}: no exact boundary integral in this build (cubic, quartic, quintic, w2, w4, "
                              f"w6, poly6 are tabulated)")


def queryAllowed(queryParticles, mode, dev):
    """which queries a boundary (a Boundary-kind source) acts on for the direction `mode` (boundaryOps.py:233-247)."""
    kinds = getattr(queryParticles, "kinds", None)
    n = queryParticles.positions.shape[0]
    allq = torch.ones(n, dtype=torch.bool, device=dev)
    nm = mode.name
    if nm in ("AllToAll", "TrueAllToToAll"):
        return allq if kinds is None else (kinds.to(dev) != 2) if nm == "TrueAllToToAll" else allq
    src, tgt = nm.split("To")
    if src not in ("Boundary", "All"):
        return torch.zeros(n, dtype=torch.bool, device=dev)
    if kinds is None:
        return allq
    k = kinds.to(dev)
    return {"Fluid": k == 0, "Boundary": k == 1, "Ghost": k == 2, "All": k != 2}[tgt]
