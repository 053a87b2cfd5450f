"""Differentiable boundary moments: a torch.autograd.Function whose backward is the hand-written adjoint kernel.

`aggregate_moments(body, rep, pos, sup, kernel, support)` returns world-frame lam [N], m1 [N, 2], m2 [N, 2, 2]
(and G, Cov) of one (body, surface); gradients flow to the particle positions `pos` and to `rep.vertices`
(body frame).  The backward recomputes the chord integrals of every neighbour pair (no per-pair storage):
d m_alpha / dx = -sum_e n_e int y^alpha W ds and the Reynolds edge adjoint
d m_alpha / d p_e = n_e int (1 - tau) y^alpha W ds, d / d q_e = n_e int tau y^alpha W ds
(src/warpSPHBoundaries/edge/np2d.py:554-565, 626-652; the reference wraps the same formulas in
warp2d.TorchMoment, src/warpSPHBoundaries/edge/warp2d.py:482-500).  The indicator term is piecewise constant and has
no derivative.  G and Cov are returned for convenience but are not differentiated: a non-zero upstream gradient on
them raises NotImplementedError.
"""
import torch

from . import _lib
from ._lib import check, lib, ptr
from .kernels import KERNEL_IDS
from .scene import _stream
from .shim import kernelName

F64 = torch.float64
_PREC = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED, "fp32": _lib.PREC_FP32}


class BoundaryMoments(torch.autograd.Function):
    @staticmethod
    def forward(ctx, pos, verts, sup, body, rep, kid, support, precision):
        dev = pos.device
        N = len(pos)
        posc = pos.detach().to(F64).contiguous()
        supc = sup.detach().to(F64).contiguous()
        ns = rep.native(support, dev)
        ws, need = ns.workspace(N)
        lam = torch.zeros(N, dtype=F64, device=dev)
        G = torch.zeros((N, 2), dtype=F64, device=dev)
        Cov = torch.zeros((N, 2, 2), dtype=F64, device=dev)
        m1 = torch.zeros((N, 2), dtype=F64, device=dev)
        m2 = torch.zeros((N, 2, 2), dtype=F64, device=dev)
        pose = body.pose_tensor(dev)
        obb = (_lib.ctypes.c_double * 4)(*body.obb())
        check(lib.wsb_aggregate(ns.handle, kid, _PREC[precision], ptr(posc), ptr(supc), None, N, ptr(pose), obb,
                                int(body.unbounded()), _lib.OUT_ALL, ptr(lam), ptr(G), ptr(Cov), ptr(m1), ptr(m2),
                                ptr(ws), need, None, _stream()), "wsb_aggregate")
        ctx.save_for_backward(posc, supc)
        ctx.body, ctx.rep, ctx.kid, ctx.support, ctx.nverts = body, rep, kid, support, len(verts)
        ctx.verts_device, ctx.verts_dtype = verts.device, verts.dtype
        return lam, m1, m2, G, Cov

    @staticmethod
    def backward(ctx, g_lam, g_m1, g_m2, g_G, g_Cov):
        for g, name in ((g_G, "G"), (g_Cov, "Cov")):
            if g is not None and bool((g != 0).any()):
                raise NotImplementedError(f"BoundaryMoments: the derivative of {name} (a kernel-Hessian integral) is "
                                          "not built; differentiate lam, m1 and m2")
        posc, supc = ctx.saved_tensors
        dev = posc.device
        N = len(posc)
        ns = ctx.rep.native(ctx.support, dev)
        ws, need = ns.workspace(N)
        d_pos = torch.zeros((N, 2), dtype=F64, device=dev)
        d_verts = torch.zeros((ctx.nverts, 2), dtype=F64, device=dev)
        gl = None if g_lam is None else g_lam.to(F64).contiguous()
        g1 = None if g_m1 is None else g_m1.to(F64).contiguous()
        g2 = None if g_m2 is None else g_m2.to(F64).contiguous()
        pose = ctx.body.pose_tensor(dev)
        obb = (_lib.ctypes.c_double * 4)(*ctx.body.obb())
        check(lib.wsb_aggregate_backward(ns.handle, ctx.kid, ptr(posc), ptr(supc), None, N, ptr(pose), obb,
                                         int(ctx.body.unbounded()), ptr(gl), ptr(g1), ptr(g2), ptr(d_pos),
                                         ptr(d_verts), ptr(ws), need, _stream()), "wsb_aggregate_backward")
        return (d_pos.to(posc.dtype), d_verts.to(ctx.verts_device, ctx.verts_dtype), None, None, None, None, None,
                None)


def aggregate_moments(body, rep, pos, sup, kernel, support, precision="fp64"):
    """{lam, m1, m2, G, Cov} of one (body, surface) at world positions `pos` [N, 2] with supports `sup` [N];
    differentiable in `pos` and `rep.vertices` through lam, m1 and m2."""
    kid = KERNEL_IDS[kernelName(kernel)]
    lam, m1, m2, G, Cov = BoundaryMoments.apply(pos, rep.vertices, sup, body, rep, kid, float(support), precision)
    return {"lam": lam, "m1": m1, "m2": m2, "G": G, "Cov": Cov}
