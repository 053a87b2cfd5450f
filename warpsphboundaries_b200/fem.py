"""Finite-element pair weights of P1 triangles (src/warpSPHBoundaries/edge/warpbc.py:486-510 `pair_weights`): for
every (query, element) pair the kernel integrals of the element's three barycentric functions and of their products
with the kernel gradient, evaluated by wsb_pair_weights on the GPU (no CPU path)."""
import torch

from . import _lib
from ._lib import check, lib, ptr
from .kernels import KERNEL_IDS

F64 = torch.float64


def _dev(a, device, dtype):
    t = a if isinstance(a, torch.Tensor) else torch.as_tensor(a)
    return t.to(device=device, dtype=dtype).contiguous()


def pair_weights(pair_q, pair_e, positions, supports, vertices, elements, kernel, device="cuda:0", plan=None,
                 as_torch=False):
    """(w [P, 3], G [P, 3, 2]) float64 in physical units (warpbc.py:486-510): w[k, i] = int_T W phi_i,
    G[k, i] = int_T grad_x W phi_i for the pairs (pair_q[k], pair_e[k]); numpy arrays, or device tensors with
    `as_torch`.  `plan` is accepted for the reference's signature and unused."""
    if kernel not in KERNEL_IDS:
        raise NotImplementedError(f"pair_weights: kernel {kernel!r} (exact-table kernels only)")
    dev = torch.device(device)
    if dev.type != "cuda":
        raise RuntimeError("pair_weights runs on a CUDA device (libwsb.so has no CPU path)")
    with torch.cuda.device(dev):                    # the launch and the allocations on `device`, whatever is current
        q = _dev(pair_q, dev, torch.int32).reshape(-1)
        e = _dev(pair_e, dev, torch.int32).reshape(-1)
        if len(q) != len(e):
            raise ValueError("pair_weights: pair_q and pair_e differ in length")
        pos = _dev(positions, dev, F64).reshape(-1, 2)
        sup = _dev(supports, dev, F64).reshape(-1)
        V = _dev(vertices, dev, F64).reshape(-1, 2)
        E = _dev(elements, dev, torch.int32).reshape(-1, 3)
        if len(sup) != len(pos):
            raise ValueError("pair_weights: positions and supports differ in length")
        P = len(q)
        if P:
            # index ranges checked before the launch (the kernel also refuses them: NaN outputs and a status word)
            lim = torch.stack([q.min(), q.max(), e.min(), e.max(), E.min() if len(E) else q.new_zeros(()),
                               E.max() if len(E) else q.new_zeros(())]).cpu().tolist()
            if lim[0] < 0 or lim[1] >= len(pos):
                raise ValueError(f"pair_weights: query index out of range [0, {len(pos)})")
            if lim[2] < 0 or lim[3] >= len(E):
                raise ValueError(f"pair_weights: element index out of range [0, {len(E)})")
            if lim[4] < 0 or lim[5] >= len(V):
                raise ValueError(f"pair_weights: vertex index out of range [0, {len(V)})")
        w = torch.empty((P, 3), dtype=F64, device=dev)
        G = torch.empty((P, 3, 2), dtype=F64, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        check(lib.wsb_pair_weights(KERNEL_IDS[kernel], ptr(q), ptr(e), P, ptr(pos), ptr(sup), len(pos), ptr(V), len(V),
                                   ptr(E), len(E), ptr(w), ptr(G), ptr(status),
                                   _lib.ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)),
              "wsb_pair_weights")
    return (w, G) if as_torch else (w.cpu().numpy(), G.cpu().numpy())
