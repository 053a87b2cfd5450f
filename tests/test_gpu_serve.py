"""The continuous-batching request loop: every request's result is bit-identical alone and in the mix (batched with
other requests, several streams, CUDA-graph buckets), and equal to the provider's own aggregate."""
import numpy as np
import pytest
import torch

from warpsphboundaries_b200 import workloads
from warpsphboundaries_b200.provider import FusedGroup, FusedWall
from warpsphboundaries_b200.scene import Body, Scene, SurfaceRep
from warpsphboundaries_b200.serve import OUT_KEYS, BoundaryServer
from warpsphboundaries_b200.shim import ParticleState

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _scenes():
    out = {}
    for k in range(3):
        loops = workloads.stars(3, (32, 200), seed=40 + k, box=1.0)
        out[f"s{k}"] = Scene([Body(center=(0.01 * k, 0.0), angle=0.2 * k, reps=[SurfaceRep.loops(loops)])], DEV)
    return out


def _requests(rng, n):
    reqs = []
    for i in range(n):
        rows = int(np.exp(rng.uniform(np.log(500), np.log(20000))))
        reqs.append((f"s{rng.integers(0, 3)}", ["w2", "w4", "w6", "cubic"][rng.integers(0, 4)], rows,
                     bool(rng.uniform() < 0.25), int(rng.integers(0, 1 << 30))))
    return reqs


def _positions(rows, seed):
    g = torch.Generator(device=DEV)
    g.manual_seed(seed)
    return torch.rand((rows, 2), dtype=torch.float64, device=DEV, generator=g) * 1.2 - 0.1


def test_alone_equals_mixed_bitwise():
    scenes = _scenes()
    h = 0.02
    reqs = _requests(np.random.default_rng(0), 40)
    mixed = BoundaryServer(DEV, streams=3, max_batch_rows=60000, use_graphs=True, graph_max_rows=1 << 14,
                           graph_after_uses=1)
    for sid, sc in scenes.items():
        mixed.register(sid, sc, h)
    ids = [mixed.submit(sid, _positions(rows, seed), h, k, grad=g) for sid, k, rows, g, seed in reqs]
    mixed.run()
    torch.cuda.synchronize()
    # at least some batches held several requests
    st = mixed.stats()
    assert st["requests"] == len(reqs)
    for (sid, k, rows, g, seed), rid in zip(reqs, ids):
        alone = BoundaryServer(DEV, streams=1, max_batch_rows=rows, use_graphs=False)
        alone.register(sid, scenes[sid], h)
        aid = alone.submit(sid, _positions(rows, seed), h, k, grad=g)
        alone.run()
        torch.cuda.synchronize()
        a, m = alone.result(aid), mixed.result(rid)
        for key in OUT_KEYS:
            assert torch.equal(a[key], m[key]), (sid, k, rows, key)
        if g:
            assert torch.equal(a["d_pos"], m["d_pos"])


def test_server_result_equals_provider():
    scenes = _scenes()
    h = 0.02
    srv = BoundaryServer(DEV, streams=2, graph_max_rows=1 << 12)
    srv.register("s1", scenes["s1"], h)
    pos = _positions(3000, 5)
    rid = srv.submit("s1", pos, h, "w4")
    srv.run()
    torch.cuda.synchronize()
    fw = FusedWall(scenes["s1"], ParticleState(pos, torch.full((3000,), h, dtype=torch.float64, device=DEV)), h,
                   (FusedGroup("w4"),))
    for key in OUT_KEYS:
        assert torch.equal(srv.result(rid)[key], fw.res[0][key])
