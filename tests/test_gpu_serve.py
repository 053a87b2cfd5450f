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


def test_closed_surfaces_in_the_mix():
    """3-D closed-surface scenes served next to 2-D ones: each request's channels equal a direct wsb_mesh_channels
    call on its own positions, bit for bit, however the requests were batched."""
    from warpsphboundaries_b200.mesh3d import ClosedMesh
    h = 0.05
    meshes = {f"m{k}": workloads.icosphere(2, 0.5 + 0.1 * k, 0.05, seed=k) for k in range(2)}
    srv = BoundaryServer(DEV, streams=3, max_batch_rows=40000)
    for sid, (V, Fc) in meshes.items():
        srv.register_mesh(sid, V, Fc, h)
    srv.register("s0", _scenes()["s0"], 0.02)
    rng = np.random.default_rng(3)
    reqs = []
    for i in range(24):
        if i % 3 == 2:
            reqs.append(("s0", "w4", int(rng.integers(500, 5000)), int(rng.integers(0, 1 << 30))))
        else:
            reqs.append((f"m{rng.integers(0, 2)}", ["w2", "w4", "w6", "cubic"][rng.integers(0, 4)],
                         int(rng.integers(300, 8000)), int(rng.integers(0, 1 << 30))))

    def pos3(rows, seed):
        g = torch.Generator(device=DEV)
        g.manual_seed(seed)
        return torch.rand((rows, 3), dtype=torch.float64, device=DEV, generator=g) * 1.6 - 0.8

    ids = [srv.submit(sid, pos3(rows, seed) if sid.startswith("m") else _positions(rows, seed),
                      h if sid.startswith("m") else 0.02, k) for sid, k, rows, seed in reqs]
    srv.run()
    torch.cuda.synchronize()
    direct = {sid: ClosedMesh(V, Fc, h, DEV) for sid, (V, Fc) in meshes.items()}
    for (sid, k, rows, seed), rid in zip(reqs, ids):
        if not sid.startswith("m"):
            continue
        p = pos3(rows, seed)
        ref = direct[sid].channels(p, torch.full((rows,), h, dtype=torch.float64, device=DEV), k)
        torch.cuda.synchronize()
        assert torch.equal(srv.result(rid)["channels"], ref), (sid, k, rows)
    with pytest.raises(NotImplementedError):
        srv.submit("m0", pos3(10, 1), h, "w4", grad=True)


def test_lowered_bodies_are_served():
    """a box, a cavity disk and a sampled distance are served as the polygons the provider integrates (bit-identical
    to FusedWall); a disk set is refused."""
    from warpsphboundaries_b200.implicit import DiskBody
    from warpsphboundaries_b200.scene import BoxRep, DiskArrayRep, ImplicitRep, SdfRep
    h = 0.02
    sdf = SdfRep.fromFunction(lambda p: (p - torch.tensor([0.5, 0.5], dtype=torch.float64)).norm(dim=1) - 0.3,
                              (0.0, 0.0), (1.0, 1.0), h / 8)
    scene = Scene([Body(reps=[BoxRep((0.1, 0.1), (0.3, 0.4))]), Body(reps=[sdf]),
                   Body(center=(0.5, 0.5), reps=[ImplicitRep(DiskBody((0.0, 0.0), 0.7, solid="outside"))])], DEV)
    srv = BoundaryServer(DEV, streams=2, graph_max_rows=1 << 12)
    srv.register("low", scene, h)
    pos = _positions(4000, 9)
    rid = srv.submit("low", pos, h, "w2")
    srv.run()
    torch.cuda.synchronize()
    fw = FusedWall(scene, ParticleState(pos, torch.full((4000,), h, dtype=torch.float64, device=DEV)), h,
                   (FusedGroup("w2"),))
    for key in OUT_KEYS:
        assert torch.equal(srv.result(rid)[key], fw.res[0][key]), key
    with pytest.raises(NotImplementedError):
        srv.register("disks", Scene([Body(reps=[DiskArrayRep([[0.5, 0.5]], [0.1])])], DEV), h)


def test_sphere_rows_in_the_mix_and_per_class_stats():
    """sphere-row requests (query, sphere) of two sphere scenes with different supports, batched together and with
    2-D requests: each equals RadialEvaluator on its rows bit for bit; the statistics report p50 / p99 per request
    class."""
    from warpsphboundaries_b200.radial import RadialEvaluator
    srv = BoundaryServer(DEV, streams=2, max_batch_rows=30000)
    srv.register_spheres("sph", 0.03)
    srv.register_spheres("sph2", 0.05)          # another sphere scene: its rows share the launches of "sph"
    for sid, sc in _scenes().items():
        srv.register(sid, sc, 0.03)
    rng = np.random.default_rng(9)
    ids, want = [], []
    for i in range(8):
        n = int(rng.integers(500, 9000))
        R = np.exp(rng.uniform(np.log(0.006), np.log(1.5), n))
        d = np.maximum(rng.uniform(-0.036, 0.036, n), -R)
        nv = rng.normal(size=(n, 3))
        nv /= np.linalg.norm(nv, axis=1, keepdims=True)
        k = ["w2", "w4", "w6"][i % 3]
        rows = torch.tensor(np.concatenate([d[:, None], nv, R[:, None]], 1), dtype=torch.float64, device=DEV)
        sid, h = ("sph", 0.03) if i % 2 == 0 else ("sph2", 0.05)
        ids.append(srv.submit(sid, rows, h, k))
        want.append(RadialEvaluator("sphere", kernel=k, device=DEV).evaluate(d, nv, h, radii=R))
        ids.append(srv.submit("s0", _positions(1000 + i, i), 0.03, "w4", grad=(i % 2 == 0)))
        want.append(None)
    srv.run()
    torch.cuda.synchronize()
    for rid, ref in zip(ids, want):
        if ref is not None:
            assert np.array_equal(srv.result(rid)["channels"].cpu().numpy(), ref)
    st = srv.stats()
    assert set(st["classes"]) == {"3d_spheres", "2d", "2d_grad"}
    assert st["classes"]["3d_spheres"]["requests"] == 8
    assert all(v["p50_ms"] <= v["p99_ms"] for v in st["classes"].values())


def test_light_lane_takes_short_requests():
    """a short 2-D request submitted after a closed-surface request of several milliseconds runs on the light lane
    (a high-priority stream) at once instead of waiting for a standard slot; both results equal a server without
    light lanes, bit for bit."""
    h = 0.05
    V, Fc = workloads.icosphere(3, 0.6, 0.05, seed=4)

    def pos3(rows, seed):
        g = torch.Generator(device=DEV)
        g.manual_seed(seed)
        return torch.rand((rows, 3), dtype=torch.float64, device=DEV, generator=g) * 1.6 - 0.8

    out = []
    for light in (1, 0):
        srv = BoundaryServer(DEV, streams=1, light_streams=light)
        srv.register_mesh("m", V, Fc, h)
        srv.register("s0", _scenes()["s0"], 0.02)
        heavy = srv.submit("m", pos3(400000, 1), h, "w4")          # estimated 2.6 ms: a standard slot
        short = srv.submit("s0", _positions(3000, 2), 0.02, "w2")   # estimated 0.02 ms: light
        srv.poll()
        on = {s.light: [r.rid for r in s.busy.reqs] for s in srv.slots if s.busy is not None}
        if light:
            assert on == {False: [heavy], True: [short]}
        else:
            assert on == {False: [heavy]}                           # the short request waits for the slot
        srv.run()
        torch.cuda.synchronize()
        out.append((srv.result(heavy)["channels"].clone(), {k: v.clone() for k, v in srv.result(short).items()}))
    assert torch.equal(out[0][0], out[1][0])
    for k in OUT_KEYS:
        assert torch.equal(out[0][1][k], out[1][1][k]), k

