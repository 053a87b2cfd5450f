"""The N > 1 host path on CPU: two gloo ranks shard the particles over the replicated geometry, reduce the time by
max, and compute shard results independently (no data-path collective: a rank's rows equal a one-process run)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from oracle import edge2d as O
    from warpsphboundaries_b200 import shard, workloads
    loops, X0, h = workloads.c2(n_particles=2048, seed=0)
    X = shard.rank_particles(len(X0), rank, X0)
    t = shard.max_over_ranks(0.5 + rank)                    # the slowest rank's time
    # a few rows of this shard through the oracle (the checker of the GPU path) with nothing from other ranks
    V, E = workloads.edges_of(loops)
    sel = np.arange(0, len(X), 256)
    ch = O.local_twelve(V, E, 0, X[sel], np.full(len(sel), h), "w4", h, np.ones(len(sel), bool))
    dist.barrier()
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), X=X, t=t, ch=ch,
             geo=np.concatenate([np.asarray(l).ravel() for l in loops]))
    dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    world, port = 2, _free_port()
    mp.start_processes(_worker, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn", join=True)
    r0, r1 = (np.load(tmp_path / f"rank{r}.npz") for r in range(world))
    assert np.array_equal(r0["geo"], r1["geo"])              # geometry replicated
    assert not np.allclose(r0["X"], r1["X"])                  # particles sharded
    assert float(r0["t"]) == float(r1["t"]) == 1.5            # max over ranks on every rank
    from warpsphboundaries_b200 import shard
    assert shard.job_rate(100.0, 2.0, world) == 100.0
    # rank 1's rows equal a one-process evaluation of the same particles
    from oracle import edge2d as O
    from warpsphboundaries_b200 import workloads
    loops, _, h = workloads.c2(n_particles=2048, seed=0)
    V, E = workloads.edges_of(loops)
    sel = np.arange(0, len(r1["X"]), 256)
    alone = O.local_twelve(V, E, 0, r1["X"][sel], np.full(len(sel), h), "w4", h, np.ones(len(sel), bool))
    assert np.array_equal(alone, r1["ch"])
