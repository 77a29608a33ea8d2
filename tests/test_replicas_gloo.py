"""The multi-GPU path on CPU: two gloo ranks, each advancing its own replica (the oracle's FP32
substep stands in for the device substep), lined up by barriers, with the job time taken as the
slowest rank's and the whole-job throughput computed from it.  No data-path collective is used:
the replicas of one seed agree bit for bit without exchanging anything."""
import os

import numpy as np
import pytest


def _worker(rank, world_size, port, out_dir):
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world_size), "LOCAL_RANK": str(rank)})
    import torch

    from oracle import restated
    from zsmpm_b200 import replicas, scenes
    ws, r, _ = replicas.init("gloo", timeout_s=60)
    assert (ws, r) == (world_size, rank)
    spec = scenes.small_scene(model=1, n_side=0.04)
    p = scenes.generate(spec)
    replicas.barrier()
    res = restated.run(spec, p, 3)
    # a rank-dependent "device time": the job time is the slowest rank's
    ms = 10.0 + 5.0 * rank
    job_ms = replicas.max_over_ranks(ms)
    value = replicas.throughput(p.n, 3, job_ms, ws)
    replicas.barrier()
    # what the ranks computed, gathered only to check them here
    xs = [torch.zeros_like(torch.from_numpy(res.x)) for _ in range(ws)]
    import torch.distributed as dist
    dist.all_gather(xs, torch.from_numpy(res.x))
    np.savez(os.path.join(out_dir, f"rank{rank}.npz"), job_ms=job_ms, value=value, n=p.n,
             same=all(torch.equal(xs[0], t) for t in xs), shard=list(replicas.shard(256, rank, ws)))
    replicas.finish()


def test_two_gloo_replicas(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"rank{k}.npz") for k in range(2))
    assert float(r0["job_ms"]) == float(r1["job_ms"]) == 15.0
    n = int(r0["n"])
    assert float(r0["value"]) == pytest.approx(n * 3 * 2 / 15e-3)
    assert bool(r0["same"]) and bool(r1["same"])
    s0, s1 = list(r0["shard"]), list(r1["shard"])
    assert s0 == list(range(0, 128)) and s1 == list(range(128, 256))


def test_shard_covers_items_once():
    from zsmpm_b200 import replicas
    for n in (0, 1, 7, 256, 1001):
        for ws in (1, 2, 3, 8):
            got = [i for r in range(ws) for i in replicas.shard(n, r, ws)]
            assert got == list(range(n))
