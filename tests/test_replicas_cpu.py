"""Multi-GPU form of the benchmark: independent replicas, slowest rank timed.
Exercised with two gloo ranks on the CPU."""
import os

import pytest
import torch.multiprocessing as mp


def _worker(rank, world, port, out):
    import torch.distributed as dist

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    got = bench.max_over_ranks(dist, 10.0 + rank * 5.0, device="cpu")
    seed = bench.replica_params("small_64x64x5", rank).seed
    out.put((rank, got, seed))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    assert res[0][2] != res[1][2]
