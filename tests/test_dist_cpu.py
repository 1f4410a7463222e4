"""Multi-rank host logic of bench.py on the CPU: two gloo ranks on 127.0.0.1.

Covers what `bench.py --gpus N` does around the GPU work: rank/world parsing, barriers, the
maximum of the per-rank device times (the job ends with the slowest rank), the per-rank values
the batch line records (each rank's DOFs and work), the whole-job rate
(units of all ranks over that time) and the sharding of the batch configuration (each rank
its own seeded problems, disjoint across ranks, rank 0's equal to the single-GPU batch).
"""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=timedelta(seconds=60))
    try:
        import bench
        from edge_to_b200 import batch
        env = bench.dist_env()
        t = bench._max_over_ranks(10.0 + 5.0 * rank, ws)   # rank 1 is the slower one
        rate = bench.whole_job_rate(3, ws, t)
        per_rank = bench._gather_over_ranks(100.0 + rank, ws)
        bench._barrier(ws)
        idx = [s["index"] for s in batch.shard_specs(4, rank, seed=0)]
        everyone = [None] * ws
        dist.all_gather_object(everyone, idx)
        q.put((rank, env, t, rate, everyone, per_rank))
    except BaseException as e:  # noqa: BLE001 - reported to the parent
        q.put((rank, repr(e), None, None, None, None))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_timing_and_batch_shards():
    import torch.multiprocessing as mp
    from edge_to_b200 import batch
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    try:
        for _ in range(2):
            r = q.get(timeout=180)
            out[r[0]] = r
    finally:
        for p in procs:
            p.join(timeout=60)
            if p.is_alive():
                p.kill()
    assert set(out) == {0, 1}
    for rank, (r, env, t, rate, everyone, per_rank) in out.items():
        assert env == (2, rank, rank), env
        assert t == 15.0
        assert per_rank == [100.0, 101.0]  # every rank's value, rank order (the batch line's per-rank work)
        assert rate == pytest.approx(2 * 3 / 15e-3)
        assert everyone == [[0, 1, 2, 3], [4, 5, 6, 7]]
    single = [s["index"] for s in [batch.random_spec(i, 0) for i in range(4)]]
    assert out[0][4][0] == single
    assert all(p.exitcode == 0 for p in procs)
