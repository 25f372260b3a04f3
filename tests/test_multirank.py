"""The multi-rank host logic of bench.py on CPU: two ranks with the gloo
backend (the GPU run uses NCCL; the path is replicas only, so the only
cross-rank steps are the timing reduction and the aggregate)."""
import argparse
import multiprocessing
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    import bench

    r, w, lr = bench.dist_env()
    t = bench.max_over_ranks(1.5 + rank)           # per-rank ms; the slowest wins
    agg = bench.replica_gbs(1e9, t * 1e-3, w)       # 1 GB per step per replica
    ref_rc = None
    if rank != 0:                                   # the reference arm: rank 0 only
        ref_rc = bench.run_reference(argparse.Namespace(steps=1, warmup=1))
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, (r, w, lr), t, agg, ref_rc))


def test_two_ranks_gloo():
    ctx = multiprocessing.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            pytest.fail("a rank did not finish")
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in procs)
    for rank, env, t, agg, ref_rc in out:
        assert env == (rank, 2, rank)
        assert t == 2.5
        assert agg == pytest.approx(1e9 / 2.5e-3 / 1e9 * 2)
    assert out[1][4] == 0


def test_single_rank_without_group():
    import bench

    assert bench.max_over_ranks(3.25) == 3.25
    assert bench.replica_gbs(2e9, 0.5, 1) == pytest.approx(4.0)
