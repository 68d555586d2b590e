"""Replica harness on CPU ranks (gloo, world size 2): work split and
max-over-ranks timing used by bench.py --gpus N."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from sigpyproc3_b200 import multi

    lo, hi = multi.shard_range(10, rank, world)
    t = multi.max_over_ranks(0.5 + rank)
    tot = multi.sum_over_ranks(float(hi - lo))
    q.put((rank, lo, hi, t, tot))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_split_and_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1:3] == (0, 5) and res[1][1:3] == (5, 10)
    assert all(r[3] == pytest.approx(1.5) for r in res)
    assert all(r[4] == pytest.approx(10.0) for r in res)


def test_shard_range_covers():
    from sigpyproc3_b200 import multi

    for n in (0, 1, 7, 64):
        for w in (1, 2, 3, 8):
            parts = [multi.shard_range(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(w - 1))
