"""Multi-process replica plumbing on CPU (gloo, world size 2): sharding, barrier, max-over-ranks
timing and the aggregate rate, as bench.py uses them under torchrun."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from qtrk_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    info = replicas.init("gloo", timeout_s=60)
    start, count = replicas.shard(10001, info.rank, info.world_size)
    replicas.barrier()
    elapsed = 1.0 + info.rank          # a slower rank 1
    mx = replicas.reduce_max(elapsed)
    rate = replicas.aggregate_rate(count, info.world_size, mx)
    q.put((info.rank, start, count, mx, rate))
    replicas.finalize()


def test_shard_covers_all_units():
    for n in (0, 1, 7, 10000, 10001):
        for ws in (1, 2, 3, 8):
            parts = [replicas.shard(n, r, ws) for r in range(ws)]
            assert sum(c for _, c in parts) == n
            assert all(parts[i][0] + parts[i][1] == parts[i + 1][0] for i in range(ws - 1))
            assert max(c for _, c in parts) - min(c for _, c in parts) <= 1


def test_two_rank_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, c0, m0, rate0), (r1, s1, c1, m1, rate1) = out
    assert (s0, c0, s1, c1) == (0, 5001, 5001, 5000)
    assert m0 == m1 == 2.0                       # slowest rank's time on every rank
    assert rate0 == pytest.approx(5001 * 2 / 2.0)
