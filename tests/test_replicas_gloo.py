"""Multi-process replica plumbing on CPU (gloo, world_size 2): work split and
max-over-ranks timing used by bench.py --gpus N and the serving loop."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    import datetime

    import torch.distributed as dist

    from flups_b200.replicas import max_over_ranks, split_items, sum_over_ranks
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        start, stop = split_items(2000, rank, world)
        local_ms = 10.0 + 5.0 * rank
        q.put((rank, start, stop, max_over_ranks(local_ms), sum_over_ranks(stop - start)))
    finally:
        dist.destroy_process_group()


def test_two_rank_split_and_max():
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
    assert res[0][1:3] == (0, 1000) and res[1][1:3] == (1000, 2000)
    assert res[0][3] == res[1][3] == 15.0          # the job time is the slowest rank's
    assert res[0][4] == res[1][4] == 2000.0        # every item is owned by exactly one rank


def test_split_is_balanced():
    from flups_b200.replicas import split_items
    for n in (0, 1, 7, 2000):
        for w in (1, 2, 3, 8):
            parts = [split_items(n, r, w) for r in range(w)]
            assert parts[0][0] == 0 and parts[-1][1] == n
            assert all(parts[i][1] == parts[i + 1][0] for i in range(w - 1))
            sizes = [b - a for a, b in parts]
            assert max(sizes) - min(sizes) <= 1
