"""Several ranks on one grid (CPU, gloo, world size 2): the block ranges of
kumo_b200.shard partition the grid into whole 128-point blocks, the host
gather rebuilds the one-rank result exactly, and timings reduce to the
slowest rank's.  The same helpers serve the GPU ranks (NCCL) of bench.py."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from kumo_b200 import shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_fields(pts: np.ndarray):
    x, y, z = pts.T
    return [np.stack([x + 2 * y + 3 * z]), np.stack([x * y, y * z, z * x])]


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        problems = []
        for npoints in (1, 127, 128, 129, 1000, 128 * 7 + 5, 2 ** 18):
            first, count = shard.block_range(npoints, rank, world)
            got = [None] * world
            dist.all_gather_object(got, (first, count))
            if rank == 0:
                got.sort()
                pos = 0
                for f, c in got:
                    if c == 0:
                        if f != npoints:
                            problems.append((npoints, got))
                        continue
                    if f != pos or (f % 128) or (c % 128 and f + c != npoints):
                        problems.append((npoints, got))
                    pos = f + c
                if pos != npoints:
                    problems.append((npoints, got))
        origin = np.array([-1.0, 0.5, 2.0])
        steps = np.array([[0.2, 0.01, 0.0], [0.0, 0.25, 0.02], [0.03, 0.0, 0.3]])
        counts = (7, 9, 11)
        full = shard.evaluate_grid_sharded(_fake_fields, origin, steps, counts, dist, rank, world)
        if rank == 0:
            ref = _fake_fields(shard.grid_points(origin, steps, counts, 0, int(np.prod(counts))))
            for a, r in zip(full, ref):
                if not np.array_equal(a, r):
                    problems.append("gather")
        slowest = shard.max_over_ranks(rank + 0.5, dist, world)
        if slowest != world - 0.5:
            problems.append(("max", slowest))
        q.put((rank, problems))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_gather():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, problems in results:
        assert problems == [], (rank, problems)


def test_block_range_single_rank_and_errors():
    assert shard.block_range(1000, 0, 1) == (0, 1000)
    assert shard.block_range(0, 0, 3) == (0, 0)
    # More ranks than blocks: the last ranks get nothing.
    assert [shard.block_range(200, r, 4) for r in range(4)] == [(0, 128), (128, 72), (200, 0), (200, 0)]
    with pytest.raises(ValueError):
        shard.block_range(10, 2, 2)
