"""Several ranks on one grid (CPU, gloo, world size 2): the block ranges of
kumo_b200.shard partition the grid into whole 128-point blocks, the host
gather rebuilds the one-rank result exactly, and timings reduce to the
slowest rank's.  The same helpers serve the GPU ranks (NCCL) of bench.py.

On CPU ranks the field function of a rank is the oracle's evaluation of a
real molecule (acrolein: rho, grad rho, lap rho, tau, ELF), which, like the
device evaluator, works block by block: the gathered grid must equal the
one-rank evaluation bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import GOLDEN

from kumo_b200 import shard


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake_fields(pts: np.ndarray):
    x, y, z = pts.T
    return [np.stack([x + 2 * y + 3 * z]), np.stack([x * y, y * z, z * x])]


FIELDS = [(0, 0, 0, 0), (1, 0, 0, 0), (3, 0, 0, 0), (4, 0, 0, 0), (6, 0, 0, 0)]  # rho, grad, lap, tau, ELF


def _acrolein_fields():
    import oracle as O
    o = O.OracleMolecule.from_fchk(os.path.join(GOLDEN, "acrolein.fchk.gz"))

    def fields(pts: np.ndarray):
        return o.evaluate(FIELDS, points=pts)[0]

    xyz = o.atom_xyz.reshape(-1, 3)
    origin = xyz.min(0) - 2.0
    return fields, origin, np.eye(3) * 0.45, tuple(int(c) for c in np.ceil((xyz.max(0) - xyz.min(0) + 4.0) / 0.45))


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
        # The real evaluation (oracle on CPU ranks), one grid over the ranks.
        fields, origin, steps, counts = _acrolein_fields()
        full = shard.evaluate_grid_sharded(fields, origin, steps, counts, dist, rank, world)
        if rank == 0:
            ref = fields(shard.grid_points(origin, steps, counts, 0, int(np.prod(counts))))
            if int(np.prod(counts)) < 128 * world * 4:
                problems.append("grid too small to spread blocks over the ranks")
            for a, r in zip(full, ref):
                if not np.array_equal(a, r):
                    problems.append("gather of the evaluated fields")
        else:
            if full != []:
                problems.append("non-destination rank received the gathered grid")
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


def test_slab_ranges_partition_the_planes():
    for nx, world in [(128, 1), (128, 2), (128, 8), (7, 3), (3, 4), (192, 8)]:
        got = [shard.slab_range((nx, 5, 6), r, world) for r in range(world)]
        assert got[0][0] == 0 and got[-1][1] == nx
        for (a0, a1), (b0, b1) in zip(got, got[1:]):
            assert a1 == b0 and a1 >= a0
        sizes = [b - a for a, b in got]
        assert max(sizes) - min(sizes) <= 1
    o, s, c = shard.slab_grid([1.0, 2.0, 3.0], np.eye(3) * 0.5, (10, 4, 4), 3, 7)
    assert c == (4, 4, 4) and np.allclose(o, [2.5, 2.0, 3.0])
