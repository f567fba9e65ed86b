"""Multi-rank host logic on CPU: world_size-2 gloo process groups (127.0.0.1)."""
import os
import socket

import pytest

from su3_ma_gauge_gpu_b200.distributed import best_copy, reduce_timing, shard, shard_weighted


def test_shard_covers_every_item_once():
    for n in (0, 1, 5, 64, 65):
        for world in (1, 2, 3, 8):
            got = sorted(i for r in range(world) for i in shard(n, r, world))
            assert got == list(range(n))
            sizes = [len(shard(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1


def test_shard_weighted_balances():
    w = [24 * 12**4] * 24 + [24 * 16**4] * 24 + [16 * 20**3 * 40] * 16  # the uneven Gribov batch
    owners = [shard_weighted(w, r, 4) for r in range(4)]
    assert sorted(i for o in owners for i in o) == list(range(len(w)))
    loads = [sum(w[i] for i in o) for o in owners]
    assert max(loads) / min(loads) < 1.1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = shard(5, rank, world)
        t = reduce_timing(ms=10.0 + rank, site_updates=1e6 * len(mine))
        best = best_copy(gff=0.9 + 0.01 * rank, copy_id=mine[0])
        q.put((rank, t.ms, t.site_updates, best))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, updates, best in res:
        assert ms == pytest.approx(11.0)          # max over ranks
        assert updates == pytest.approx(5e6)      # every copy counted once
        assert best == (pytest.approx(0.91), 3)   # rank 1 owns copies 3, 4
