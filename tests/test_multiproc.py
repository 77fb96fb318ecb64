"""Multi-rank placement (nebula_b200/shard.py) on the CPU.

The batched form spreads scenes over ranks by a particle-balanced partition
that every rank computes alone; the measurement only needs a barrier and
the maximum of the per-rank times.  Two gloo ranks on 127.0.0.1 check that
the ranks agree on a disjoint cover of all scenes and on the reductions.
"""
import datetime
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from nebula_b200 import scenes as S
from nebula_b200 import shard


def test_partition_covers_and_balances():
    sizes = S.batch_mix_sizes()
    for world in (1, 2, 3, 4, 8):
        parts = shard.partition_scenes(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # greedy LPT: no rank exceeds the mean by more than the largest scene
        assert max(loads) <= sum(sizes) / world + max(sizes)
        assert parts == shard.partition_scenes(sizes, world)  # deterministic
    assert shard.partition_scenes([5, 5, 5], 5)[3:] == [[], []]
    with pytest.raises(ValueError):
        shard.partition_scenes(sizes, 0)


def test_reductions_without_a_process_group():
    assert shard.max_over_ranks(2.5) == 2.5 and shard.sum_over_ranks(2.5) == 2.5


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, w, _ = shard.rank_info()
        sizes = S.batch_mix_sizes()
        mine = shard.partition_scenes(sizes, w)[r]
        everyone = [None] * w
        dist.all_gather_object(everyone, mine)
        dist.barrier()
        t_max = shard.max_over_ranks(10.0 * (r + 1), dist)
        n_sum = shard.sum_over_ranks(sum(sizes[i] for i in mine), dist)
        torch.save({"rank": r, "everyone": everyone, "t_max": t_max, "n_sum": n_sum, "mine": mine}, os.path.join(out_dir, "r%d.pt" % r))
    finally:
        dist.destroy_process_group()


def test_two_ranks_gloo(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    res = [torch.load(tmp_path / ("r%d.pt" % r)) for r in range(world)]
    sizes = S.batch_mix_sizes()
    for r in res:
        assert r["everyone"] == res[0]["everyone"]          # every rank computed the same partition
        assert r["mine"] == r["everyone"][r["rank"]]
        assert r["t_max"] == 10.0 * world
        assert r["n_sum"] == sum(sizes)
    cover = sorted(i for p in res[0]["everyone"] for i in p)
    assert cover == list(range(len(sizes)))


def _rank_leaves(rank, world, port, out_dir):
    """Rank 1 leaves between steps (after the first collective, none in
    flight); rank 0's next collective must end with an error within the
    process group's short timeout instead of hanging."""
    import time
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    shard.max_over_ranks(1.0, dist)
    if rank == 1:
        os._exit(0)  # leaves without destroying the group
    t0 = time.time()
    failed = False
    try:
        shard.max_over_ranks(2.0, dist)
    except Exception:
        failed = True
    torch.save({"failed": failed, "waited": time.time() - t0}, os.path.join(out_dir, "leave.pt"))
    os._exit(0)


def test_a_rank_that_leaves_is_detected(tmp_path):
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_leaves, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        if p.is_alive():
            p.kill()
    r = torch.load(tmp_path / "leave.pt")
    assert r["failed"] and r["waited"] < 60
