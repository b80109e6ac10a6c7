"""Scene sharding of the batched workload over ranks (bench.py --workload
batched_64 under torchrun): the longest-processing-time-first split, and a
world_size-2 gloo run of the host-side bookkeeping (each rank takes its
shard, the particle totals and the max-over-ranks time are combined with
the same collectives the bench uses).  CPU only."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_lpt_shards_cover_and_balance():
    from bench import lpt_shards
    from graphics_b200.scene import config_batched_dfsph
    sizes = [s.n_fluid for s in config_batched_dfsph(64, seed=0)]
    for world in (1, 2, 4, 8):
        parts = lpt_shards(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(64))
        loads = [sum(sizes[i] for i in p) for p in parts]
        # LPT is within 4/3 of the optimum; the optimum is >= the mean
        assert max(loads) <= 4 / 3 * sum(sizes) / world + max(sizes)


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from bench import lpt_shards
    sizes = [10, 50, 20, 40, 30, 5]
    mine = lpt_shards(sizes, world)[rank]
    n = torch.tensor([float(sum(sizes[i] for i in mine))])
    dist.all_reduce(n)
    t = torch.tensor([1.0 + rank])  # this rank's elapsed time
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out[rank] = (sorted(mine), n.item(), t.item())
    dist.destroy_process_group()


def test_sharded_totals_gloo_world2():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = 29651
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert sorted(res[0][0] + res[1][0]) == list(range(6))
    assert res[0][1] == res[1][1] == 155.0
    assert res[0][2] == res[1][2] == 2.0
