"""Host logic of the ensemble and its multi-rank path (gloo, 2 ranks, CPU)."""
import multiprocessing as mp
import os

import pytest

from smaiso_quasi_b200 import ensemble as en


def test_members_are_seeded_and_in_range():
    a, b = en.make_members(48, seed=5), en.make_members(48, seed=5)
    assert a == b
    assert all(0.01 <= m.eps_h <= 0.1 and 1 <= m.m <= 8 and m.grid in en.GRIDS for m in a)


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_partition_covers_once_and_balances_cells(world):
    ms = en.make_members(48, seed=1)
    parts = en.partition(ms, world)
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(48))
    loads = [sum(ms[i].cells for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(m.cells for m in ms)


def _rank(rank, world, port, q):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = en.make_members(12, seed=3)
    mine = en.partition(ms, world)[rank]
    # stand-in for run_members (no device here): a result keyed by member
    local = {"indices": mine, "growth": [float(i) * 0.5 for i in mine], "wall_s": 1.0 + rank,
             "instance_steps_per_s": 10.0, "cell_updates_per_s": 100.0}
    merged = en.merge(en.gather(local, dist), len(ms))
    q.put((rank, merged))
    dist.destroy_process_group()


def test_two_rank_gather_merges_all_members():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    got = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r in (0, 1):
        assert got[r]["growth"] == [i * 0.5 for i in range(12)]
        assert got[r]["max_wall_s"] == 2.0
        assert got[r]["instance_steps_per_s"] == 20.0
