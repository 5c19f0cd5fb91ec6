"""Event sharding over ranks (the multi-GPU split of event-by-event batches).

The split is host logic: it runs here on CPU, with two gloo ranks standing in
for two GPUs. Each rank takes its share of the events and reports per-event
results; the gather must see every event exactly once, and the shares must be
balanced in cells.
"""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fivo2d.events import EVENT_SIZES, event_grids, shard_events


def test_event_grids_follow_the_batch_definition():
    gs = event_grids(64, seed=7)
    assert len(gs) == 64
    for g in gs:
        assert g.Nx == g.Ny and g.Nx in EVENT_SIZES
        assert abs(g.dx - 30.0 / 384.0) < 1e-15 and abs(g.dy - g.dx) < 1e-15
    assert [g.Nx for g in gs] == [g.Nx for g in event_grids(64, seed=7)]      # seeded
    assert len({g.Nx for g in gs}) > 3                                         # uneven


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shards_cover_once_and_balance(world):
    cells = [g.Nx * g.Ny for g in event_grids(50, seed=11)]
    parts = shard_events(cells, world)
    flat = sorted(k for p in parts for k in p)
    assert flat == list(range(len(cells)))
    loads = [sum(cells[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(cells)
    for r in range(world):
        assert shard_events(cells, world, r) == parts[r]


def test_shard_rejects_empty_world():
    with pytest.raises(ValueError):
        shard_events([1, 2], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        grids = event_grids(24, seed=3)
        cells = [g.Nx * g.Ny for g in grids]
        mine = shard_events(cells, world, rank)
        # stand-in for a per-event result: (event, cells advanced) from this rank only
        out = [None] * world
        dist.all_gather_object(out, [(k, cells[k]) for k in mine])
        if rank == 0:
            seen = sorted(k for part in out for k, _ in part)
            total = sum(c for part in out for _, c in part)
            loads = [sum(c for _, c in part) for part in out]
            q.put((seen == list(range(len(cells))), total == sum(cells), max(loads) - min(loads) <= max(cells)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_gather_sees_every_event_once():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) == (True, True, True)
