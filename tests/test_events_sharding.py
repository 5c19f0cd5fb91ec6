"""Event sharding over ranks (the multi-GPU split of event-by-event batches).

The split is host logic: it runs here on CPU, with two gloo ranks standing in
for two GPUs. Each rank takes its share of the events and reports per-event
results; the gather must see every event exactly once, and the shares must be
balanced in cells. The results check runs real events: each rank advances its
share of small MC-Glauber events on the oracle (the CPU stand-in for its GPU)
and the gathered per-event bulk results (dQ, maxu, nsteps, the final state's
digest) must equal a single-rank run of all events.
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


# ----------------------------------------------------------------------------- sharded results

SMALL_SIZES = (24, 32, 40)


def _small_events(nevents=6):
    import fivo2d
    grids = event_grids(nevents, seed=5, sizes=SMALL_SIZES)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True, enable_diff=True,
                              eta_over_s=0.16, zeta_over_s=0.05, bulk_model="gaussian", bulk_T0=0.18,
                              bulk_width=0.024, kappa_coeff=0.5)
    return m, grids


def _run_event_on_oracle(m, g, k, nsteps=3):
    """event k (seed 1000 + k): IC, finalize_ic!, nsteps SSPRK3 steps of run_sim_2d!"""
    import _oracle as O
    from fivo2d import _abi as A
    from fivo2d import ic
    from fivo2d.events import event_record
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1000 + k)
    U, _ = O.set_cells(m.params, 0.6, T, a, ux, uy, m.nv)
    s = O.OracleSolver(m, g)
    s.set_state(U)
    s.finalize_ic(0.6)
    r = s.run(0.6, 1e9, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=nsteps)
    rec = event_record(k, r, s.get_state())
    s.close()
    return rec


def _results_rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="2")
    import datetime
    from fivo2d.events import gather_event_results
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        m, grids = _small_events()
        mine = shard_events([g.Nx * g.Ny for g in grids], world, rank)
        local = [_run_event_on_oracle(m, grids[k], k) for k in mine]
        merged = gather_event_results(local, len(grids))
        if rank == 0:
            single = [_run_event_on_oracle(m, g, k) for k, g in enumerate(grids)]
            q.put((merged, single))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_results_equal_single_rank_run():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_results_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged, single = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs)
    assert len(merged) == len(single) == 6
    for a, b in zip(merged, single):
        assert a["ok"] and a["nsteps"] == 3
        for key in ("event", "tau", "nsteps", "nprimfail", "maxu", "dQ", "Q0", "Q1", "minPtot", "state_sha1"):
            assert a[key] == b[key], (key, a, b)


def test_gather_refuses_a_missing_event():
    ctx = mp.get_context("spawn")
    port = _free_port()
    q = ctx.Queue()
    procs = [ctx.Process(target=_missing_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert sorted(q.get(timeout=5) for _ in range(2)) == [True, True]


def _missing_rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    from fivo2d.events import gather_event_results
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local = [{"event": 0}] if rank == 0 else []          # event 1 is never run
        try:
            gather_event_results(local, 2)
            q.put(False)
        except RuntimeError:
            q.put(True)
        dist.barrier()
    finally:
        dist.destroy_process_group()
