"""Event-by-event workloads: the uneven event list and its split over GPUs.

Events are independent (own grid, own dt, no coupling), so a multi-GPU run
gives each rank a share of the events and exchanges nothing on the data path;
only per-event results are gathered at the end. The split balances the cell
counts: events are dealt largest first to the rank with the least work so far
(longest-processing-time rule), which keeps ranks within one event of each
other.
"""
from __future__ import annotations

import numpy as np

from .model import Grid2D, make_grid2d

EVENT_SIZES = (96, 128, 192, 256, 320, 400)   # grid sizes of the event-by-event batch
EVENT_DX = 30.0 / 384.0                        # fm: the box scales with N at fixed dx


def event_grids(nevents: int, seed: int = 2026, sizes=EVENT_SIZES, dx: float = EVENT_DX) -> list[Grid2D]:
    """nevents grids with N drawn uniformly from `sizes` (seeded), box half-width N*dx/2."""
    rng = np.random.default_rng(seed)
    ns = rng.choice(np.asarray(sizes), size=nevents)
    return [make_grid2d(int(n), int(n), xmax=n * dx / 2, ymax=n * dx / 2) for n in ns]


def shard_events(cells, world: int, rank: int | None = None):
    """Assign events (given their interior cell counts) to `world` ranks.

    Returns the list of event indices of `rank`, or, when rank is None, the
    list of all ranks' lists. Deterministic: ties go to the lower rank, events
    of equal size keep their order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    cells = [int(c) for c in cells]
    order = sorted(range(len(cells)), key=lambda k: (-cells[k], k))
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += cells[k]
    parts = [sorted(p) for p in parts]
    return parts if rank is None else parts[rank]


def event_record(k: int, result: dict, U=None) -> dict:
    """The per-event bulk results of one run_sim_2d! (main2D.jl:558-560) that a
    multi-GPU batch gathers: ok, tau, nsteps, failure counts and the end-of-run
    diagnostics, plus a digest of the final state when U is given."""
    rec = {"event": int(k)}
    for key in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu", "dQ", "Q0", "Q1", "minPtot"):
        rec[key] = result[key]
    if U is not None:
        import hashlib
        rec["state_sha1"] = hashlib.sha1(np.ascontiguousarray(U, dtype=np.float64).tobytes()).hexdigest()
    return rec


def gather_event_results(local_records: list, nevents: int) -> list:
    """All-gather the per-event records of every rank over the default process
    group (the one collective of an event-sharded run, after the data path) and
    return them ordered by event index, on every rank. Raises when an event is
    missing or was run twice."""
    import torch.distributed as dist
    world = dist.get_world_size()
    parts = [None] * world
    dist.all_gather_object(parts, list(local_records))
    merged = sorted((rec for part in parts for rec in part), key=lambda r: r["event"])
    if [r["event"] for r in merged] != list(range(nevents)):
        raise RuntimeError("gather_event_results: an event is missing or was run on two ranks")
    return merged
