"""Batches of events (fivo_batch_*): many independent events of uneven grid
sizes advanced together, one context and stream per event, driven by the
library's worker threads.

The batch is a scheduling layer only: every event's run must equal, to the bit,
the same event run alone through fivo_run (and, for one of them, the oracle).
Grid sizes follow the event-by-event workload: the box half-width scales with N
so that dx = 30/384 fm for every event.
"""
import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.solver import GPUBatch2D, GPUWork2D, set_cells

pytestmark = pytest.mark.gpu

DX = 30.0 / 384.0


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    same = a.view(np.int64) == b.view(np.int64)
    return bool(np.all(same | (np.isnan(a) & np.isnan(b))))


def _model():
    return fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                                 enable_diff=True, eta_over_s=0.16, tauShear_coeff=0.2, zeta_over_s=0.05,
                                 bulk_model="gaussian", bulk_T0=0.180, bulk_width=0.024, kappa_coeff=0.5)


def _events(sizes, tau0=0.6, seed0=1001):
    m = _model()
    grids, states = [], []
    for k, (nx, ny) in enumerate(sizes):
        g = fivo2d.make_grid2d(nx, ny, xmax=nx * DX / 2, ymax=ny * DX / 2)
        T, a, ux, uy, _ = ic.glauber_fields(g, tau0, seed0 + k)
        U, _ = set_cells(m, tau0, T, a, ux, uy)
        grids.append(g)
        states.append(U)
    return m, grids, states


def test_batch_run_equals_single_runs(gpu_lib):
    sizes = [(24, 24), (40, 32), (32, 48), (56, 56)]
    m, grids, states = _events(sizes)
    b = GPUBatch2D(m, grids, nworkers=3, lib=gpu_lib)
    for e, U in zip(b.events, states):
        e.set_state(U)
        e.finalize_ic(0.6)
    rb = b.run(0.6, 1.4, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=12)
    for k, (g, U) in enumerate(zip(grids, states)):
        w = GPUWork2D(m, g, lib=gpu_lib)
        w.set_state(U)
        w.finalize_ic(0.6)
        rw = w.run(0.6, 1.4, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=12)
        assert rb[k]["status"] == A.FIVO_OK
        for key in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu", "max_shear_res", "dQ"):
            assert rb[k][key] == rw[key] or (np.isnan(rb[k][key]) and np.isnan(rw[key])), (k, key)
        assert bits_equal(b.events[k].get_state(), w.get_state()), k
        hb, hw = b.events[k].get_history(), w.get_history()
        for name in hb:
            assert bits_equal(hb[name], hw[name]), (k, name)
        w.close()
    # and one event against the oracle
    o = O.OracleSolver(m, grids[1])
    o.set_state(states[1])
    o.finalize_ic(0.6)
    ro = o.run(0.6, 1.4, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=12)
    assert ro["tau"] == rb[1]["tau"] and ro["nsteps"] == rb[1]["nsteps"]
    assert bits_equal(o.get_state(), b.events[1].get_state())
    b.close()


def test_batch_advance_in_chunks(gpu_lib):
    """fivo_batch_advance step by step (per-event tau) equals one batch run."""
    sizes = [(24, 32), (36, 36), (28, 20)]
    m, grids, states = _events(sizes, seed0=1101)
    ba = GPUBatch2D(m, grids, nworkers=2, lib=gpu_lib)
    bb = GPUBatch2D(m, grids, nworkers=2, lib=gpu_lib)
    for bt in (ba, bb):
        for e, U in zip(bt.events, states):
            e.set_state(U)
            e.finalize_ic(0.6)
            e.rhs(0.6)
    taus = [0.6] * len(sizes)
    for _ in range(5):
        r = ba.advance(taus, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=1)
        assert all(x["ok"] and x["nsteps"] == 1 for x in r)
        taus = [x["tau"] for x in r]
    r5 = bb.advance([0.6] * len(sizes), 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=5)
    for k in range(len(sizes)):
        assert r5[k]["tau"] == taus[k]
        assert bits_equal(ba.events[k].get_state(), bb.events[k].get_state())
    ba.close()
    bb.close()


def test_batch_rejects_bad_event(gpu_lib):
    m = _model()
    grids = [fivo2d.make_grid2d(24, 24, xmax=1.0, ymax=1.0), fivo2d.make_grid2d(24, 24, xmax=1.0, ymax=1.0)]
    grids[1].Nx = 4                                      # make_grid2d refuses N <= 8; so must the library
    with pytest.raises(A.FivoError) as e:
        GPUBatch2D(m, grids, lib=gpu_lib)
    assert "event 1" in str(e.value)


def _single_runs(gpu_lib, m, grids, states, tau0, taufinal, cfl, cfltau, integrator, max_steps, precision=None,
                 guess=None, mode=None):
    out = []
    for g, U in zip(grids, states):
        w = GPUWork2D(m, g, lib=gpu_lib)
        if precision is not None:
            w.set_precision(precision)
        if guess is not None:
            guess.attach(w, mode)
        w.set_state(U)
        w.finalize_ic(tau0)
        r = w.run(tau0, taufinal, cfl, cfltau, integrator, max_steps=max_steps)
        out.append((r, w.get_state(), w.get_history()))
        w.close()
    return out


def _assert_batch_equals(b, rb, singles):
    for k, (rw, Uw, hw) in enumerate(singles):
        assert rb[k]["status"] == A.FIVO_OK
        for key in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu", "max_shear_res", "dQ", "Q0", "Q1",
                    "minPtot"):
            assert rb[k][key] == rw[key] or (np.isnan(rb[k][key]) and np.isnan(rw[key])), (k, key, rb[k][key], rw[key])
        assert bits_equal(b.events[k].get_state(), Uw), k
        hb = b.events[k].get_history()
        for name in hb:
            assert bits_equal(hb[name], hw[name]), (k, name)


@pytest.mark.parametrize("integrator,graphs,tune", [(A.FIVO_SSPRK3, True, True), (A.FIVO_SSPRK3, False, False),
                                                    (A.FIVO_SSPRK2, True, False)])
def test_lockstep_batch_equals_single_runs(gpu_lib, integrator, graphs, tune):
    """Lockstep mode: one launch per kernel over all events (uneven grids), the
    launch sequences replayed from CUDA graphs or launched directly, the
    schedule timed and chosen on the first steps. Every event equals its
    separate fivo_run bit for bit (state, history and the run's results), events
    leave the lockstep at different steps (taufinal), and one event also equals
    the oracle."""
    sizes = [(24, 24), (40, 32), (32, 48), (56, 56), (20, 28)]
    m, grids, states = _events(sizes, seed0=1201)
    b = GPUBatch2D(m, grids, nworkers=3, lib=gpu_lib)
    b.set_lockstep(True, graphs=graphs, tune=tune)
    for e, U in zip(b.events, states):
        e.set_state(U)
        e.finalize_ic(0.6)
    rb = b.run(0.6, 1.2, 0.2, 0.05, integrator, max_steps=60)
    info = b.lockstep_info()
    assert info["enabled"] and info["graphs"] == graphs and info["steps"] >= 12
    assert len({r["nsteps"] for r in rb}) > 1      # events leave the lockstep at different steps
    if tune:   # every candidate timed; one kept once the 16 tuning steps are done
        assert all(c["best_step_ms"] > 0 for c in info["candidates"])
        assert info["chosen"] >= 0 or info["steps"] < 16
        assert any(c["faces_one_launch"] for c in info["candidates"])
    singles = _single_runs(gpu_lib, m, grids, states, 0.6, 1.2, 0.2, 0.05, integrator, 60)
    _assert_batch_equals(b, rb, singles)
    o = O.OracleSolver(m, grids[4])
    o.set_state(states[4])
    o.finalize_ic(0.6)
    ro = o.run(0.6, 1.2, 0.2, 0.05, integrator, max_steps=60)
    assert ro["tau"] == rb[4]["tau"] and ro["nsteps"] == rb[4]["nsteps"]
    assert bits_equal(o.get_state(), b.events[4].get_state())
    b.close()


@pytest.mark.parametrize("integrator,cfl", [(A.FIVO_SSPRK2, 1.5), (A.FIVO_SSPRK3, 3.0)])
def test_lockstep_fallback_steps(gpu_lib, integrator, cfl):
    """A CFL number far above the stable one makes optimistic steps find
    inadmissible cells: those events are undone and stepped alone with MOOD
    retries and halvings, and still equal their separate runs bit for bit."""
    sizes = [(32, 32), (24, 40), (36, 28)]
    m, grids, states = _events(sizes, seed0=1201)
    b = GPUBatch2D(m, grids, nworkers=2, lib=gpu_lib)
    b.set_lockstep(True, graphs=True)
    for e, U in zip(b.events, states):
        e.set_state(U)
        e.finalize_ic(0.6)
    rb = b.run(0.6, 10.0, cfl, 0.5, integrator, max_steps=8)
    assert b.lockstep_info()["fallbacks"] > 0
    singles = _single_runs(gpu_lib, m, grids, states, 0.6, 10.0, cfl, 0.5, integrator, 8)
    _assert_batch_equals(b, rb, singles)
    b.close()


def test_lockstep_fp32_and_advance(gpu_lib):
    """The FP32 form in lockstep equals the FP32 form of separate runs bit for
    bit, and lockstep advance in chunks equals one lockstep run."""
    sizes = [(24, 32), (36, 36), (28, 20)]
    m, grids, states = _events(sizes, seed0=1301)
    b = GPUBatch2D(m, grids, nworkers=2, lib=gpu_lib)
    b.set_lockstep(True, graphs=True)
    for e, U in zip(b.events, states):
        e.set_precision(A.FIVO_PRECISION_FP32)
        e.set_state(U)
        e.finalize_ic(0.6)
    rb = b.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=6)
    singles = _single_runs(gpu_lib, m, grids, states, 0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, 6,
                           precision=A.FIVO_PRECISION_FP32)
    _assert_batch_equals(b, rb, singles)
    b.close()
    ba = GPUBatch2D(m, grids, nworkers=2, lib=gpu_lib)
    bb = GPUBatch2D(m, grids, nworkers=2, lib=gpu_lib)
    ba.set_lockstep(True, graphs=True)
    for bt in (ba, bb):
        for e, U in zip(bt.events, states):
            e.set_state(U)
            e.finalize_ic(0.6)
            e.rhs(0.6)
    taus = [0.6] * len(sizes)
    for _ in range(4):
        r = ba.advance(taus, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=1)
        assert all(x["ok"] and x["nsteps"] == 1 for x in r)
        taus = [x["tau"] for x in r]
    r4 = bb.advance([0.6] * len(sizes), 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=4)
    for k in range(len(sizes)):
        assert r4[k]["tau"] == taus[k]
        assert bits_equal(ba.events[k].get_state(), bb.events[k].get_state())
    ba.close()
    bb.close()


@pytest.fixture(scope="module")
def small_guess(gpu_lib):
    """a network trained briefly on pairs harvested from one small event"""
    from fivo2d.guess import RecoveryGuess
    m, grids, states = _events([(48, 48)], seed0=2301)
    g = RecoveryGuess(seed=5, lib=gpu_lib)
    g.reserve(400_000)
    w = GPUWork2D(m, grids[0], lib=gpu_lib)
    w.set_state(states[0])
    w.finalize_ic(0.6)
    tau = 0.6
    for _ in range(12):
        r = w.advance(tau, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=1)
        assert r["ok"]
        tau = r["tau"]
        w.update_primitives(tau)
        g.harvest(w, tau)
    w.close()
    g.fit_norm()
    g.train(300, ctas_per_step=64, lr=2e-3, seed=9)
    yield g
    g.close()


@pytest.mark.parametrize("mode", [A.FIVO_GUESS_EVERY_CELL, A.FIVO_GUESS_DEFERRED])
def test_lockstep_learned_guess_equals_single_runs(gpu_lib, small_guess, mode):
    """The learned guess in lockstep: every cell's tile (k_prim_learned's body per
    block) or the union of the events' deferred cells in shared tensor-core tiles
    (the retry across events), then the full recovery of what is left. Each event
    equals its separate run with the same network attached, bit for bit, and the
    Newton statistics of the guess agree event by event."""
    from fivo2d.guess import newton_stats
    g = small_guess
    sizes = [(24, 24), (40, 32), (32, 48), (20, 28)]
    m, grids, states = _events(sizes, seed0=1501)
    b = GPUBatch2D(m, grids, nworkers=2, lib=gpu_lib)
    b.set_lockstep(True, graphs=True)
    for e, U in zip(b.events, states):
        g.attach(e, mode)
        e.set_state(U)
        e.finalize_ic(0.6)
        newton_stats(e, reset=True)
    rb = b.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=10)
    stats_b = [newton_stats(e) for e in b.events]
    out = []
    for gr, U in zip(grids, states):
        w = GPUWork2D(m, gr, lib=gpu_lib)
        g.attach(w, mode)
        w.set_state(U)
        w.finalize_ic(0.6)
        newton_stats(w, reset=True)
        r = w.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=10)
        out.append((r, w.get_state(), w.get_history(), newton_stats(w)))
        w.close()
    _assert_batch_equals(b, rb, [o[:3] for o in out])
    for k, o in enumerate(out):
        for key in ("n_learn", "ok_learn", "it_learn", "deferred"):
            assert stats_b[k][key] == o[3][key], (k, key, stats_b[k][key], o[3][key])
    assert sum(s["n_learn"] for s in stats_b) > 0 and sum(s["ok_learn"] for s in stats_b) > 0
    b.close()


def test_lockstep_graphs_follow_the_boundary_condition(gpu_lib):
    """Lockstep advances with outflow, then periodic, then outflow boundaries on the
    same batch (each launch sequence is a graph per boundary condition): every event
    equals a separate context advanced with the same boundaries, bit for bit."""
    sizes = [(24, 24), (28, 20)]
    m, grids, states = _events(sizes, seed0=1601)
    b = GPUBatch2D(m, grids, lib=gpu_lib)
    b.set_lockstep(True, graphs=True)
    singles = [GPUWork2D(m, g, lib=gpu_lib) for g in grids]
    for e, w, U in zip(b.events, singles, states):
        for x in (e, w):
            x.set_state(U)
            x.finalize_ic(0.6)
            x.rhs(0.6)
    taus, tw = [0.6] * len(sizes), [0.6] * len(sizes)
    for bc in (A.FIVO_BC_OUTFLOW, A.FIVO_BC_PERIODIC, A.FIVO_BC_OUTFLOW):
        r = b.advance(taus, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, bc=bc, max_steps=2)
        assert all(x["ok"] and x["nsteps"] == 2 for x in r)
        taus = [x["tau"] for x in r]
        for k, w in enumerate(singles):
            tw[k] = w.advance(tw[k], 10.0, 0.2, 0.05, A.FIVO_SSPRK3, bc=bc, max_steps=2)["tau"]
    assert taus == tw
    for e, w in zip(b.events, singles):
        assert bits_equal(e.get_state(), w.get_state())
        w.close()
    b.close()


def test_lockstep_refuses_mixed_precision(gpu_lib):
    sizes = [(24, 24), (28, 28)]
    m, grids, states = _events(sizes, seed0=1401)
    b = GPUBatch2D(m, grids, lib=gpu_lib)
    b.set_lockstep(True)
    b.events[0].set_precision(A.FIVO_PRECISION_FP32)
    for e, U in zip(b.events, states):
        e.set_state(U)
        e.finalize_ic(0.6)
    with pytest.raises(A.FivoError) as e:
        b.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=2)
    assert "same precision" in str(e.value)
    b.close()


@pytest.mark.parametrize("integrator,mode", [(A.FIVO_SSPRK2, 1), (A.FIVO_SSPRK3, 1), (A.FIVO_SSPRK3, 2)])
def test_single_context_graphs_bitwise(gpu_lib, integrator, mode):
    """fivo_ctx_set_graphs: one context's run and advance through the lockstep
    sequences, replayed as CUDA graphs on the context's stream (mode 1) or launched
    kernel by kernel (mode 2), equal the per-kernel path bit for bit (state,
    history, run results), and the sequences count their kernels."""
    m, grids, states = _events([(40, 36)], seed0=1701)
    w1, w2 = GPUWork2D(m, grids[0], lib=gpu_lib), GPUWork2D(m, grids[0], lib=gpu_lib)
    w2.set_graphs(mode)
    for w in (w1, w2):
        w.set_state(states[0])
        w.finalize_ic(0.6)
    r1 = w1.run(0.6, 10.0, 0.2, 0.05, integrator, max_steps=15)
    r2 = w2.run(0.6, 10.0, 0.2, 0.05, integrator, max_steps=15)
    for key in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu", "max_shear_res", "dQ"):
        assert r1[key] == r2[key], (key, r1[key], r2[key])
    t1, t2 = r1["tau"], r2["tau"]
    for _ in range(3):
        t1 = w1.advance(t1, 10.0, 0.2, 0.05, integrator, max_steps=1)["tau"]
        t2 = w2.advance(t2, 10.0, 0.2, 0.05, integrator, max_steps=1)["tau"]
    assert t1 == t2
    assert bits_equal(w1.get_state(), w2.get_state())
    h1, h2 = w1.get_history(), w2.get_history()
    for name in h1:
        assert bits_equal(h1[name], h2[name]), name
    info = w2.lockstep_info()
    assert info["enabled"] and info["graphs"] == (mode == 1) and info["steps"] == 18 and info["kernels"] > 18 * 20
    assert not w1.lockstep_info()["enabled"]
    w1.close()
    w2.close()
