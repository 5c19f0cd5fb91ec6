"""The learned recovery guess on the device (fivo_guess_*, k_prim_learned).

The network's tensor-core forward and backward passes are checked against the
CPU oracle (oracle/guess_oracle.py, which rounds to BF16 where the device does);
training on pairs harvested from the solver's own runs must drive the loss down;
a network whose every guess is rejected must leave a run bit-identical to the
plain one (the fallback is the plain warm-started recovery); and a trained
network's run must agree with the plain path to far better than the 1e-6 bound
on L2(T), while its guesses are accepted and save Newton updates.
"""
import pathlib
import sys

import numpy as np
import pytest

import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.guess import RecoveryGuess, newton_stats
from fivo2d.solver import GPUWork2D, set_cells

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1] / "oracle"))
import guess_oracle as GO  # noqa: E402

pytestmark = pytest.mark.gpu

DX = 30.0 / 384.0


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return bool(np.all((a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))))


def _model():
    return fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                                 enable_diff=True, eta_over_s=0.16, tauShear_coeff=0.2, zeta_over_s=0.05,
                                 bulk_model="gaussian", bulk_T0=0.180, bulk_width=0.024, kappa_coeff=0.5)


def _event(m, n, seed, tau0=0.6):
    g = fivo2d.make_grid2d(n, n, xmax=n * DX / 2, ymax=n * DX / 2)
    T, a, ux, uy, _ = ic.glauber_fields(g, tau0, seed)
    U, ok = set_cells(m, tau0, T, a, ux, uy)
    return g, U


def _norm():
    rng = np.random.default_rng(2)
    return np.concatenate([rng.normal(size=8) * 0.3, 1.0 + rng.random(8), rng.normal(size=3) * 0.2,
                           0.5 + rng.random(3)]).astype(np.float32)


def test_forward_matches_oracle(gpu_lib):
    g = RecoveryGuess(seed=11, lib=gpu_lib)
    nm = _norm()
    g.set_params(norm=nm)
    P, nm2 = g.get_params()
    assert np.array_equal(nm, nm2)
    raw = np.random.default_rng(5).normal(size=(1000, 8)).astype(np.float32)   # a ragged last tile
    y = g.forward(raw)
    yo, _ = GO.forward(P, GO.normalise(nm, raw))
    err = np.abs(y - yo)
    assert err.max() < 1e-2 and err.mean() < 1e-4, (err.max(), err.mean())
    g.close()


def test_gradient_matches_oracle(gpu_lib):
    g = RecoveryGuess(seed=12, lib=gpu_lib)
    nm = _norm()
    g.set_params(norm=nm)
    P, _ = g.get_params()
    rng = np.random.default_rng(6)
    samples = np.hstack([rng.normal(size=(512, 8)), rng.normal(size=(512, 3))]).astype(np.float32)
    gd, ld = g.grad(samples)
    go, lo = GO.grad(P, nm, samples)
    assert abs(ld - lo) <= 1e-4 * lo, (ld, lo)
    for a, b in ((GO.P_W1, GO.P_B1), (GO.P_B1, GO.P_W2), (GO.P_W2, GO.P_B2), (GO.P_B2, GO.P_W3),
                 (GO.P_W3, GO.P_B3), (GO.P_B3, GO.NPARAM)):
        rel = np.linalg.norm(gd[a:b] - go[a:b]) / max(np.linalg.norm(go[a:b]), 1e-30)
        assert rel < 1e-2, (a, b, rel)
    # the padding entries carry no gradient
    assert not gd[GO.P_W1:GO.P_B1].reshape(64, 16)[:, 8:].any()
    assert not gd[GO.P_B3 + 3:].any()
    g.close()


def _harvest(m, guess, seeds, n=96, steps=24):
    for seed in seeds:
        gr, U = _event(m, n, seed)
        w = GPUWork2D(m, gr, lib=guess.lib)
        w.set_state(U)
        w.finalize_ic(0.6)
        tau = 0.6
        for _ in range(steps):
            r = w.advance(tau, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=1)
            assert r["ok"]
            tau = r["tau"]
            w.update_primitives(tau)                # primitives of the current (relaxed) state
            guess.harvest(w, tau)
        w.close()


@pytest.fixture(scope="module")
def trained(gpu_lib):
    m = _model()
    g = RecoveryGuess(seed=3, lib=gpu_lib)
    g.reserve(2_000_000)
    _harvest(m, g, seeds=(2001, 2002, 2003))
    n = g.nsamples()
    assert n > 100_000
    g.fit_norm()
    l0, l1 = g.train(800, ctas_per_step=148, lr=2e-3, seed=9)
    return m, g, (l0, l1)


def test_training_reduces_the_loss(trained):
    _, g, (l0, l1) = trained
    assert l1 < l0 / 50, (l0, l1)


def _run(m, gr, U, lib, guess=None, steps=24, mode=A.FIVO_GUESS_EVERY_CELL):
    w = GPUWork2D(m, gr, lib=lib)
    if guess is not None:
        guess.attach(w, mode)
    w.set_state(U)
    w.finalize_ic(0.6)
    newton_stats(w, reset=True)
    r = w.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=steps)
    st = newton_stats(w)
    out = (r, w.get_state(), w.primitives(), st)
    w.close()
    return out


def test_rejected_guesses_fall_back_bitwise(gpu_lib):
    """zero weights and an absurd output mean: every learned attempt is rejected and
    the run is the plain run to the bit"""
    m = _model()
    gr, U = _event(m, 80, 2101)
    g = RecoveryGuess(seed=1, lib=gpu_lib)
    g.set_params(np.zeros(A.FIVO_GUESS_NPARAM, dtype=np.float32),
                 np.concatenate([np.zeros(8), np.ones(8), [8.0, 900.0, -900.0], np.ones(3)]).astype(np.float32))
    rp, Up, pp, sp = _run(m, gr, U, gpu_lib)
    rl, Ul, pl, sl = _run(m, gr, U, gpu_lib, guess=g)
    assert rp["nsteps"] == rl["nsteps"] and rp["tau"] == rl["tau"]
    assert bits_equal(Up, Ul)
    assert sl["n_learn"] > 0 and sl["ok_learn"] == 0
    assert sp["n_learn"] == 0 and sp["n_fast"] > 0
    g.close()


def test_trained_guess_run_agrees_and_saves_updates(trained, gpu_lib):
    m, g, _ = trained
    gr, U = _event(m, 96, 2199)                     # an event the network has not seen
    rp, Up, pp, sp = _run(m, gr, U, gpu_lib)
    rl, Ul, pl, sl = _run(m, gr, U, gpu_lib, guess=g)
    assert rl["ok"] and rl["nsteps"] == rp["nsteps"]
    sx, sy = gr.interior()
    ok = (pp["ok"] == 1).reshape(gr.Nxtot, gr.Nytot)[sx, sy]
    T_p = np.exp(pp["yT"]).reshape(gr.Nxtot, gr.Nytot)[sx, sy][ok]
    T_l = np.exp(pl["yT"]).reshape(gr.Nxtot, gr.Nytot)[sx, sy][ok]
    l2T = np.linalg.norm(T_l - T_p) / np.linalg.norm(T_p)
    assert l2T < 1e-6, l2T
    for k in ("ux", "uy"):
        a = pp[k].reshape(gr.Nxtot, gr.Nytot)[sx, sy][ok]
        b = pl[k].reshape(gr.Nxtot, gr.Nytot)[sx, sy][ok]
        assert np.linalg.norm(b - a) <= 1e-6 * max(np.linalg.norm(a), 1e-12)
    acc = sl["ok_learn"] / sl["n_learn"]
    assert acc > 0.9, sl
    # Newton updates per recovered cell: the learned attempts (plus their fallbacks)
    # against the plain warm-started pass
    it_l = (sl["it_learn"] + sl["it_fb"]) / sl["n_learn"]
    it_p = sp["it_fast"] / sp["n_fast"]
    print(f"updates per cell: learned {it_l:.3f} (accept {acc:.4f}), plain {it_p:.3f}; "
          f"deferred learned {sl['deferred']} plain {sp['deferred']}")


def test_rejected_deferred_guesses_fall_back_bitwise(gpu_lib):
    """the deferred mode with a network whose every guess is rejected: the deferred
    cells all go on to the full recovery and the run is the plain run to the bit"""
    m = _model()
    gr, U = _event(m, 80, 2101)
    g = RecoveryGuess(seed=1, lib=gpu_lib)
    g.set_params(np.zeros(A.FIVO_GUESS_NPARAM, dtype=np.float32),
                 np.concatenate([np.zeros(8), np.ones(8), [8.0, 900.0, -900.0], np.ones(3)]).astype(np.float32))
    rp, Up, pp, sp = _run(m, gr, U, gpu_lib)
    rl, Ul, pl, sl = _run(m, gr, U, gpu_lib, guess=g, mode=A.FIVO_GUESS_DEFERRED)
    assert rp["nsteps"] == rl["nsteps"] and rp["tau"] == rl["tau"]
    assert bits_equal(Up, Ul)
    assert sl["n_learn"] > 0 and sl["ok_learn"] == 0
    assert sl["n_fast"] == sp["n_fast"] and sl["deferred"] == sp["deferred"]
    g.close()


def test_deferred_guess_agrees_and_takes_cells_off_the_full_recovery(trained, gpu_lib):
    """the deferred mode with the trained network, over a longer window (the fireball
    edge forms and cells leave vacuum without a warm start): the same primitives as the
    plain run to L2(T) <= 1e-6, and the network converges a share of the cells that the
    plain path sends to the full cons_to_prim_2d!"""
    m, g, _ = trained
    gr, U = _event(m, 96, 2199)
    rp, Up, pp, sp = _run(m, gr, U, gpu_lib, steps=80)
    rl, Ul, pl, sl = _run(m, gr, U, gpu_lib, guess=g, steps=80, mode=A.FIVO_GUESS_DEFERRED)
    assert rl["ok"] and rl["nsteps"] == rp["nsteps"]
    sx, sy = gr.interior()
    ok = ((pp["ok"] == 1) & (pl["ok"] == 1)).reshape(gr.Nxtot, gr.Nytot)[sx, sy]
    T_p = np.exp(pp["yT"]).reshape(gr.Nxtot, gr.Nytot)[sx, sy][ok]
    T_l = np.exp(pl["yT"]).reshape(gr.Nxtot, gr.Nytot)[sx, sy][ok]
    l2T = np.linalg.norm(T_l - T_p) / np.linalg.norm(T_p)
    print(f"deferred mode: {sl['n_learn']} guesses on deferred cells, {sl['ok_learn']} converged "
          f"({sl['it_learn'] / max(1, sl['n_learn']):.2f} updates each); full recoveries: plain "
          f"{sp['deferred']}, with the network {sl['deferred']}; L2(T) {l2T:.2e}")
    assert l2T < 1e-6, l2T
    assert sl["n_learn"] > 0 and sl["ok_learn"] > 0
    assert sl["deferred"] < sp["deferred"]


def test_guess_argument_refusals(gpu_lib):
    import ctypes as C
    g = RecoveryGuess(seed=2, lib=gpu_lib)
    s = np.zeros((100, 11), dtype=np.float32)                # not a multiple of 128
    grad = np.zeros(A.FIVO_GUESS_NPARAM, dtype=np.float32)
    loss = C.c_double()
    fp = C.POINTER(C.c_float)
    assert gpu_lib.fivo_guess_grad(g.h, s.ctypes.data_as(fp), 100, grad.ctypes.data_as(fp),
                                   C.byref(loss)) == A.FIVO_ERR_ARG
    out = np.zeros(2)
    assert gpu_lib.fivo_guess_train(g.h, 10, 4, C.c_float(1e-3), 1, out.ctypes.data_as(A._D)) == A.FIVO_ERR_ARG  # no samples
    y = g.forward(np.zeros((1, 8), dtype=np.float32))      # one row, a ragged tile
    assert y.shape == (1, 3) and np.isfinite(y).all()
    m = _model()
    w = GPUWork2D(m, fivo2d.make_grid2d(16, 16), lib=gpu_lib)
    assert gpu_lib.fivo_ctx_set_guess_mode(w.h, 5) == A.FIVO_ERR_ARG
    w.close()
    g.close()
