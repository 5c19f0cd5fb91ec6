"""The consistent charm first moment on the device, against the oracle.

The closure adds a source vector to the charge row of the relaxation (the gradient
of T, the acceleration, nu.grad u, the expansion and D ln h, each behind its Terms
switch; src2d/hq_consistent_firstmoment2d.jl:218-282, src2d/dissipation2d.jl:589-623).
Every run here must equal the oracle's to the bit: the reference's own gate solves
(test/test_consistent_fm2d.jl Gc5 and Gc7) and a switched-term variant.
"""
import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d.solver import GPUWork2D

import test_oracle_consistent_fm as G

pytestmark = pytest.mark.gpu


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    same = a.view(np.int64) == b.view(np.int64)
    return bool(np.all(same | (np.isnan(a) & np.isnan(b))))


@pytest.mark.parametrize("terms", [None, {"fm_dlnh": False, "fm_inertial": False}, {"fm_gradT": False}],
                         ids=["all", "no_dlnh_inertial", "no_gradT"])
def test_gradient_solve_matches_oracle(gpu_lib, terms):
    """Gc5's solve (48^2, a 10 % Gaussian bump, tau 0.4 -> 0.6) with the closure on."""
    g = fivo2d.make_grid2d(48, 48, xmax=6.0, ymax=6.0)
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.2, consistent_fm=True,
                              terms=terms)
    U = G.gc5_state(g, m)
    o = O.OracleSolver(m, g)
    o.set_state(U)
    ro = o.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)
    w = GPUWork2D(m, g, lib=gpu_lib)
    w.set_state(U)
    rw = w.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)
    assert ro["ok"] and rw["ok"] and ro["nsteps"] == rw["nsteps"] and ro["tau"] == rw["tau"]
    assert bits_equal(o.get_state(), w.get_state())
    ho, hw = o.get_history(), w.get_history()
    for name in ho:
        assert bits_equal(ho[name], hw[name]), name
    o.close()
    w.close()


def test_closure_moves_the_device_solve(gpu_lib):
    """Off and on differ on the device too (a source that changes nothing is not wired in)."""
    g = fivo2d.make_grid2d(48, 48, xmax=6.0, ymax=6.0)
    out = []
    for cfm in (False, True):
        m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.2,
                                  consistent_fm=cfm)
        w = GPUWork2D(m, g, lib=gpu_lib)
        w.set_state(G.gc5_state(g, m))
        assert w.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)["ok"]
        out.append(w.get_state())
        w.close()
    assert np.max(np.abs(out[1] - out[0])) > 0


def test_bjorken_current_sign_on_the_device(gpu_lib):
    """Gc7 on the device: the step-by-step trajectory equals the oracle's to the bit,
    and it follows the derived ODE, not the sign-flipped one."""
    s = G.GC7
    g, m, U = G.gc7_setup()
    traj = []
    for solver in (O.OracleSolver(m, g), GPUWork2D(m, g, lib=gpu_lib)):
        solver.set_state(U)
        solver.finalize_ic(s["TAU0"], A.FIVO_BC_PERIODIC)
        traj.append(G.gc7_trajectory(solver, g, m))
        final = solver.get_state()
        traj[-1] = traj[-1] + (final,)
        solver.close()
    for a, b in zip(traj[0], traj[1]):
        assert bits_equal(a, b)
    ts, nus, Ts, ns, _ = traj[1]
    dev_phys = np.max(np.abs(nus - G.gc7_ode(m, ts, nus, Ts, ns, +1.0))) / abs(nus[0])
    dev_flip = np.max(np.abs(nus - G.gc7_ode(m, ts, nus, Ts, ns, -1.0))) / abs(nus[0])
    assert dev_phys < 2e-3 and dev_flip > 0.1
    assert ts[-1] * nus[-1] < ts[0] * nus[0]
