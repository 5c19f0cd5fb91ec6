"""The workload configurations at their own sizes on the GPU.

  config 1  ideal conformal Gubser flow, 128^2 on [-10, 10] fm, tau 1 -> 4, SSPRK2,
            CFLtau = 0.25, T0hat = 5.55 fm^-1, e = (pi^2/30) 47.5 T^4, no charge: the
            whole run bit for bit against the oracle, and L2(T), L2(u) against the
            exact solution (test/test_gubser2d.jl's measure: cells with r <= 3 fm).
  config 2  the viscous MC-Glauber event at 384^2 on [-15, 15] fm, SSPRK3: the first
            steps bit for bit against the oracle (the grid-size-dependent indexing,
            tile remainders and queue capacities of the full size), and the whole
            run to tau = 10 fm/c without a failed step.
  config 4  the same physics at 512^2: the FP32 face pass against FP64 on one event,
            L2 and Linf of T, u^x, u^y, pibar and n at tau = 4 fm/c.
"""
import math

import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.solver import GPUWork2D

from test_gpu_parity import _assert_same_work, _pair

pytestmark = pytest.mark.gpu


def _viscous_model():
    return fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True, enable_diff=True,
                                 eta_over_s=0.16, tauShear_coeff=0.2, deltaShear_factor=4 / 3, zeta_over_s=0.05,
                                 bulk_model="gaussian", bulk_T0=0.180, bulk_width=0.024, kappa_coeff=0.5)


def test_config1_gubser_128_whole_run(gpu_lib):
    g = fivo2d.make_grid2d(128, 128, xmax=10.0, ymax=10.0)
    m = fivo2d.build_model_2d(eos=fivo2d.ConformalHQEOS(g_eff=47.5, g_hq=0.0), with_charge=False)
    Tsc = 5.55 * fivo2d.model.HBARC
    T, a, ux, uy = ic.gubser_fields(g, 1.0, q=1.0, Tscale=Tsc, alpha=0.0)
    U, _ = O.set_cells(m.params, 1.0, T, a, ux, uy, m.nv)
    w, o = _pair(m, g, U)
    rw = w.run(1.0, 4.0, 0.2, 0.25, A.FIVO_SSPRK2)
    ro = o.run(1.0, 4.0, 0.2, 0.25, A.FIVO_SSPRK2)
    for k in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu"):
        assert rw[k] == ro[k], (k, rw[k], ro[k])
    assert rw["ok"] and rw["tau"] == 4.0 and rw["nprimfail"] == 0
    _assert_same_work(w, o, "config 1")
    w.update_primitives(4.0)
    p = w.primitives()
    Te, uxe, uye, r = ic.gubser_exact(g, 4.0, q=1.0, Tscale=Tsc)
    sx, sy = g.interior()
    msk = r[sx, sy] <= 3.0
    Tn = np.exp(p["yT"]).reshape(g.Nxtot, g.Nytot)[sx, sy]
    uxn = p["ux"].reshape(g.Nxtot, g.Nytot)[sx, sy]
    uyn = p["uy"].reshape(g.Nxtot, g.Nytot)[sx, sy]
    L2T = math.sqrt(((Tn - Te[sx, sy])[msk] ** 2).sum() / (Te[sx, sy][msk] ** 2).sum())
    L2u = math.sqrt((((uxn - uxe[sx, sy]) ** 2 + (uyn - uye[sx, sy]) ** 2)[msk]).sum() /
                    ((uxe[sx, sy] ** 2 + uye[sx, sy] ** 2)[msk]).sum())
    print(f"config 1: {rw['nsteps']} steps, L2(T) = {L2T:.3e}, L2(u) = {L2u:.3e}")
    # measured 94 steps, L2(T) = 3.19e-3, L2(u) = 7.12e-3 (the reference's gate figures
    # at dx = 0.2 fm over tau 1 -> 2 are 3.29e-3 and 7.73e-3)
    assert L2T < 1e-2 and L2u < 2e-2
    w.close()
    o.close()


def test_config2_event_384_first_steps_bitwise(gpu_lib):
    g = fivo2d.make_grid2d(384, 384, xmax=15.0, ymax=15.0)
    m = _viscous_model()
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1001)
    U, _ = O.set_cells(m.params, 0.6, T, a, ux, uy, m.nv)
    w, o = _pair(m, g, U)
    for s in (w, o):
        s.finalize_ic(0.6)
    rw = w.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=3)
    ro = o.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=3)
    for k in ("ok", "tau", "nsteps", "nprimfail", "nvacuum", "maxu", "max_shear_res"):
        assert rw[k] == ro[k], (k, rw[k], ro[k])
    assert rw["nsteps"] == 3
    _assert_same_work(w, o, "config 2, 384^2")
    w.close()
    o.close()


def test_config2_event_384_runs_to_tau_10(gpu_lib):
    g = fivo2d.make_grid2d(384, 384, xmax=15.0, ymax=15.0)
    m = _viscous_model()
    w = GPUWork2D(m, g, lib=gpu_lib)
    w.glauber_ic(0.6, 1001)
    r = w.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3)
    print(f"config 2: {r['nsteps']} steps to tau = {r['tau']}, nprimfail {r['nprimfail']}, maxu {r['maxu']:.3f}, "
          f"dQ {r['dQ']:.3e}, minPtot {r['minPtot']:.3e}")
    assert r["ok"] and r["tau"] == 10.0
    assert r["nprimfail"] == 0
    w.close()


def _fields(w, g, m):
    p = w.primitives()
    U = w.get_state()
    sx, sy = g.interior()
    okm = (p["ok"] == 1).reshape(g.Nxtot, g.Nytot)[sx, sy]
    f = {}
    f["T"] = np.exp(p["yT"]).reshape(g.Nxtot, g.Nytot)[sx, sy]
    f["ux"] = p["ux"].reshape(g.Nxtot, g.Nytot)[sx, sy]
    f["uy"] = p["uy"].reshape(g.Nxtot, g.Nytot)[sx, sy]
    f["n"] = p["n"].reshape(g.Nxtot, g.Nytot)[sx, sy]
    wpl = (p["e"] + p["P"]).reshape(g.Nxtot, g.Nytot)[sx, sy]
    f["pibar"] = U.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, m.layout.idx("pieta")] / wpl
    return f, okm


def test_config4_fp32_faces_at_512(gpu_lib):
    g = fivo2d.make_grid2d(512, 512, xmax=15.0, ymax=15.0)
    m = _viscous_model()
    runs = []
    for prec in (A.FIVO_PRECISION_FP64, A.FIVO_PRECISION_FP32_FACES):
        w = GPUWork2D(m, g, lib=gpu_lib)
        w.glauber_ic(0.6, 1001)
        w.set_precision(prec)
        r = w.run(0.6, 4.0, 0.2, 0.05, A.FIVO_SSPRK3)
        assert r["ok"] and r["tau"] == 4.0
        runs.append(_fields(w, g, m))
        w.close()
    (f64, ok64), (f32, ok32) = runs
    ok = ok64 & ok32
    errs = {}
    for k in ("T", "ux", "uy", "pibar", "n"):
        a, b = f32[k][ok], f64[k][ok]
        errs[k] = (float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)),
                   float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)))
    print("config 4 at tau = 4, FP32 faces vs FP64 (L2, Linf):", errs)
    # Over 3.4 fm/c of an MC-Glauber event the FP32 rounding of the faces grows to
    # 1.9e-5 in T and 1.0e-4 in pibar (measured on this seed): the 1e-6 target of the
    # mixed-precision form holds over short windows only (a 30-step batch: 1.2e-7).
    # The bounds below are a regression guard a decade above the measurement.
    assert errs["T"][0] < 2e-4
    assert errs["pibar"][0] < 1e-3
    assert errs["ux"][0] < 1e-3 and errs["uy"][0] < 1e-3
