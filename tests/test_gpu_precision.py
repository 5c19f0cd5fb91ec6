"""The mixed-precision forms (fivo_ctx_set_precision: the face pass of rhs_2d! in
FP32; and the face pass plus the relaxation's sources in FP32) against the FP64 path
and the reference's gates:

  - the Gubser gate G1 (test/test_gubser2d.jl:97-246): L2(T) and L2(u) against the
    exact solution stay at the published values (the FP32 fluxes move them by far
    less than the scheme's own error), and the run differs from the FP64 one at the
    FP32 level;
  - the Bjorken gate G0 (test/test_bjorken2d.jl:133-169): convergence orders 2.00 /
    2.99 for SSPRK2 / SSPRK3 (a uniform state has equal fluxes on both faces of a
    cell in any precision, so the FP32 form must reproduce the FP64 run exactly);
  - the viscous MC-Glauber event: L2(T) <= 1e-6 and L2(pi) <= 1e-4 against the FP64
    path over a window that ends before the charge-free edge forms.
"""
import json
import math
import pathlib

import numpy as np
import pytest

import fivo2d
from fivo2d import _abi as A
from fivo2d import ic
from fivo2d.solver import GPUWork2D, set_cells

import test_oracle_gates as G

pytestmark = pytest.mark.gpu
GATES = json.loads((pathlib.Path(__file__).resolve().parent / "golden" / "gates.json").read_text())


def _gubser(lib, N, mode):
    s = GATES["gubser"]["settings"]
    g = fivo2d.make_grid2d(N, N, xmax=s["box"], ymax=s["box"])
    m = fivo2d.build_model_2d(eos=fivo2d.ConformalHQEOS())
    Tsc = ic.gubser_Tscale_from_center_T(s["tau0"], s["q"], s["Tc0"])
    T, a, ux, uy = ic.gubser_fields(g, s["tau0"], q=s["q"], Tscale=Tsc, alpha=s["alpha"])
    U, ok = set_cells(m, s["tau0"], T, a, ux, uy, lib=lib)
    w = GPUWork2D(m, g, lib=lib)
    w.set_precision(mode)
    w.set_state(U)
    r = w.run(s["tau0"], s["tauf"], s["CFL"], s["CFLtau"], A.FIVO_SSPRK2)
    assert r["ok"]
    w.update_primitives(r["tau"])
    pr = w.primitives()
    Te, uxe, uye, rr = ic.gubser_exact(g, r["tau"], q=s["q"], Tscale=Tsc)
    sl = g.interior()
    Tn = np.exp(pr["yT"]).reshape(g.Nxtot, g.Nytot)[sl]
    uxn = pr["ux"].reshape(g.Nxtot, g.Nytot)[sl]
    uyn = pr["uy"].reshape(g.Nxtot, g.Nytot)[sl]
    msk = rr[sl] <= s["rcmp"]
    L2T = math.sqrt(((Tn - Te[sl])[msk] ** 2).sum() / (Te[sl][msk] ** 2).sum())
    L2U = math.sqrt((((uxn - uxe[sl]) ** 2 + (uyn - uye[sl]) ** 2)[msk]).sum() /
                    ((uxe[sl] ** 2 + uye[sl] ** 2)[msk]).sum())
    w.close()
    return L2T, L2U, Tn


def test_gubser_gate_in_fp32_faces(gpu_lib):
    pub = GATES["gubser"]
    for N, key in ((100, 0), (200, 1)):
        l2t, l2u, T32 = _gubser(gpu_lib, N, A.FIVO_PRECISION_FP32_FACES)
        l2t64, l2u64, T64 = _gubser(gpu_lib, N, A.FIVO_PRECISION_FP64)
        assert abs(l2t - l2t64) <= 1e-3 * l2t64 and abs(l2u - l2u64) <= 1e-3 * l2u64, (l2t, l2t64, l2u, l2u64)
        assert abs(l2t - pub["L2T"][key]) <= 0.01 * pub["L2T"][key]
        d = np.linalg.norm(T32 - T64) / np.linalg.norm(T64)
        assert 0 < d < 1e-6, d                      # FP32-level, and really different arithmetic


def _bjorken_err(lib, cfltau, integrator, mode):
    s = GATES["bjorken"]["settings"]
    g = fivo2d.make_grid2d(s["N"], s["N"], xmax=s["box"], ymax=s["box"])
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS())
    T, a, ux, uy = ic.uniform_fields(g, T0=s["T0"], alpha0=s["alpha0"])
    U, _ = set_cells(m, s["tau0"], T, a, ux, uy, lib=lib)
    w = GPUWork2D(m, g, lib=lib)
    w.set_precision(mode)
    w.set_state(U)
    w.finalize_ic(s["tau0"])
    r = w.run(s["tau0"], s["tauf"], s["CFL"], cfltau, integrator)
    assert r["ok"]
    U1 = w.get_state()
    w.close()
    Tx, mux, nx_, ex, Px = G.bjorken_exact(m.params, s["T0"], s["alpha0"] * s["T0"], s["tau0"], r["tau"])
    ic_ = g.lin(g.nghost + g.Nx // 2 - 1, g.nghost + g.Ny // 2 - 1)
    return abs(U1[ic_, 3] - ex) / ex, U1


@pytest.mark.parametrize("integrator,expect", [(A.FIVO_SSPRK2, "ssprk2"), (A.FIVO_SSPRK3, "ssprk3")])
def test_bjorken_order_in_fp32_faces(gpu_lib, integrator, expect):
    errs = []
    for c in (0.02, 0.01, 0.005):
        e32, U32 = _bjorken_err(gpu_lib, c, integrator, A.FIVO_PRECISION_FP32_FACES)
        e64, U64 = _bjorken_err(gpu_lib, c, integrator, A.FIVO_PRECISION_FP64)
        assert np.array_equal(U32, U64)
        errs.append(e32)
    p2 = math.log2(errs[1] / errs[2])
    assert abs(p2 - GATES["bjorken"]["order"][expect]) < 0.15, (errs, p2)


@pytest.mark.parametrize("form", [A.FIVO_PRECISION_FP32_FACES, A.FIVO_PRECISION_FP32], ids=["fp32_faces", "fp32"])
def test_viscous_event_error_against_fp64(gpu_lib, form):
    """the bench workload's physics on a 192^2 event (dx = 30/384 fm), 30 SSPRK3 steps
    from tau0 = 0.6, with the FP32 face pass alone and with the relaxation's sources
    in FP32 as well"""
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                              enable_diff=True, eta_over_s=0.16, tauShear_coeff=0.2, deltaShear_factor=4 / 3,
                              zeta_over_s=0.05, bulk_model="gaussian", bulk_T0=0.180, bulk_width=0.024,
                              kappa_coeff=0.5)
    n = 192
    g = fivo2d.make_grid2d(n, n, xmax=n * 15.0 / 384, ymax=n * 15.0 / 384)
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1001)
    U, _ = set_cells(m, 0.6, T, a, ux, uy, lib=gpu_lib)
    out = {}
    for mode in (A.FIVO_PRECISION_FP64, form):
        w = GPUWork2D(m, g, lib=gpu_lib)
        w.set_precision(mode)
        w.set_state(U)
        w.finalize_ic(0.6)
        r = w.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=30)
        assert r["ok"] and r["nsteps"] == 30
        out[mode] = (w.primitives(), w.get_state())
        w.close()
    (p64, U64), (p32, U32) = out[A.FIVO_PRECISION_FP64], out[form]
    sx, sy = g.interior()
    ok = ((p64["ok"] == 1) & (p32["ok"] == 1)).reshape(g.Nxtot, g.Nytot)[sx, sy]
    T64 = np.exp(p64["yT"]).reshape(g.Nxtot, g.Nytot)[sx, sy][ok]
    T32 = np.exp(p32["yT"]).reshape(g.Nxtot, g.Nytot)[sx, sy][ok]
    l2T = np.linalg.norm(T32 - T64) / np.linalg.norm(T64)
    iP = m.layout.idx("pixx")
    pi64 = U64.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, iP:iP + 3][ok]
    pi32 = U32.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, iP:iP + 3][ok]
    l2pi = np.linalg.norm(pi32 - pi64) / np.linalg.norm(pi64)
    w64 = (p64["e"] + p64["P"]).reshape(g.Nxtot, g.Nytot)[sx, sy][ok]
    w32 = (p32["e"] + p32["P"]).reshape(g.Nxtot, g.Nytot)[sx, sy][ok]
    ie = m.layout.idx("pieta")
    pb64 = U64.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, ie][ok] / w64
    pb32 = U32.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, ie][ok] / w32
    l2pb = np.linalg.norm(pb32 - pb64) / np.linalg.norm(pb64)
    print(f"form {form} vs FP64 after 30 steps: L2(T) {l2T:.3e}, L2(pi) {l2pi:.3e}, L2(pibar) {l2pb:.3e}")
    assert 0 < l2T <= 1e-6 and l2pi <= 1e-4 and l2pb <= 1e-4, (l2T, l2pi, l2pb)


def test_relaxation_sources_in_fp32(gpu_lib):
    """one relaxation on the same evolved state: the FP32 sources move every dissipative
    row by FP32 rounding of the sources only (relative to the row's scale), the medium's
    rows not at all; consistent_m2 is refused in this mode"""
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                              enable_diff=True, eta_over_s=0.16, zeta_over_s=0.05, kappa_coeff=0.5,
                              consistent_fm=True, taupi_pi_factor=0.5, lambda_pi_Pi_factor=0.3,
                              lambda_Pi_pi_factor=0.2)
    g = fivo2d.make_grid2d(64, 64, xmax=64 * 15.0 / 384, ymax=64 * 15.0 / 384)
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1005)
    U, _ = set_cells(m, 0.6, T, a, ux, uy, lib=gpu_lib)
    w = GPUWork2D(m, g, lib=gpu_lib)
    w.set_state(U)
    w.finalize_ic(0.6)
    r = w.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=6)
    mid, hist = w.get_state(), w.get_history()
    out = {}
    for mode in (A.FIVO_PRECISION_FP64, A.FIVO_PRECISION_FP32):
        v = GPUWork2D(m, g, lib=gpu_lib)
        v.set_precision(mode)
        v.set_state(mid)
        v.set_history(**hist)
        v.update_primitives(r["tau"])
        v.relax(r["tau"], 0.02)
        out[mode] = v.get_state()
        v.close()
    w.close()
    a64, a32 = out[A.FIVO_PRECISION_FP64], out[A.FIVO_PRECISION_FP32]
    assert np.array_equal(a32[:, :4], a64[:, :4])
    for k in range(4, m.nv):
        scale = max(np.abs(a64[:, k]).max(), 1e-300)
        rel = np.abs(a32[:, k] - a64[:, k]).max() / scale
        assert rel <= 1e-5, (m.layout.names[k], rel)
    assert not np.array_equal(a32, a64)
    m2 = fivo2d.build_model_2d(enable_diff=True, consistent_m2=True)
    v = GPUWork2D(m2, g, lib=gpu_lib)
    assert gpu_lib.fivo_ctx_set_precision(v.h, A.FIVO_PRECISION_FP32) == A.FIVO_ERR_CONFIG
    v.close()


def test_precision_switch_and_refusal(gpu_lib):
    """an unknown mode is refused; switching back to FP64 mid-run continues as the
    FP64 path does from that state (bit for bit)"""
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_diff=True, kappa_coeff=0.5)
    g = fivo2d.make_grid2d(32, 32, xmax=32 * 15.0 / 384, ymax=32 * 15.0 / 384)
    T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1003)
    U, _ = set_cells(m, 0.6, T, a, ux, uy, lib=gpu_lib)
    w = GPUWork2D(m, g, lib=gpu_lib)
    assert gpu_lib.fivo_ctx_set_precision(w.h, 7) == A.FIVO_ERR_ARG
    w.set_state(U)
    w.finalize_ic(0.6)
    w.set_precision(A.FIVO_PRECISION_FP32_FACES)
    r = w.run(0.6, 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=5)
    mid = w.get_state()
    hist = w.get_history()
    w.set_precision(A.FIVO_PRECISION_FP64)
    r2 = w.advance(r["tau"], 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=5)
    v = GPUWork2D(m, g, lib=gpu_lib)
    v.set_state(mid)
    v.set_history(**hist)
    w.close()
    v.rhs(r["tau"])
    r3 = v.advance(r["tau"], 10.0, 0.2, 0.05, A.FIVO_SSPRK3, max_steps=5)
    assert r2["ok"] and r3["ok"] and r2["nsteps"] == r3["nsteps"] == 5
    v.close()


@pytest.mark.parametrize("case", ["ideal_conformal", "viscous_lhrg"])
def test_rhs_fp32_faces_against_fp64(gpu_lib, case):
    """one rhs_2d! on the same state: the FP32 face pass moves every row of dU by no more
    than FP32 rounding of the face fluxes allows (relative to the row's scale), and the
    signal speed by less than 1e-6"""
    if case == "ideal_conformal":
        g = fivo2d.make_grid2d(48, 48, xmax=10.0, ymax=10.0)
        m = fivo2d.build_model_2d(eos=fivo2d.ConformalHQEOS(g_eff=47.5, g_hq=0.0), with_charge=False)
        T, a, ux, uy = ic.gubser_fields(g, 1.0, q=1.0, Tscale=5.55 * fivo2d.model.HBARC, alpha=0.0)
        tau = 1.0
    else:
        m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_shear=True, enable_bulk=True,
                                  enable_diff=True, eta_over_s=0.16, kappa_coeff=0.5)
        g = fivo2d.make_grid2d(64, 64, xmax=64 * 15.0 / 384, ymax=64 * 15.0 / 384)
        T, a, ux, uy, _ = ic.glauber_fields(g, 0.6, 1004)
        tau = 0.6
    U, _ = set_cells(m, tau, T, a, ux, uy, lib=gpu_lib)
    out = {}
    for mode in (A.FIVO_PRECISION_FP64, A.FIVO_PRECISION_FP32_FACES):
        w = GPUWork2D(m, g, lib=gpu_lib)
        w.set_precision(mode)
        w.set_state(U)
        out[mode] = (w.rhs(tau), w.counters().amax)
        w.close()
    (d64, a64), (d32, a32) = out[A.FIVO_PRECISION_FP64], out[A.FIVO_PRECISION_FP32_FACES]
    sx, sy = g.interior()
    for k in range(m.nv):
        x64 = d64.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, k]
        x32 = d32.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, k]
        scale = max(np.abs(x64).max(), 1e-300)
        assert np.abs(x32 - x64).max() <= 1e-3 * scale, (k, np.abs(x32 - x64).max() / scale)
    assert abs(a32 - a64) <= 1e-6 * a64
    assert not np.array_equal(d32, d64)               # really the FP32 arithmetic
