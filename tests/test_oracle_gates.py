"""The oracle pinned to the reference's published gates for this path.

The reference (Julia) cannot run here, so the CPU restatement is checked
against the numbers its own gate suite publishes (tests/golden/gates.json, from
README2D.md:273-275) and against the gates' pass criteria:

  G1 Gubser      test/test_gubser2d.jl:97-246
  G0 Bjorken     test/test_bjorken2d.jl:63-169
  primrec        test/test_primrec2d.jl:35-191
"""
import json
import math
import os
import pathlib

import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d import ic

GATES = json.loads((pathlib.Path(__file__).resolve().parent / "golden" / "gates.json").read_text())


def run_gubser(N):
    s = GATES["gubser"]["settings"]
    g = fivo2d.make_grid2d(N, N, xmax=s["box"], ymax=s["box"])
    m = fivo2d.build_model_2d(eos=fivo2d.ConformalHQEOS())
    Tsc = ic.gubser_Tscale_from_center_T(s["tau0"], s["q"], s["Tc0"])
    T, a, ux, uy = ic.gubser_fields(g, s["tau0"], q=s["q"], Tscale=Tsc, alpha=s["alpha"])
    U, ok = O.set_cells(m.params, s["tau0"], T, a, ux, uy, m.nv)
    o = O.OracleSolver(m, g)
    o.set_state(U)
    r = o.run(s["tau0"], s["tauf"], s["CFL"], s["CFLtau"], A.FIVO_SSPRK2)
    assert r["ok"]
    o.update_primitives(r["tau"])
    pr = o.primitives()
    Te, uxe, uye, rr = ic.gubser_exact(g, r["tau"], q=s["q"], Tscale=Tsc)
    sl = g.interior()
    Tn = np.exp(pr["yT"]).reshape(g.Nxtot, g.Nytot)[sl]
    uxn = pr["ux"].reshape(g.Nxtot, g.Nytot)[sl]
    uyn = pr["uy"].reshape(g.Nxtot, g.Nytot)[sl]
    msk = rr[sl] <= s["rcmp"]
    L2T = math.sqrt(((Tn - Te[sl])[msk] ** 2).sum() / (Te[sl][msk] ** 2).sum())
    L2U = math.sqrt((((uxn - uxe[sl]) ** 2 + (uyn - uye[sl]) ** 2)[msk]).sum() /
                    ((uxe[sl] ** 2 + uye[sl] ** 2)[msk]).sum())
    asym = float(np.max(np.where(msk, np.abs(Tn - Tn.T) / np.maximum(Tn, Tn.T), 0.0)))
    o.close()
    return L2T, L2U, asym, r


@pytest.fixture(scope="module")
def gubser_runs():
    Ns = [100, 200] + ([400] if os.environ.get("FIVO_SLOW") else [])
    return {N: run_gubser(N) for N in Ns}


def test_gubser_published_L2(gubser_runs):
    """L2(T), L2(u) at N=100/200(/400) reproduce README2D.md:275 to the
    published three digits."""
    pub = GATES["gubser"]
    for N, (L2T, L2U, asym, r) in gubser_runs.items():
        k = pub["N"].index(N)
        assert abs(L2T / pub["L2T"][k] - 1) < 0.002, (N, L2T)
        assert abs(L2U / pub["L2u"][k] - 1) < 0.003, (N, L2U)
        assert asym < pub["xy_symmetry_max"]
        assert r["nprimfail"] == 0


def test_gubser_convergence_order(gubser_runs):
    Ns = sorted(gubser_runs)
    oT = math.log2(gubser_runs[Ns[0]][0] / gubser_runs[Ns[1]][0])
    oU = math.log2(gubser_runs[Ns[0]][1] / gubser_runs[Ns[1]][1])
    assert abs(oT - GATES["gubser"]["order_T"][0]) < 0.02
    assert abs(oU - GATES["gubser"]["order_u"][0]) < 0.02


# ------------------------------------------------------------------ Bjorken G0

def bjorken_exact(params, T0, mu0, tau0, tau):
    """test/test_bjorken2d.jl:65-90: T from tau*s = const, mu from tau*n = const."""
    P0, n0, e0 = (v[0] for v in O.eos_Pne(params, np.array([T0]), np.array([mu0])))
    star = (e0 + P0) / T0 * tau0 / tau
    ntar = n0 * tau0 / tau
    lo, hi = 1e-4, 5.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        P, n, e = (v[0] for v in O.eos_Pne(params, np.array([mid]), np.array([mu0])))
        if (e + P) / mid > star:
            hi = mid
        else:
            lo = mid
    T = 0.5 * (lo + hi)
    mlo, mhi = -40.0, 40.0
    for _ in range(200):
        mid = 0.5 * (mlo + mhi)
        nm = O.eos_Pne(params, np.array([T]), np.array([mid]))[1][0]
        if nm > ntar:
            mhi = mid
        else:
            mlo = mid
    mu = 0.5 * (mlo + mhi)
    P, n, e = (v[0] for v in O.eos_Pne(params, np.array([T]), np.array([mu])))
    return T, mu, n, e, P


def run_bjorken(cfltau, integrator):
    s = GATES["bjorken"]["settings"]
    g = fivo2d.make_grid2d(s["N"], s["N"], xmax=s["box"], ymax=s["box"])
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS())
    T, a, ux, uy = ic.uniform_fields(g, T0=s["T0"], alpha0=s["alpha0"])
    U, ok = O.set_cells(m.params, s["tau0"], T, a, ux, uy, m.nv)
    assert ok.all()
    o = O.OracleSolver(m, g)
    o.set_state(U)
    o.finalize_ic(s["tau0"])
    U0 = o.get_state()
    r = o.run(s["tau0"], s["tauf"], s["CFL"], cfltau, integrator)
    assert r["ok"]
    U1 = o.get_state()
    pr = o.primitives()
    sx, sy = g.interior()
    Ui = U1.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy]
    D0 = U0.reshape(g.Nxtot, g.Nytot, m.nv)[sx, sy, 0]
    drift = float(np.max(np.abs(Ui[..., 0] - D0) / np.abs(D0)))
    maxu = max(float(np.max(np.abs(pr["ux"]))), float(np.max(np.abs(pr["uy"]))))
    E = Ui[..., 3]
    spread = float((E.max() - E.min()) / abs(E.max()))
    Tx, mux, nx_, ex, Px = bjorken_exact(m.params, s["T0"], s["alpha0"] * s["T0"], s["tau0"], r["tau"])
    ic_ = g.lin(g.nghost + g.Nx // 2 - 1, g.nghost + g.Ny // 2 - 1)
    Eerr = abs(U1[ic_, 3] - ex) / ex
    o.close()
    return dict(r=r, drift=drift, maxu=maxu, spread=spread, Eerr=Eerr)


def test_bjorken_exact_invariants():
    b = run_bjorken(0.02, A.FIVO_SSPRK2)
    assert b["r"]["nprimfail"] == 0
    assert b["drift"] < GATES["bjorken"]["drift_max"]
    assert b["maxu"] == 0.0
    assert b["spread"] < GATES["bjorken"]["E_spread_max"]


def test_bjorken_energy_vs_exact():
    b = run_bjorken(0.005, A.FIVO_SSPRK2)
    assert b["Eerr"] < GATES["bjorken"]["err_max_at_cfltau_0.005"]


@pytest.mark.parametrize("integrator,expect", [(A.FIVO_SSPRK2, "ssprk2"), (A.FIVO_SSPRK3, "ssprk3")])
def test_bjorken_order(integrator, expect):
    errs = [run_bjorken(c, integrator)["Eerr"] for c in (0.02, 0.01, 0.005)]
    p2 = math.log2(errs[1] / errs[2])
    pub = GATES["bjorken"]["order"][expect]
    assert abs(p2 - pub) < 0.15, (errs, p2)


# ------------------------------------------------------------------ recovery

def _random_states(eos, n, diss, umax, rng, tau):
    m = fivo2d.build_model_2d(eos=eos, enable_shear=True, enable_bulk=True)
    T = 0.12 + 0.43 * rng.random(n)
    phi = 4.0 * (2 * rng.random(n) - 1)
    ux = umax * (2 * rng.random(n) - 1)
    uy = umax * (2 * rng.random(n) - 1)
    P, nq, _ = O.eos_Pne(m.params, T, eos.m_hq + T * phi)
    Pi, pxx, pxy, pyy = (diss * P * (2 * rng.random(n) - 1) for _ in range(4))
    nux, nuy = (diss * nq * (2 * rng.random(n) - 1) for _ in range(2))
    U, ok = O.set_cells(m.params, tau, T, (eos.m_hq + T * phi) / T, ux, uy, m.nv, Pi, pxx, pxy, pyy, nux, nuy)
    cons = np.column_stack([U[:, 0] / tau] + [U[:, k] for k in range(1, 11)])
    return m, cons, T, eos.m_hq + T * phi, ux, uy


@pytest.mark.parametrize("eos", [fivo2d.ConformalHQEOS(), fivo2d.LatticeHRGEOS()], ids=["conformal", "lhrg"])
@pytest.mark.parametrize("diss,umax", [(0.0, 1.5), (0.1, 1.5), (0.1, 4.0)])
def test_primrec_roundtrip(eos, diss, umax):
    """prim -> cons -> prim, 1500 seeded states, 0 failures, 1e-9
    (test/test_primrec2d.jl:59-99). Seeds: numpy PCG64, not Julia's MT."""
    rng = np.random.default_rng(20260901)
    tau = 0.4 + 12 * rng.random()
    m, cons, T, mu, ux, uy = _random_states(eos, GATES["primrec"]["ntrial"], diss, umax, rng, tau)
    prim, ok, reason = O.cons_to_prim(m.params, tau, cons)
    tol = GATES["primrec"]["tol"]
    assert ok.all()
    assert np.max(np.abs(prim[:, 0] - T) / T) < tol
    assert np.max(np.maximum(np.abs(prim[:, 2] - ux), np.abs(prim[:, 3] - uy)) /
                  np.maximum(1.0, np.maximum(np.abs(ux), np.abs(uy)))) < tol
    assert np.max(np.abs(prim[:, 1] - mu) / np.maximum(np.abs(mu), 1e-3)) < tol


def test_primrec_y_symmetric_and_tilt():
    """test/test_primrec2d.jl:121-166: u^y = 0 states recover |u^y| < 1e-12; the
    shear genuinely tilts S away from u."""
    eos = fivo2d.LatticeHRGEOS()
    rng = np.random.default_rng(5)
    m = fivo2d.build_model_2d(eos=eos, enable_shear=True, enable_bulk=True)
    n = 1500
    T = 0.12 + 0.43 * rng.random(n)
    phi = 4.0 * (2 * rng.random(n) - 1)
    ux = 1.5 * (2 * rng.random(n) - 1)
    P, nq, _ = O.eos_Pne(m.params, T, eos.m_hq + T * phi)
    Pi, pxx, pyy = (0.1 * P * (2 * rng.random(n) - 1) for _ in range(3))
    nux = 0.1 * nq * (2 * rng.random(n) - 1)
    z = np.zeros(n)
    U, ok = O.set_cells(m.params, 1.0, T, (eos.m_hq + T * phi) / T, ux, z, m.nv, Pi, pxx, z, pyy, nux, z)
    cons = np.column_stack([U[:, 0]] + [U[:, k] for k in range(1, 11)])
    prim, okr, _ = O.cons_to_prim(m.params, 1.0, cons)
    assert np.max(np.abs(prim[okr, 3])) < GATES["primrec"]["y_symmetric_uy"]
    uy = 1.5 * (2 * rng.random(n) - 1)
    pxy = 0.1 * P * (2 * rng.random(n) - 1)
    U, ok = O.set_cells(m.params, 1.0, T, (eos.m_hq + T * phi) / T, ux, uy, m.nv, Pi, pxx, pxy, pyy, nux, z)
    Sx, Sy = U[:, 1], U[:, 2]
    cosang = np.clip((Sx * ux + Sy * uy) / (np.hypot(Sx, Sy) * np.hypot(ux, uy)), -1, 1)
    assert np.max(np.arccos(cosang)) > GATES["primrec"]["tilt_min_rad"]


def test_primrec_vacuum_and_zero_flow():
    eos = fivo2d.LatticeHRGEOS()
    m = fivo2d.build_model_2d(eos=eos)
    cons = np.zeros((2, 11))
    U, ok = O.set_cells(m.params, 1.0, np.array([0.30]), np.array([eos.m_hq / 0.30]), np.zeros(1), np.zeros(1), m.nv)
    cons[1, :4] = U[0, :4]
    prim, ok, reason = O.cons_to_prim(m.params, 1.0, cons)
    assert not ok[0] and reason[0] == 1 and np.all(np.isfinite(prim[0]))
    assert ok[1]
    assert abs(prim[1, 0] - 0.30) / 0.30 < GATES["primrec"]["zero_flow_T"]
    assert np.hypot(prim[1, 2], prim[1, 3]) < GATES["primrec"]["zero_flow_u"]
