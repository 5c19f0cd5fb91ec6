"""The freeze-out surface and Cooper-Frye yield on the CPU: the radial-profile
loader against its definition (src/io.jl:51-260, src/utils.jl:27-29), the oracle's
pion_yield (freezeout2d.jl:144-190) against an independent numpy evaluation of
the same sum, and the oracle's surface recorder (freezeout2d.jl:94-115) on a
short axisymmetric run."""
import ctypes as C
import math
import pathlib

import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d.freezeout import axisym_fields, freeze_model, load_initial_interpolants, smoothstep01_5

PROFILE = pathlib.Path(__file__).resolve().parent / "golden" / "initial_profiles_physical.csv"
PRM = dict(T_fo=0.156, m=0.138, pt_lo=0.1, pt_hi=5.0, eta_max=6.0, f_yield=5.0, n_eta=40, n_pt=40, n_phi=24)


def test_smoothstep_and_loader():
    assert smoothstep01_5(-1) == 0.0 and smoothstep01_5(2) == 1.0 and smoothstep01_5(0.5) == 0.5
    data = np.loadtxt(PROFILE, delimiter=",", skiprows=1)
    itpT, itpF, rmax = load_initial_interpolants(PROFILE)
    assert rmax == data[:, 0].max()
    for r, T, a in data[100:700:50]:
        if r >= 0 and r < rmax - 1.0:
            assert itpT(r) == max(T, 1e-20) and itpF(r) == a
    assert itpT(rmax + 0.5) == 1e-20 and itpF(rmax + 0.5) == 0.0
    # inside the taper: between the profile and the floor
    r = rmax - 0.5
    assert 1e-20 < itpT(r) < np.interp(r, data[:, 0], data[:, 1])


def pion_yield_numpy(tau_fo, uxf, uyf, dx, p):
    """the same sum, vectorised over (p_T, phi, eta) per cell"""
    nx, ny = tau_fo.shape
    pt = p["pt_lo"] + np.arange(p["n_pt"]) * ((p["pt_hi"] - p["pt_lo"]) / (p["n_pt"] - 1))
    phi = np.arange(p["n_phi"]) * (2 * math.pi / p["n_phi"])
    eta = -p["eta_max"] + np.arange(p["n_eta"]) * (2 * p["eta_max"] / (p["n_eta"] - 1))
    dpt, dphi, deta = pt[1] - pt[0], 2 * math.pi / p["n_phi"], eta[1] - eta[0]
    PT, PHI, ETA = np.meshgrid(pt, phi, eta, indexing="ij")
    mT = np.sqrt(PT * PT + p["m"] ** 2)
    px, py, ch = PT * np.cos(PHI), PT * np.sin(PHI), np.cosh(ETA)

    def g1(a, b, d):
        lo = tau_fo[a - 1, b] if d == 1 else tau_fo[a, b - 1]
        hi = tau_fo[a + 1, b] if d == 1 else tau_fo[a, b + 1]
        c = tau_fo[a, b]
        if not np.isnan(lo) and not np.isnan(hi):
            return (hi - lo) / (2 * dx)
        if not np.isnan(hi):
            return (hi - c) / dx
        if not np.isnan(lo):
            return (c - lo) / dx
        return math.nan
    tot = totB = neg = pos = 0.0
    for a in range(1, nx - 1):
        for b in range(1, ny - 1):
            if np.isnan(tau_fo[a, b]):
                continue
            gx, gy = g1(a, b, 1), g1(a, b, 2)
            if np.isnan(gx) or np.isnan(gy):
                continue
            ux, uy = uxf[a, b], uyf[a, b]
            ut = math.sqrt(1 + ux * ux + uy * uy)
            dSp = tau_fo[a, b] * (mT * ch - gx * px - gy * py)
            x = (ut * mT * ch - ux * px - uy * py) / p["T_fo"]
            w = dSp * PT * dpt * dphi * deta * dx * dx
            fB = np.exp(-x)
            with np.errstate(over="ignore"):
                fb = np.where(x > 1e-8, 1 / np.expm1(np.maximum(x, 1e-300)), 0.0)
            tot += float(np.sum(w * fB))
            totB += float(np.sum(w * fb))
            neg += float(np.sum(np.where(dSp < 0, -w * fB, 0.0)))
            pos += float(np.sum(np.where(dSp < 0, 0.0, w * fB)))
    pref = p["f_yield"] / (2 * math.pi * 0.1973269804) ** 3
    return pref * tot, pref * totB, neg / max(pos + neg, 1e-30)


def oracle_pion_yield(tau_fo, uxf, uyf, dx, p):
    nx, ny = tau_fo.shape
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (tau_fo, uxf, uyf)]
    prm = np.array([p["T_fo"], p["m"], p["pt_lo"], p["pt_hi"], p["eta_max"], p["f_yield"]])
    ng = (C.c_int * 3)(p["n_eta"], p["n_pt"], p["n_phi"])
    out = np.zeros(3)
    O.lib().oracle_pion_yield(nx, ny, dx, *[O._ptr(a) for a in arrs], O._ptr(prm), ng, O._ptr(out))
    return tuple(out)


def synthetic_surface(n=14, seed=3):
    """a dome tau_fo = 8 - 0.05 r^2 with outward flow, a ring of never-frozen cells
    and a few holes"""
    rng = np.random.default_rng(seed)
    x = (np.arange(n) - (n - 1) / 2) * 1.0
    X, Y = np.meshgrid(x, x, indexing="ij")
    tau = 8.0 - 0.05 * (X * X + Y * Y)
    tau[np.hypot(X, Y) > 0.45 * n] = np.nan
    tau[rng.random(tau.shape) < 0.04] = np.nan
    return tau, 0.08 * X, 0.08 * Y


def test_oracle_pion_yield_matches_numpy():
    tau, ux, uy = synthetic_surface()
    p = dict(PRM, n_eta=12, n_pt=10, n_phi=8)
    a = oracle_pion_yield(tau, ux, uy, 1.0, p)
    b = pion_yield_numpy(tau, ux, uy, 1.0, p)
    assert a[0] > 0 and a[1] > a[0]              # Bose above Boltzmann for pions
    for u, v in zip(a, b):
        assert abs(u - v) <= 1e-11 * max(abs(v), 1e-30), (a, b)


def oracle_freeze_surface(m, g, U, tau0, tau_max, dtau=0.02, cfl=0.15, cfltau=0.05, T_fo=0.156):
    o = O.OracleSolver(m, g)
    o.set_state(U)
    o.finalize_ic(tau0)
    n = g.Nx * g.Ny
    tau_fo, uxf, uyf = np.full(n, np.nan), np.zeros(n), np.zeros(n)
    Tprev, above = np.full(n, np.nan), np.zeros(n, dtype=np.uint8)
    refroze = C.c_int64(0)

    def record(tau, tau_prev):
        O.lib().oracle_fo_record(o.h, tau, tau_prev, T_fo, *[O._ptr(a) for a in (tau_fo, uxf, uyf, Tprev)],
                                 O._ptr(above), C.byref(refroze))
    o.rhs(tau0)
    record(tau0, tau0)
    tau = tau0
    while tau < tau_max - 1e-9:
        r = o.run(tau, min(tau + dtau, tau_max), cfl, cfltau, A.FIVO_SSPRK2, reset_history=False)
        assert r["ok"]
        prev, tau = tau, r["tau"]
        o.update_primitives(tau)
        record(tau, prev)
    o.close()
    shape = (g.Nx, g.Ny)
    return dict(tau_fo=tau_fo.reshape(shape), uxf=uxf.reshape(shape), uyf=uyf.reshape(shape),
                nhot=int(above.sum()), nfroze=int((~np.isnan(tau_fo)).sum()), refroze=int(refroze.value))


def small_control():
    g = fivo2d.make_grid2d(24, 24, xmax=18.0, ymax=18.0)
    m = freeze_model()
    T, a, ux, uy = axisym_fields(g, PROFILE)
    U, ok = O.set_cells(m.params, 0.4, T, a, ux, uy, m.nv)
    return g, m, U


SHORT = dict(tau_max=3.0, T_fo=0.30)   # a high isotherm, so that a short run freezes most hot cells


def test_oracle_surface_on_a_short_run():
    g, m, U = small_control()
    s = oracle_freeze_surface(m, g, U, 0.4, SHORT["tau_max"], T_fo=SHORT["T_fo"])
    fro = ~np.isnan(s["tau_fo"])
    assert s["nhot"] > 0 and s["nfroze"] == int(fro.sum()) and s["nhot"] // 2 < s["nfroze"] <= s["nhot"]
    assert np.all((s["tau_fo"][fro] >= 0.4) & (s["tau_fo"][fro] <= SHORT["tau_max"]))
    # the surface is symmetric under x <-> y like the initial profile
    t = np.where(fro, s["tau_fo"], -1.0)
    assert np.allclose(t, t.T, rtol=0, atol=1e-12)
