"""The consistent charm first moment (consistent_fm) in the oracle, pinned to the
reference's gate Gc (test/test_consistent_fm2d.jl):

  Gc1  the 1-D limit: with u^y = 0 and d_y = 0 the 2-D source equals the 1-D
       radial one (src/hq_consistent_firstmoment.jl, hq_consistent_extras, its
       all-on expression restated below) to 1e-12            (:77-128)
  Gc2  the source is a transverse vector: rotating the state rotates it (:133-177)
  Gc3  Bjorken limit: at rest, no gradients, s = tau_n nu / tau   (:182-207)
  Gc4  zero current and zero gradients give exactly zero          (:212-220)
  Gc5  consistent_fm moves a solve with a transverse gradient; off is the
       shipped path                                                (:225-257)
  Gc6  tauN_coeff != 1 is refused with the closure on, allowed off (:262-289)
  Gc7  the sign on a solve: a uniform Bjorken nu^x follows
       tau_n dnu/dtau = -(1 + b) nu and not the flipped ODE        (:294-339)

plus the closed forms h' and dn/dT (src2d/hq_consistent_firstmoment2d.jl:145-182)
against finite differences of h = m K3/K2 and of the heavy-quark density.
"""
import math

import numpy as np
import pytest

import _oracle as O
import fivo2d
from fivo2d import _abi as A
from fivo2d import ic

FMGEV = 1.0 / 0.1973269804                      # 1 fm in GeV^-1 (hbar c = 0.1973269804 GeV fm)
ALL_FM = sum(A.TERM_BIT[n] for n in ("fm_gradT", "fm_inertial", "fm_nu_gradu", "fm_expansion", "fm_dlnh"))


def source(ux, uy, ut, T, dxT, dyT, dtT, nux, nuy, n, dn_dT, tn, Ds, hp, th, ax, ay, dxux, dxuy, dyux, dyuy,
           terms=ALL_FM):
    v = np.array([ux, uy, ut, T, dxT, dyT, dtT, nux, nuy, n, dn_dT, tn, Ds, hp, th, ax, ay, dxux, dxuy, dyux,
                  dyuy], dtype=np.float64)
    sx, sy = np.zeros(1), np.zeros(1)
    O.lib().oracle_cfm_source(O._ptr(v), terms, O._ptr(sx), O._ptr(sy))
    return float(sx[0]), float(sy[0])


def extras_1d(tau, r, ur, T, dtT, drT, drur, dtur, n, dn_dT, nu, tn, Ds, h, hp):
    """hq_consistent_extras with every term on (src/hq_consistent_firstmoment.jl:88-101)."""
    ut = math.sqrt(1.0 + ur * ur)
    ex = (Ds / T) * (drur * h * n * ur + dtur * h * n * ut + dtT * n * ur * ut + dtT * dn_dT * T * ur * ut
                     + drT * (n + dn_dT * T) * ut * ut)
    ex += (Ds / T) * nu * (2.0 * drur * h + drT * hp * ur + (2.0 * dtur * h * ur + dtT * hp * ut * ut) / ut)
    ex += tn * nu * (ut / tau + ur / r)
    return ex


GC1_POINTS = [
    dict(tau=2.3, r=3.1, ur=0.42, T=0.31, dtT=-0.055, drT=-0.021, drur=0.13, dtur=0.07, n=0.9, dn_dT=1.7,
         nu=0.031, Ds=0.44, h=2.20, hp=-0.9),
    dict(tau=1.1, r=0.7, ur=-0.30, T=0.45, dtT=-0.120, drT=0.033, drur=-0.21, dtur=0.15, n=1.4, dn_dT=2.9,
         nu=-0.070, Ds=0.30, h=1.90, hp=-1.4),
    dict(tau=5.0, r=8.0, ur=0.90, T=0.20, dtT=-0.010, drT=-0.005, drur=0.02, dtur=0.01, n=0.3, dn_dT=0.8,
         nu=0.010, Ds=0.60, h=2.60, hp=-0.5),
    dict(tau=0.6, r=0.05, ur=-1.30, T=0.55, dtT=0.300, drT=-0.440, drur=0.55, dtur=-0.62, n=2.2, dn_dT=4.1,
         nu=0.190, Ds=0.12, h=1.75, hp=-2.2),
    dict(tau=3.7, r=12.0, ur=0.05, T=0.16, dtT=-0.002, drT=-0.0007, drur=0.004, dtur=0.002, n=0.05,
         dn_dT=0.3, nu=1e-4, Ds=0.80, h=3.10, hp=-0.2),
]


@pytest.mark.parametrize("p", GC1_POINTS, ids=[f"r{p['r']}" for p in GC1_POINTS])
def test_gc1_one_dimensional_limit(p):
    tn = p["Ds"] * p["h"] / p["T"]                    # the tie tau_n = D_s h / T
    ref = extras_1d(p["tau"], p["r"], p["ur"], p["T"], p["dtT"], p["drT"], p["drur"], p["dtur"], p["n"],
                    p["dn_dT"], p["nu"], tn, p["Ds"], p["h"], p["hp"])
    ur = p["ur"]
    ut = math.sqrt(1 + ur * ur)
    ax = ut * p["dtur"] + ur * p["drur"]
    dyuy = ur / p["r"]                                # the phi-direction divergence on the +x axis
    th = ur * p["dtur"] / ut + p["drur"] + dyuy + ut / p["tau"]
    sx, sy = source(ur, 0.0, ut, p["T"], p["drT"], 0.0, p["dtT"], p["nu"], 0.0, p["n"], p["dn_dT"], tn, p["Ds"],
                    p["hp"], th, ax, 0.0, p["drur"], 0.0, 0.0, dyuy)
    assert abs(sx - ref) / max(abs(ref), 1e-300) < 1e-12
    assert abs(sy) < 1e-14 * max(abs(sx), 1.0)


def test_gc2_rotational_invariance():
    ux, uy = 0.31, -0.22
    ut = math.sqrt(1 + ux * ux + uy * uy)
    nux, nuy = 0.017, 0.009
    dxT, dyT = -0.03, 0.012
    G = np.array([[0.11, -0.07], [0.05, 0.09]])       # G[i, j] = d_i u^j
    tau, T, dtT, n, dn_dT, tn, Ds, hp = 2.0, 0.28, -0.04, 1.1, 2.0, 0.55, 0.35, -1.0
    dtut = 0.02
    th = dtut + (G[0, 0] + G[1, 1]) + ut / tau
    a = np.array([ut * 0.03 + ux * G[0, 0] + uy * G[1, 0], ut * 0.01 + ux * G[0, 1] + uy * G[1, 1]])
    s0 = np.array(source(ux, uy, ut, T, dxT, dyT, dtT, nux, nuy, n, dn_dT, tn, Ds, hp, th, a[0], a[1],
                         G[0, 0], G[0, 1], G[1, 0], G[1, 1]))
    worst = 0.0
    for phi in (0.3, 1.0, 2.4, -0.8):
        c, s = math.cos(phi), math.sin(phi)
        R = np.array([[c, -s], [s, c]])
        u2, nu2, gT2, a2 = R @ [ux, uy], R @ [nux, nuy], R @ [dxT, dyT], R @ a
        G2 = R @ G @ R.T
        th2 = dtut + (G2[0, 0] + G2[1, 1]) + ut / tau
        s2 = np.array(source(u2[0], u2[1], ut, T, gT2[0], gT2[1], dtT, nu2[0], nu2[1], n, dn_dT, tn, Ds, hp, th2,
                             a2[0], a2[1], G2[0, 0], G2[0, 1], G2[1, 0], G2[1, 1]))
        worst = max(worst, float(np.max(np.abs(s2 - R @ s0))) / max(math.hypot(*s0), 1e-300))
    assert worst < 1e-12


def test_gc3_bjorken_limit():
    tau, T, n, tn, Ds, hp = 3.0, 0.30, 1.0, 0.7, 0.4, -1.0
    nux, nuy = 0.02, -0.013
    sx, sy = source(0.0, 0.0, 1.0, T, 0.0, 0.0, 0.0, nux, nuy, n, 0.0, tn, Ds, hp, 1.0 / tau, 0, 0, 0, 0, 0, 0)
    ex, ey = tn * nux / tau, tn * nuy / tau
    assert abs(sx - ex) <= 1e-13 * abs(ex) and abs(sy - ey) <= 1e-13 * abs(ey)


def test_gc4_no_current_no_gradients_no_source():
    sx, sy = source(0.0, 0.0, 1.0, 0.30, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 2.0, 0.7, 0.4, -1.0, 1.0 / 3.0,
                    0, 0, 0, 0, 0, 0)
    assert sx == 0.0 and sy == 0.0


def test_terms_switch_each_source():
    """Each fm_* switch removes its own piece; the pieces add up to the all-on value
    up to rounding (the sum is formed in one order only)."""
    args = (0.31, -0.22, math.sqrt(1 + 0.31 ** 2 + 0.22 ** 2), 0.28, -0.03, 0.012, -0.04, 0.017, 0.009, 1.1,
            2.0, 0.55, 0.35, -1.0, 0.9, 0.05, -0.02, 0.11, -0.07, 0.05, 0.09)
    full = np.array(source(*args))
    assert np.all(np.array(source(*args, terms=0)) == 0.0)
    parts = sum(np.array(source(*args, terms=A.TERM_BIT[n]))
                for n in ("fm_gradT", "fm_inertial", "fm_nu_gradu", "fm_expansion", "fm_dlnh"))
    assert np.allclose(parts, full, rtol=1e-13, atol=0)


def _hq_params():
    return fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.1163,
                                 consistent_fm=True).params


@pytest.mark.parametrize("T", [0.12, 0.2, 0.3, 0.45, 0.6])
def test_h_hprime_and_dn_dT_closed_forms(T):
    """h = m K3(z)/K2(z) and its T-derivative; dn/dT at fixed alpha for n ~ T^3 z^2 K2(z)
    (src2d/hq_consistent_firstmoment2d.jl:145-182), against central differences."""
    p = _hq_params()
    m = p.m_hq

    def h_of(TT):
        z = m / TT
        return m * O.besselkx(3, np.array([z]))[0] / O.besselkx(2, np.array([z]))[0]

    def dens(TT):                                     # Boltzmann heavy-quark density at fixed alpha, any prefactor
        z = m / TT
        return TT ** 3 * z * z * O.besselkx(2, np.array([z]))[0] * math.exp(-z)

    h, hp = np.zeros(1), np.zeros(1)
    O.lib().oracle_cfm_h_hprime(C_params(p), T, O._ptr(h), O._ptr(hp))
    d = 1e-5 * T
    assert abs(h[0] - h_of(T)) <= 1e-14 * h_of(T)
    assert abs(hp[0] - (h_of(T + d) - h_of(T - d)) / (2 * d)) < 1e-7 * abs(hp[0])
    n = 0.37
    dndT = O.lib().oracle_cfm_dn_dT(C_params(p), T, n)
    fd = n * (dens(T + d) - dens(T - d)) / (2 * d) / dens(T)
    assert abs(dndT - fd) < 1e-7 * abs(dndT)


def C_params(p):
    import ctypes
    return ctypes.byref(p)


def test_gc5_flag_moves_a_solve_with_a_gradient():
    def run(cfm):
        g = fivo2d.make_grid2d(48, 48, xmax=6.0, ymax=6.0)
        m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.2,
                                  consistent_fm=cfm)
        U = gc5_state(g, m)
        o = O.OracleSolver(m, g)
        o.set_state(U)
        r = o.run(0.4, 0.6, 0.2, 0.05, A.FIVO_SSPRK2)
        assert r["ok"]
        out = o.get_state()
        o.close()
        return out
    a, b, c = run(False), run(False), run(True)
    assert np.array_equal(a, b)
    assert np.max(np.abs(c - a)) > 0


def gc5_state(g, m, tau0=0.4):
    """initialize_uniform! at T0 = 0.40, alpha0 = -4.2 (main2D.jl:174-182), then a Gaussian
    bump of 10 % in tau*T^tautau on the interior (test/test_consistent_fm2d.jl:230-238)."""
    T, a, ux, uy = ic.uniform_fields(g, T0=0.40, alpha0=-4.2)
    U, ok = O.set_cells(m.params, tau0, T, a, ux, uy, m.nv)
    assert ok.all()
    o = O.OracleSolver(m, g)
    o.set_state(U)
    o.finalize_ic(tau0)
    U = o.get_state()
    o.close()
    X, Y = np.meshgrid(g.xC, g.yC, indexing="ij")
    bump = 1 + 0.10 * np.exp(-(X ** 2 + Y ** 2) / 8)
    V = U.reshape(g.Nxtot, g.Nytot, m.nv)
    sx, sy = g.interior()
    V[sx, sy, 0] *= bump[sx, sy]
    return U


def test_gc6_tauN_coeff_refused_with_the_closure():
    with pytest.raises(ValueError):
        fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.1163,
                              consistent_fm=True, tauN_coeff=1.5)
    fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.1163, consistent_fm=False,
                          tauN_coeff=1.5)
    # the oracle refuses the same combination on its own
    p = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=0.1163,
                              consistent_fm=True).params
    p.tauN_coeff = 1.5
    assert not O.lib().oracle_ctx_create(C_params(p), 16, 16, 3, 4.0, 4.0)


GC7 = dict(T0=0.40, A0=-4.2, TAU0=0.4, TAU1=1.2, DST=0.1163, N=16, box=4.0, cfltau=0.005)


def gc7_setup():
    s = GC7
    g = fivo2d.make_grid2d(s["N"], s["N"], xmax=s["box"], ymax=s["box"])
    m = fivo2d.build_model_2d(eos=fivo2d.LatticeHRGEOS(), enable_diff=True, kappa_coeff=s["DST"],
                              consistent_fm=True)
    _, n0, _ = (v[0] for v in O.eos_Pne(m.params, np.array([s["T0"]]), np.array([s["A0"] * s["T0"]])))
    T, a, ux, uy = ic.uniform_fields(g, T0=s["T0"], alpha0=s["A0"])
    U, ok = O.set_cells(m.params, s["TAU0"], T, a, ux, uy, m.nv, nux=np.full(g.Ntot, 0.05 * n0))
    assert ok.all()
    return g, m, U


def gc7_ode(m, ts, nus, Ts, ns, sgn):
    """Backward Euler of tau_n dnu/dtau = -(1 + sgn b) nu on the solver's own T(tau)
    (test/test_consistent_fm2d.jl:314-328)."""
    s = GC7
    nu = nus[0]
    out = [nu]
    kap, tn, dN = np.zeros(1), np.zeros(1), np.zeros(1)
    h, hp = np.zeros(1), np.zeros(1)
    for k in range(1, len(ts)):
        tau, dtau, T = ts[k - 1], ts[k] - ts[k - 1], Ts[k - 1]
        O.lib().oracle_diff_coeffs(C_params(m.params), T, s["A0"] * T, ns[k - 1], O._ptr(kap), O._ptr(tn),
                                   O._ptr(dN))
        O.lib().oracle_cfm_h_hprime(C_params(m.params), T, O._ptr(h), O._ptr(hp))
        Ds = (s["DST"] / T) / FMGEV
        b = tn[0] / tau + (Ds / T) * hp[0] * (Ts[k] - Ts[k - 1]) / dtau
        nu = (tn[0] / dtau * nu) / (tn[0] / dtau + 1 + sgn * b)
        out.append(nu)
    return np.array(out)


def gc7_trajectory(solver, g, m):
    """run_sim_2d! with a dump every step (main2D.jl:428-515): nu^x, T and n at the
    cell (ng+8, ng+8) (1-based) at tau0 and after each accepted step."""
    s = GC7
    ic_ = g.lin(g.nghost + 7, g.nghost + 7)
    iN = m.layout.idx("nux")
    ts, nus, Ts, ns = [], [], [], []
    solver.rhs(s["TAU0"], A.FIVO_BC_PERIODIC)          # run_sim_2d!'s opening rhs fills the primitives

    def dump(tau):
        pr = solver.primitives()
        ts.append(tau)
        nus.append(solver.get_state()[ic_, iN])
        Ts.append(math.exp(pr["yT"][ic_]))
        ns.append(pr["n"][ic_])
    dump(s["TAU0"])
    tau = s["TAU0"]
    while tau < s["TAU1"]:
        r = solver.advance(tau, s["TAU1"], 0.2, s["cfltau"], A.FIVO_SSPRK2, A.FIVO_BC_PERIODIC, max_steps=1)
        assert r["ok"] and r["nsteps"] == 1
        tau = r["tau"]
        dump(tau)
    return np.array(ts), np.array(nus), np.array(Ts), np.array(ns)


def test_gc7_sign_on_a_solve():
    s = GC7
    g, m, U = gc7_setup()
    o = O.OracleSolver(m, g)
    o.set_state(U)
    o.finalize_ic(s["TAU0"], A.FIVO_BC_PERIODIC)
    ts, nus, Ts, ns = gc7_trajectory(o, g, m)
    o.close()
    phys = gc7_ode(m, ts, nus, Ts, ns, +1.0)
    flip = gc7_ode(m, ts, nus, Ts, ns, -1.0)
    dev_phys = np.max(np.abs(nus - phys)) / abs(nus[0])
    dev_flip = np.max(np.abs(nus - flip)) / abs(nus[0])
    dil = ts[-1] * nus[-1] / (ts[0] * nus[0])
    assert dev_phys < 2e-3, dev_phys
    assert dev_flip > 0.1, dev_flip
    assert dil < 1.0, dil
