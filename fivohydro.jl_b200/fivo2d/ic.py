"""Initial-condition fields for the 2+1D stage.

Each builder returns per-cell primitive fields (T, alpha = mu/T, u^x, u^y) on all
Ntot cells in flat order (i = ix*Nytot + iy); `set_cells` (the C ABI's
fivo_set_cells, i.e. set_cell!) turns them into conserved variables.

  gubser_*        src/gubser.jl:20-56 (ideal conformal Gubser flow)
  uniform         initialize_uniform!, main2D.jl:174-182 (Bjorken)
  glauber         seeded MC-Glauber event (the reference's builder is not public;
                  this one follows the event description: two Woods-Saxon Pb
                  nuclei, participants by the distance criterion, Gaussian sources
                  with Gamma(1)-distributed weights, charm from binary collisions)
"""
from __future__ import annotations

import math

import numpy as np

from .model import HBARC, T_MIN, Grid2D, LatticeHRGEOS

# ----------------------------------------------------------------------------- Gubser


def posden(x):
    return np.where(x > 1e-50, x, 1e-50)


def gubser_den(tau, r, q):
    q2 = q * q
    return 1.0 + 2.0 * q2 * (tau * tau + r * r) + (q2 * q2) * ((tau * tau - r * r) ** 2)


def gubser_vr(tau, r, q):
    q2 = q * q
    num = 2.0 * q2 * tau * r
    den = 1.0 + q2 * (tau * tau) + q2 * (r * r)
    return num / posden(den)


def gubser_ur(tau, r, q):
    v = np.clip(gubser_vr(tau, r, q), -0.999999999, 0.999999999)
    return v / np.sqrt(1.0 - v * v)


def gubser_temperature(tau, r, q, Tscale):
    Den = gubser_den(tau, r, q)
    qpos = max(abs(q), 1e-50)
    return Tscale * (2.0 * qpos) ** (2 / 3) / (max(tau, 1e-50) ** (1 / 3) * posden(Den) ** (1 / 3))


def gubser_Tscale_from_center_T(tau0, q, Tc0):
    qpos = max(abs(q), 1e-50)
    fac = (max(tau0, 1e-50) ** (1 / 3)) * (1.0 + (qpos * tau0) ** 2) ** (2 / 3)
    return max(Tc0, 1e-50) * fac / (2.0 * qpos) ** (2 / 3)


def gubser_fields(g: Grid2D, tau0: float, *, q: float, Tscale: float, alpha: float):
    """Exact Gubser state on every cell (the loop of test/test_gubser2d.jl:103-109)."""
    X, Y = np.meshgrid(g.xC, g.yC, indexing="ij")
    r = np.hypot(X, Y)
    ur = gubser_ur(tau0, r, q)
    with np.errstate(invalid="ignore", divide="ignore"):
        ux = np.where(r > 0, ur * X / r, 0.0)
        uy = np.where(r > 0, ur * Y / r, 0.0)
    T = gubser_temperature(tau0, r, q, Tscale)
    a = np.full_like(T, alpha)
    return T.ravel(), a.ravel(), ux.ravel(), uy.ravel()


def gubser_exact(g: Grid2D, tau: float, *, q: float, Tscale: float):
    X, Y = np.meshgrid(g.xC, g.yC, indexing="ij")
    r = np.hypot(X, Y)
    T = gubser_temperature(tau, r, q, Tscale)
    ur = gubser_ur(tau, r, q)
    with np.errstate(invalid="ignore", divide="ignore"):
        ux = np.where(r > 0, ur * X / r, 0.0)
        uy = np.where(r > 0, ur * Y / r, 0.0)
    return T, ux, uy, r


# ----------------------------------------------------------------------------- uniform


def uniform_fields(g: Grid2D, *, T0: float = 0.5, alpha0: float = -4.2):
    n = g.Ntot
    return np.full(n, T0), np.full(n, alpha0), np.zeros(n), np.zeros(n)


# ----------------------------------------------------------------------------- MC-Glauber

# Pb-208 Woods-Saxon nuclei of the event-by-event workload
WS_R, WS_A, WS_N = 6.62, 0.546, 208
SIGMA_NN = 6.8          # fm^2
SRC_WIDTH = 0.5         # fm, Gaussian width per participant


def _sample_woods_saxon(rng: np.random.Generator, n: int) -> np.ndarray:
    """n nucleon positions (x, y, z) from rho(r) ~ 1/(1+exp((r-R)/a)) by rejection."""
    out = np.empty((0, 3))
    rmax = WS_R + 10 * WS_A
    while out.shape[0] < n:
        m = 4 * n
        r = rmax * rng.random(m) ** (1 / 3)
        acc = rng.random(m) < 1.0 / (1.0 + np.exp((r - WS_R) / WS_A))
        r = r[acc]
        cth = 2 * rng.random(r.size) - 1
        ph = 2 * np.pi * rng.random(r.size)
        sth = np.sqrt(1 - cth * cth)
        pts = np.stack([r * sth * np.cos(ph), r * sth * np.sin(ph), r * cth], axis=1)
        out = np.concatenate([out, pts])
    return out[:n]


def glauber_event(seed: int, bmax: float = 8.0):
    """One seeded Pb+Pb MC-Glauber event: participant and binary-collision
    positions in the transverse plane, the impact parameter, and Gamma(k=1)
    weights per participant."""
    rng = np.random.default_rng(seed)
    b = bmax * rng.random()
    A = _sample_woods_saxon(rng, WS_N)[:, :2] + np.array([-b / 2, 0.0])
    B = _sample_woods_saxon(rng, WS_N)[:, :2] + np.array([b / 2, 0.0])
    d2 = ((A[:, None, :] - B[None, :, :]) ** 2).sum(-1)
    hit = d2 <= SIGMA_NN / np.pi
    partA = hit.any(1)
    partB = hit.any(0)
    parts = np.concatenate([A[partA], B[partB]])
    ia, ib = np.nonzero(hit)
    binary = 0.5 * (A[ia] + B[ib])
    w = rng.gamma(1.0, 1.0, parts.shape[0])
    return dict(b=b, participants=parts, weights=w, binary=binary)


def _deposit(X, Y, pts, w, width):
    out = np.zeros_like(X)
    inv = 1.0 / (2 * width * width)
    norm = 1.0 / (2 * np.pi * width * width)
    for (px, py), wk in zip(pts, w):
        out += wk * norm * np.exp(-((X - px) ** 2 + (Y - py) ** 2) * inv)
    return out


def _lhrg_e_of_T(T, eos: LatticeHRGEOS):
    """Light-sector energy density e = -P + T dP/dT of the LatticeHRG fit
    (src/eos.jl:357-412) in numpy; used only to invert e(T) for the IC."""
    fm3 = (1.0 / HBARC) ** 3
    k0, k1, k2, k3, k4 = 0.0005624486560000001, 0.003652264, 0.023716, 0.154, 5.208957878352717
    T = np.maximum(T, T_MIN)
    A = 0.01 * eos.d ** 2
    B = 0.1 * eos.c ** 2
    E = np.clip(-(A / (T * T)) - (B / T), -700, 700)
    eE = np.exp(E)
    N = k0 * eos.a4 + k1 * eos.a3 * T + k2 * eos.a2 * T ** 2 + k3 * eos.a1 * T ** 3 + k4 * T ** 4
    D = k0 * eos.b4 + k1 * eos.b3 * T + k2 * eos.b2 * T ** 2 + k3 * eos.b1 * T ** 3 + T ** 4
    Np = k1 * eos.a3 + 2 * k2 * eos.a2 * T + 3 * k3 * eos.a1 * T ** 2 + 4 * k4 * T ** 3
    Dp = k1 * eos.b3 + 2 * k2 * eos.b2 * T + 3 * k3 * eos.b1 * T ** 2 + 4 * T ** 3
    Ep = 2 * A / T ** 3 + B / T ** 2
    G = T ** 4 * N
    Gp = 4 * T ** 3 * N + T ** 4 * Np
    F = G / D
    Fp = (Gp * D - G * Dp) / (D * D)
    P = fm3 * eE * F
    dP = fm3 * eE * (Fp + F * Ep)
    return -P + T * dP


def _lhrg_n_alpha0(T, eos: LatticeHRGEOS):
    """Charm density n(T, alpha = 0) of LatticeHRGEOS (src/eos.jl:483-519)."""
    from scipy.special import kve
    fm3 = (1.0 / HBARC) ** 3
    m = eos.m_hq
    x = np.minimum(m / np.maximum(T, T_MIN), 1e5)
    A = eos.canon_factor * eos.g_hq * m * m / (2 * np.pi ** 2)
    z = np.clip((0.0 - m) / np.maximum(T, T_MIN), -700, 700)
    n = A * T * np.exp(z) * kve(2, x)
    return n * fm3 if eos.hq_times_fmGeV3 else n


def invert_e_for_T(e, eos: LatticeHRGEOS, iters: int = 90):
    lo = np.full_like(e, math.log(T_MIN))
    hi = np.full_like(e, math.log(10.0))
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        em = _lhrg_e_of_T(np.exp(mid), eos)
        big = em > e
        hi = np.where(big, mid, hi)
        lo = np.where(big, lo, mid)
    return np.exp(0.5 * (lo + hi))


# The edge state of the reference's production radial profile (the last row of
# data/initial_profiles_physical.csv: T0 = 0.1278551418360245 GeV, alpha0 =
# 1.8877972332059278). The reference's floors and vacuum cut were tuned against a
# profile that carries this edge (examples2d/04_fluctuating_event.jl:16-31), so the
# event is laid on it: the medium never reaches vacuum and every cell carries charm.
EDGE_T = 0.1278551418360245
EDGE_ALPHA = 1.8877972332059278


def glauber_fields(g: Grid2D, tau0: float, seed: int, *, eos: LatticeHRGEOS | None = None,
                   Tpeak: float = 0.450, ncharm: float = 10.0, bmax: float = 8.0,
                   alpha_min: float = -20.0, T_edge: float = EDGE_T, alpha_edge: float = EDGE_ALPHA):
    """MC-Glauber-like IC on every cell: energy density from the participants, on top
    of the edge state's energy density e(T_edge) and scaled so the peak is T = Tpeak,
    T from the EOS inverse; charm density = n(T_edge, alpha_edge) + a part
    proportional to the binary-collision density with tau0 * sum(n u^tau) dx dy =
    ncharm; alpha = log(n / n(T, alpha=0)); u = 0. T_edge <= 0 builds the event on
    vacuum instead (no edge state; alpha floored at alpha_min where there is no charm)."""
    eos = eos or LatticeHRGEOS()
    ev = glauber_event(seed, bmax)
    X, Y = np.meshgrid(g.xC, g.yC, indexing="ij")
    s = _deposit(X, Y, ev["participants"], ev["weights"], SRC_WIDTH)
    e_peak = float(_lhrg_e_of_T(np.array([Tpeak]), eos)[0])
    edge = T_edge > 0
    e_edge = float(_lhrg_e_of_T(np.array([T_edge]), eos)[0]) if edge else 0.0
    e = s * ((e_peak - e_edge) / s.max()) + e_edge
    T = np.maximum(invert_e_for_T(e, eos), T_MIN)
    nb = _deposit(X, Y, ev["binary"], np.ones(len(ev["binary"])), SRC_WIDTH)
    ng = g.nghost
    interior = nb[ng:ng + g.Nx, ng:ng + g.Ny].sum() * g.dx * g.dy
    n_tgt = nb * (ncharm / (tau0 * interior)) if interior > 0 else nb * 0.0
    if edge:
        n_tgt = n_tgt + float(_lhrg_n_alpha0(np.array([T_edge]), eos)[0]) * math.exp(alpha_edge)
    with np.errstate(divide="ignore", invalid="ignore"):
        n0 = _lhrg_n_alpha0(T, eos)
        a = np.log(n_tgt / n0)
    a = np.where(np.isfinite(a), np.maximum(a, alpha_min), alpha_min)
    z = np.zeros_like(T)
    return T.ravel(), a.ravel(), z.ravel(), z.ravel().copy(), ev
