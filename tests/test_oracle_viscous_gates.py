"""The oracle's dissipative sectors pinned to the reference's published gates.

The relaxation (bulk, shear, charge diffusion, the DNMR couplings) and the
transport coefficients are checked against the reference's own gate ladder and
its published numbers (README2D.md:273-285, quoted in tests/golden/gates.json):

  G0b  test/test_bjorken_bulk2d.jl       published: T to 1e-4, Pi to 7.5e-3
                                         (0.52 / 0.75 / 0.16 % at zeta/s = 0.05 / 0.15 / 0.30)
  G2   test/test_dissipation2d.jl        published: NS target to 2.4e-15, order 1.05
  G3   test/test_charge2d.jl             published: drift 1.9e-15, 0 of 2104 up-gradient
                                         nu^x, x<->y asymmetry exactly zero
  Gk   test/test_charge_dispersion2d.jl  published: tau_n = D_s z K3/K2 to 1.0000
  Gd   test/test_dnmr2d.jl               published: extrapolated to <= 3e-4 at order
                                         0.97-0.99; wrong-sign referees miss by 5e-3 to 1.7
  G1v  test/test_gubser_viscous2d.jl     published: the ODE reduces to ideal Gubser to 3.6e-11
  Gs   test/test_sound2d.jl              published: c_s to 0.05 %

The long solver ladders (Gk's propagating branch and k_* scan, Gs, G1v's
N = 100/200/400 solver runs) run on the GPU by default (tests/test_gpu_viscous_gates.py,
bitwise the oracle's arithmetic) and on the oracle with FIVO_SLOW=1.
"""
import json
import math
import os
import pathlib

import numpy as np
import pytest
from scipy.special import kve

import _gates as G
import _oracle as O

GATES = json.loads((pathlib.Path(__file__).resolve().parent / "golden" / "gates.json").read_text())
SLOW = bool(os.environ.get("FIVO_SLOW"))
BE = G.OracleBackend()


# ------------------------------------------------------------------ G0b

@pytest.fixture(scope="module")
def g0b():
    return G.gate_g0b(BE)


def test_g0b_bulk_tracer_inversion_is_one_dimensional():
    m = G.g0b_model(0.15)
    P1, n1, e1 = G.eos1(m.params, 0.30, 0.0)
    P2, n2, e2 = G.eos1(m.params, 0.30, -2.0)
    assert abs(P1 - P2) / P1 < 1e-12 and abs(e1 - e2) / e1 < 1e-12


def test_g0b_nonlinear_bulk_vs_ode(g0b):
    pub = GATES["viscous"]["G0b"]
    for row, dPi_pub in zip(g0b["rows"], pub["dPi_production_cfl"]):
        assert row["Tspread"] < 1e-12
        assert row["dT"] < pub["T_tol"]
        assert row["dPi"] < 1e-2
        assert row["PiP"] > 0.05                      # the run is in a bulk regime
        assert abs(row["dPi"] - dPi_pub) < 5e-5, (row, dPi_pub)   # the published per-mille figures


def test_g0b_published_tables(g0b):
    """every entry of the reference's two G0b tables (TWOD_PROGRAM.md:1800-1812), to
    the three printed digits"""
    pub = GATES["viscous"]["G0b"]
    for row, dT, PiP in zip(g0b["rows"], pub["dT_production_cfl"], pub["PiP"]):
        assert abs(row["dT"] / dT - 1) < 6e-3, (row, dT)
        assert abs(row["PiP"] / PiP - 1) < 6e-3, (row, PiP)
    for c, dT, dPi in zip(g0b["conv"], pub["cfl_scan_dT"], pub["cfl_scan_dPi"]):
        assert abs(c["dT"] / dT - 1) < 6e-3, (c, dT)
        assert abs(c["dPi"] / dPi - 1) < 6e-3, (c, dPi)


def test_g0b_residual_is_the_timestep(g0b):
    last = g0b["conv"][-1]
    assert last["dT"] < 1e-4
    assert last["dPi"] < 1e-3


# ------------------------------------------------------------------ G2

def test_g2ab_ns_target_identities():
    r = G.g2_identities()
    assert r["worst_a"] < 1e-11
    assert r["worst_a"] < GATES["viscous"]["G2"]["ns_target_max"] * 10
    assert r["worst_phi"] < 1e-12 and r["worst_eta"] < 1e-12
    assert r["max_nsxy"] == 0.0


@pytest.fixture(scope="module")
def g2_runs():
    return {c: G.g2_run(BE, cfltau=c) for c in (0.016, 0.008, 0.004)}


def test_g2c_viscous_bjorken_vs_ode(g2_runs):
    r = g2_runs[0.004]
    assert r["primfail"] == 0
    assert r["maxU"] == 0.0
    assert r["spread"] < 1e-12
    assert r["shear_res"] < 1e-12
    assert r["eerr"] < 2e-3
    assert r["perr"] < 2e-2


def test_g2d_shear_slows_bjorken_cooling(g2_runs):
    ideal = G.g2_run(BE, eta_over_s=0.0)
    visc = g2_runs[0.004]
    assert visc["pieta"] < 0.0
    assert visc["e"] > ideal["e"]


def test_g2e_operator_split_is_first_order(g2_runs):
    errs = [g2_runs[c]["eerr"] for c in (0.016, 0.008, 0.004)]
    p = math.log2(errs[1] / errs[2])
    assert p > 0.7
    assert abs(p - GATES["viscous"]["G2"]["order"]) < 0.15


# ------------------------------------------------------------------ G3

def test_g3b_nu_ns_reduces_to_1d_form():
    r = G.g3_identity()
    assert r["worst"] < 1e-13
    assert r["worst_y"] == 0.0


@pytest.fixture(scope="module")
def g3():
    return G.g3_runs(BE)


def test_g3c_charge_conserved_on_closed_domain(g3):
    assert g3["primfail"] == (0, 0)
    assert g3["dper"] < 1e-12
    assert g3["dper"] <= GATES["viscous"]["G3"]["drift_max"] * 10


def test_g3d_diffusion_runs_down_the_gradient(g3):
    assert g3["peak_on"] < g3["peak_off"]
    assert g3["ntot"] > 100 and g3["nsame"] == 0
    assert g3["ntot"] == GATES["viscous"]["G3"]["cells_counted"]


def test_g3e_xy_symmetry(g3):
    assert g3["asym"] < 1e-12


# ------------------------------------------------------------------ Gk

def test_gk0_setup_and_bare_tau_n():
    m = G.gk_model(0.75, 1.0)
    p = m.params
    T0, A0 = G.GK_T0, G.GK_A0
    P1, n1, e1 = G.eos1(p, T0, -6.0 * T0)
    P2, n2, e2 = G.eos1(p, T0, 1.0 * T0)
    assert abs(e2 - e1) / e1 < 1e-14 and abs(P2 - P1) / P1 < 1e-14
    assert abs(math.log(n2 / n1) / 7.0 - 1) < 1e-12
    _, n0, _ = G.eos1(p, T0, A0 * T0)
    assert O.vacuum_weight(p, n0) == 1.0 and n0 > 10 * p.vacuum_n_hi
    assert O.diff_coeffs(p, T0, A0 * T0, n0)[2] == 0.0
    # tau_n against the bare moment ratio D_s z K3/K2, written here with scipy's Bessel K
    mhq = p.m_hq
    worst = 0.0
    for T in (0.500, 0.300, 0.200, 0.156):
        a = O.diff_tauN(p, T, A0, 0.7458, 1.0)
        z = mhq / T
        b = ((0.7458 / T) * z * (kve(3, z) / kve(2, z))) * 0.1973269804
        worst = max(worst, abs(b / a - 1))
    assert worst < 1e-12


@pytest.fixture(scope="module")
def tauD():
    return dict(over=G.gk_tauD_for_kstar(2.5 * G.GK_KFUND), prop=G.gk_tauD_for_kstar(1.4 * G.GK_KFUND))


def test_gka_overdamped_branch(tauD):
    for harm in (1, 2):
        r = G.gk_run_mode(BE, harmonic=harm, DsT=0.75, tauD=tauD["over"], trun=18.0)
        gam, gref = -r["w_meas"].imag, -r["w_ref"].imag
        xk = (r["k"] / r["kstar"]) ** 2
        assert abs(r["w_meas"].real) < 0.02 * gam
        assert r["split"] < 0.05
        assert r["Tdrift"] < 5e-3
        assert r["ysprd"] < 1e-12
        assert 0.98 < gam / gref < 1.02
        assert 0.98 < gam / (r["D"] * r["k"] ** 2) / G.gk_fick_excess(xk) < 1.02


@pytest.mark.skipif(not SLOW, reason="long oracle ladder; runs on the GPU by default (FIVO_SLOW=1 here)")
def test_gkb_propagating_branch_slow(tauD):
    from test_gpu_viscous_gates import check_gkb
    check_gkb(BE, tauD["prop"])


@pytest.mark.skipif(not SLOW, reason="long oracle ladder; runs on the GPU by default (FIVO_SLOW=1 here)")
def test_gkc_collision_slow(tauD):
    from test_gpu_viscous_gates import check_gkc
    check_gkc(BE, tauD["prop"])


# ------------------------------------------------------------------ Gd

def test_gd3_pi_sigma_contractions():
    assert G.gd_contractions() < 1e-12


@pytest.mark.parametrize("case", G.GD_CASES, ids=[c[0] for c in G.GD_CASES])
def test_gd1_dnmr_couplings_on_bjorken(case):
    r = G.gd_case(BE, case)
    pub = GATES["viscous"]["Gd"]
    assert max(abs(x) for x in r["eext"]) < 1e-3
    assert max(abs(x) for x in r["eext"]) <= pub["extrapolated_max"]
    assert r["order"] > 0.7
    assert pub["order_min"] - 0.01 <= r["order"] <= pub["order_max"] + 0.01
    assert abs(r["ebad"]) > 10 * abs(r["key_err"])


# ------------------------------------------------------------------ G1v

def test_g1v_referee_validations():
    v = G.g1v_validate()
    assert v["worst_ideal"] < 1e-8
    assert abs(v["worst_ideal"] / GATES["viscous"]["G1v"]["ideal_limit"] - 1) < 0.05
    assert v["max_pb0"] == 0.0
    for etas, (w, finite) in v["ns_dev"].items():
        assert w < 0.5 and finite
        assert v["attractor"][etas] < 5e-2


@pytest.mark.skipif(not SLOW, reason="N = 400 on the oracle is long; runs on the GPU by default (FIVO_SLOW=1 here)")
def test_g1v_solver_slow():
    from test_gpu_viscous_gates import check_g1v
    check_g1v(BE)


# ------------------------------------------------------------------ Gs

@pytest.mark.skipif(not SLOW, reason="long oracle ladder; runs on the GPU by default (FIVO_SLOW=1 here)")
def test_gs_sound_slow():
    from test_gpu_viscous_gates import check_gs
    check_gs(BE, Ny=16)
