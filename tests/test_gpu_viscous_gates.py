"""The reference's dissipative gates on the GPU, and the device equal to the
oracle bit for bit on each gate's own setup.

The same gate code as tests/test_oracle_viscous_gates.py (tests/_gates.py),
with the CUDA library as the solver: G0b, G2, G3, Gd, the whole of Gk
(test/test_charge_dispersion2d.jl, including the propagating branch, the k_*
scan, the tau_n control and the dx ladder), Gs (test/test_sound2d.jl) and the
G1v solver ladder (test/test_gubser_viscous2d.jl, N = 100/200/400). The
`check_*` functions are shared with the oracle's FIVO_SLOW runs.
"""
import json
import math
import pathlib

import numpy as np
import pytest

import _gates as G
import _oracle as O
from fivo2d import _abi as A

GATES = json.loads((pathlib.Path(__file__).resolve().parent / "golden" / "gates.json").read_text())


# ------------------------------------------------------------------ shared checks (oracle FIVO_SLOW + GPU)

def check_gkb(be, tauD_prop):
    """Gk-b, test/test_charge_dispersion2d.jl:333-366"""
    rs = []
    for harm in (2, 3):
        r = G.gk_run_mode(be, harmonic=harm, DsT=0.75, tauD=tauD_prop, trun=18.0, dts=0.2)
        Om, Omr = r["w_meas"].real, r["w_ref"].real
        gam, g0 = -r["w_meas"].imag, 1 / (2 * r["tn"])
        assert r["k"] > r["kstar"]
        assert abs(r["w_ref"].imag + 1 / (2 * r["tn"])) < 1e-10
        assert 0.97 < Om / Omr < 1.03
        assert g0 <= gam <= g0 + 0.20 * r["dx"] * r["k"] ** 2
        rs.append((Om, gam, r))
    assert rs[1][0] / rs[0][0] > 1.2
    assert abs(rs[1][1] / rs[0][1] - 1) < 0.10
    return rs


def check_gkc(be, tauD_prop):
    """Gk-c, :369-396: the measured transition brackets the predicted k_*"""
    m = G.gk_model(0.75, tauD_prop)
    _, n0, _ = G.eos1(m.params, G.GK_T0, G.GK_A0 * G.GK_T0)
    kap, tn, _ = O.diff_coeffs(m.params, G.GK_T0, G.GK_A0 * G.GK_T0, n0)
    ks = G.gk_kstar(kap / n0, tn)
    assert abs(ks - GATES["viscous"]["Gk"]["kstar_predicted"]) < 1e-3
    lastflat, firstosc = 0.0, math.inf
    for harm in range(1, 7):
        r = G.gk_run_mode(be, harmonic=harm, DsT=0.75, tauD=tauD_prop, trun=10.0, dts=0.2)
        osc = abs(r["w_meas"].real) > 0.05 * abs(r["w_meas"].imag)
        if osc:
            firstosc = min(firstosc, r["k"])
        else:
            lastflat = max(lastflat, r["k"])
    assert lastflat < ks < firstosc
    return ks, lastflat, firstosc


def check_gkd(be, tauD_prop):
    """Gk-d, :399-441: the oscillation is the transient mode, not the scheme"""
    rows = []
    for fac, trun, dts in ((1.0, 20.0, 0.2), (0.25, 6.0, 0.1), (0.0025, 1.2, 0.04)):
        rows.append(G.gk_run_mode(be, harmonic=6, DsT=0.75, tauD=tauD_prop * fac, trun=trun, dts=dts))
    assert abs(rows[0]["w_meas"].real) > 0.2 * abs(rows[0]["w_meas"].imag)
    assert abs(rows[1]["w_meas"].real) > 0.2 * abs(rows[1]["w_meas"].imag)
    assert rows[2]["k"] < rows[2]["kstar"]
    assert abs(rows[2]["w_meas"].real) < 1e-9 * abs(rows[2]["w_meas"].imag)
    xk3 = (rows[2]["k"] / rows[2]["kstar"]) ** 2
    rat = -rows[2]["w_meas"].imag / (rows[2]["D"] * rows[2]["k"] ** 2) / G.gk_fick_excess(xk3)
    assert 0.98 < rat < 1.06
    assert rows[1]["w_meas"].real > rows[0]["w_meas"].real
    return rows


def check_gke(be, tauD_over, tauD_prop):
    """Gk-e, :444-539: the charge row's numerical diffusion is first order in dx,
    only on the propagating branch, and not the timestep"""
    dn = []
    for N in (96, 192, 384):
        r = G.gk_run_mode(be, harmonic=4, DsT=0.75, tauD=tauD_prop, trun=12.0, dts=0.2, N=N)
        dn.append((-r["w_meas"].imag - 1 / (2 * r["tn"])) / r["k"] ** 2)
    ords = [math.log2(dn[i] / dn[i + 1]) for i in range(2)]
    assert all(d > 0 for d in dn)
    assert dn[1] < dn[0] and dn[2] < dn[1]
    for o in ords:
        assert 0.80 < o < 1.35
    devs = []
    for N in (96, 192, 384):
        r = G.gk_run_mode(be, harmonic=1, DsT=0.75, tauD=tauD_over, trun=12.0, N=N)
        devs.append(-r["w_meas"].imag / -r["w_ref"].imag - 1)
    assert max(abs(d) for d in devs) < 3e-3
    assert min(devs) < 0 < max(devs)
    gs = []
    for cfl in (0.30, 0.15):
        r = G.gk_run_mode(be, harmonic=4, DsT=0.75, tauD=tauD_prop, trun=12.0, dts=0.2, CFL=cfl)
        gs.append(-r["w_meas"].imag)
    k4 = 2 * math.pi * 4 / G.GK_LBOX
    assert abs(gs[1] - gs[0]) < 0.25 * abs(dn[1] - dn[0]) * k4 ** 2
    return dn, ords, devs


def check_gs(be, N=128, Ny=None):
    """Gs, test/test_sound2d.jl:172-218"""
    r = G.gate_gs(be, N=N, Ny=Ny)
    base = r["base"]
    cs_err = abs(base["cs"] - base["cs_exact"]) / base["cs_exact"]
    assert cs_err < 0.02
    assert cs_err < 10 * GATES["viscous"]["Gs"]["cs_rel"]
    assert abs(base["G"]) < 5e-3
    for row in r["shear"]:
        assert 0.98 < row["ratio"] < 1.02
    assert max(row["split"] for row in r["shear"]) < 0.01
    for row in r["bulk"]:
        assert 0.85 < row["ratio"] < 1.25
    assert abs(r["bulk"][0]["ratio"] - r["bulk"][1]["ratio"]) / r["bulk"][0]["ratio"] < 0.08
    return r, cs_err


def check_g1v(be):
    """the solver half of G1v, test/test_gubser_viscous2d.jl:217-241"""
    out = {}
    for etas in (0.005, 0.02):
        rs, Th, pb = G.g1v_ode(etas)
        Ti, Pi = G.g1v_interp(rs, Th), G.g1v_interp(rs, pb)
        runs = [G.g1v_run(be, N, etas, 2.0, Ti, Pi) for N in (100, 200, 400)]
        for r in runs:
            assert r["nc"] > 100
            assert r["asym"] < 1e-11
        oT = math.log2(runs[1]["L2T"] / runs[2]["L2T"])
        op = math.log2(runs[1]["L2p"] / runs[2]["L2p"])
        assert runs[-1]["L2T"] < 5e-3
        assert runs[-1]["L2p"] < 8e-2
        assert oT > 1.0
        assert op > 0.7
        out[etas] = (runs, oT, op)
    return out


# ------------------------------------------------------------------ GPU tests

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def be(gpu_lib):
    return G.GPUBackend(gpu_lib)


def _bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return bool(np.all((a.view(np.int64) == b.view(np.int64)) | (np.isnan(a) & np.isnan(b))))


@pytest.mark.parametrize("name", G.GATE_SETUPS)
def test_gate_setup_bitwise_with_oracle(be, name):
    """Each gate's own configuration, a few run_sim_2d! steps on the device and on
    the oracle: state, primitives and warm starts to the bit."""
    m, g, U0, tau0, bc, integ, cfl, cfltau, finalize = G.gate_setup(name)
    sols = [be.solver(m, g), G.OracleBackend().solver(m, g)]
    res = []
    for s in sols:
        s.set_state(U0)
        if finalize:
            s.finalize_ic(tau0, bc)
        r = s.run(tau0, 1e9, cfl, cfltau, integ, bc, max_steps=4)
        assert r["ok"] and r["nsteps"] == 4
        res.append((r, s.get_state(), s.primitives(), s.get_history()))
        s.close()
    (rg, Ug, pg, hg), (ro, Uo, po, ho) = res
    assert rg["tau"] == ro["tau"]
    assert _bits_equal(Ug, Uo)
    for k in ("yT", "phi", "ux", "uy", "P", "n", "e"):
        assert _bits_equal(pg[k], po[k]), k
    for k in ("x0_yT", "x0_phi", "x0_ux", "x0_uy", "ux_prev", "uy_prev"):
        assert _bits_equal(hg[k], ho[k]), k


def test_gpu_g0b(be):
    r = G.gate_g0b(be)
    for row, pub in zip(r["rows"], GATES["viscous"]["G0b"]["dPi_production_cfl"]):
        assert row["Tspread"] < 1e-12 and row["dT"] < 1e-4 and row["PiP"] > 0.05
        assert abs(row["dPi"] - pub) < 5e-5
    assert r["conv"][-1]["dT"] < 1e-4 and r["conv"][-1]["dPi"] < 1e-3


def test_gpu_g2(be):
    runs = {c: G.g2_run(be, cfltau=c) for c in (0.016, 0.008, 0.004)}
    r = runs[0.004]
    assert r["primfail"] == 0 and r["maxU"] == 0.0 and r["spread"] < 1e-12 and r["shear_res"] < 1e-12
    assert r["eerr"] < 2e-3 and r["perr"] < 2e-2
    ideal = G.g2_run(be, eta_over_s=0.0)
    assert r["pieta"] < 0.0 and r["e"] > ideal["e"]
    errs = [runs[c]["eerr"] for c in (0.016, 0.008, 0.004)]
    assert math.log2(errs[1] / errs[2]) > 0.7


def test_gpu_g3(be):
    r = G.g3_runs(be)
    assert r["primfail"] == (0, 0) and r["dper"] < 1e-12
    assert r["peak_on"] < r["peak_off"]
    assert r["nsame"] == 0 and r["ntot"] == GATES["viscous"]["G3"]["cells_counted"]
    assert r["asym"] < 1e-12


@pytest.mark.parametrize("case", G.GD_CASES, ids=[c[0] for c in G.GD_CASES])
def test_gpu_gd1(be, case):
    r = G.gd_case(be, case)
    assert max(abs(x) for x in r["eext"]) <= GATES["viscous"]["Gd"]["extrapolated_max"]
    assert 0.96 <= r["order"] <= 1.0
    assert abs(r["ebad"]) > 10 * abs(r["key_err"])


@pytest.fixture(scope="module")
def tauD():
    return dict(over=G.gk_tauD_for_kstar(2.5 * G.GK_KFUND), prop=G.gk_tauD_for_kstar(1.4 * G.GK_KFUND))


def test_gpu_gka(be, tauD):
    for harm in (1, 2):
        r = G.gk_run_mode(be, harmonic=harm, DsT=0.75, tauD=tauD["over"], trun=18.0)
        gam, gref = -r["w_meas"].imag, -r["w_ref"].imag
        assert abs(r["w_meas"].real) < 0.02 * gam and r["split"] < 0.05
        assert r["Tdrift"] < 5e-3 and r["ysprd"] < 1e-12
        assert 0.98 < gam / gref < 1.02


def test_gpu_gkb(be, tauD):
    check_gkb(be, tauD["prop"])


def test_gpu_gkc(be, tauD):
    check_gkc(be, tauD["prop"])


def test_gpu_gkd(be, tauD):
    check_gkd(be, tauD["prop"])


def test_gpu_gke(be, tauD):
    check_gke(be, tauD["over"], tauD["prop"])


def test_gpu_gs(be):
    check_gs(be)


def test_gpu_g1v(be):
    check_g1v(be)
