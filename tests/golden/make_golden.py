"""Generate the golden fixtures of tests/golden/.

  besselkx.json      e^x K_nu(x), nu in {0,1,2,3,5}, at 40 significant digits
                     (mpmath), the referee for the scaled Bessel functions the
                     reference takes from SpecialFunctions.jl 2.6.1 (Amos).
  gates.json         the reference's published gate numbers for this path
                     (README2D.md:273-285) and their test settings
                     (test/test_gubser2d.jl:50-55, 97-129; test/test_bjorken2d.jl:94-169;
                     the dissipative gates under "viscous": test/test_bjorken_bulk2d.jl:122-131,
                     test/test_dissipation2d.jl, test/test_charge2d.jl,
                     test/test_charge_dispersion2d.jl, test/test_dnmr2d.jl,
                     test/test_gubser_viscous2d.jl, test/test_sound2d.jl).

Run from the repository root: python tests/golden/make_golden.py
"""
import json
import pathlib

import mpmath as mp

HERE = pathlib.Path(__file__).resolve().parent


def besselkx():
    mp.mp.dps = 40
    xs = [mp.mpf(10) ** (mp.mpf(k) / 40) * mp.mpf("0.001") for k in range(0, 281)]  # 1e-3 .. 1e4
    xs = [x for x in xs if x < 9999]
    xs += [mp.mpf(v) for v in ("0.15", "0.5", "0.999", "1.0", "1.001", "1.9", "2.5", "7.5", "50", "1000", "9999")]
    out = []
    for x in sorted(set(xs)):
        xf = float(x)
        row = {"x": xf}
        for nu in (0, 1, 2, 3, 5):
            row[str(nu)] = mp.nstr(mp.besselk(nu, xf) * mp.exp(xf), 30)
        out.append(row)
    return out


GATES = {
    "source": "README2D.md:273-275 (run of 2026-09-15)",
    "gubser": {
        "settings": {"box": 10.0, "tau0": 1.0, "tauf": 2.0, "q": 1.0, "Tc0": 0.6, "alpha": -20.0,
                     "CFL": 0.15, "CFLtau": 0.05, "rcmp": 3.0, "eos": "ConformalHQEOS()"},
        "N": [100, 200, 400],
        "L2T": [3.29e-3, 8.81e-4, 2.26e-4],
        "L2u": [7.73e-3, 1.92e-3, 4.57e-4],
        "order_T": [1.90, 1.96],
        "order_u": [2.01, 2.07],
        "xy_symmetry_max": 1e-12,
    },
    "bjorken": {
        "settings": {"N": 24, "box": 6.0, "tau0": 0.4, "tauf": 4.0, "T0": 0.50, "alpha0": -4.2,
                     "CFL": 0.2, "eos": "LatticeHRGEOS()"},
        "order": {"ssprk2": 2.00, "ssprk3": 2.99},
        "drift_max": 1e-13, "E_spread_max": 1e-13, "err_max_at_cfltau_0.005": 5e-4,
    },
    "primrec": {"ntrial": 1500, "tol": 1e-9, "zero_flow_T": 1e-10, "zero_flow_u": 1e-12,
                "y_symmetric_uy": 1e-12, "tilt_min_rad": 1e-3},
    "viscous": {
        "source": "README2D.md:274-285; per-case figures quoted in the test files' comments",
        "G0b": {"T_tol": 1e-4, "Pi_tol": 7.5e-3, "zeta_over_s": [0.05, 0.15, 0.30],
                "dPi_production_cfl": [0.0052, 0.0075, 0.0016],
                "source_tables": "TWOD_PROGRAM.md:1800-1812",
                "dT_production_cfl": [9.90e-5, 9.93e-5, 3.53e-5],
                "PiP": [0.066, 0.236, 0.600],
                "cfl_scan": [0.20, 0.10, 0.05, 0.025],
                "cfl_scan_dT": [1.42e-4, 4.92e-5, 1.16e-5, 2.17e-5],
                "cfl_scan_dPi": [9.72e-3, 5.00e-3, 2.17e-3, 9.34e-4]},
        "G1v": {"ideal_limit": 3.6e-11},
        "G2": {"ns_target_max": 2.4e-15, "order": 1.05},
        "G3": {"drift_max": 1.9e-15, "cells_counted": 2104, "up_gradient": 0},
        "Gk": {"tau_n_ratio": 1.0000, "kstar_predicted": 0.733},
        "Gd": {"extrapolated_max": 3e-4, "order_min": 0.97, "order_max": 0.99, "wrong_sign_miss": [5e-3, 1.7]},
        "Gs": {"cs_rel": 5e-4},
    },
}


if __name__ == "__main__":
    (HERE / "besselkx.json").write_text(json.dumps(besselkx(), indent=0))
    (HERE / "gates.json").write_text(json.dumps(GATES, indent=1))
    print("wrote", HERE / "besselkx.json", HERE / "gates.json")
