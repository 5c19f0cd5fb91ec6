"""The oracle's scalar math (oracle/jlmath.h) against independent references.

The reference takes exp/log from Julia and e^x K_nu(x) from SpecialFunctions.jl
(Amos); the oracle and the CUDA library restate them from published methods, so
they are pinned here against numpy (correctly rounded to within an ulp) and
against 40-digit mpmath values (tests/golden/besselkx.json).
"""
import json
import re
import pathlib

import numpy as np
import pytest

import _oracle as O

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"
ROOT = pathlib.Path(__file__).resolve().parent.parent


def test_exp_log_within_an_ulp():
    rng = np.random.default_rng(1)
    x = np.concatenate([rng.uniform(-745, 709, 50000), rng.uniform(-1, 1, 50000), [0.0, -0.0, 1e-300]])
    e = O.vec(O.lib().oracle_exp, x)
    ref = np.exp(x)
    ok = ref > 2.3e-308
    assert np.max(np.abs(e[ok] / ref[ok] - 1)) <= 2.3e-16 * 2
    y = np.exp(rng.uniform(-740, 709, 50000))
    lg = O.vec(O.lib().oracle_log, y)
    assert np.max(np.abs(lg - np.log(y)) / np.maximum(np.abs(np.log(y)), 1e-300)) <= 2.3e-16 * 2


def test_exp_log_special_values():
    e = O.vec(O.lib().oracle_exp, np.array([np.nan, 710.0, -746.0, 0.0, -745.0]))
    assert np.isnan(e[0]) and e[1] == np.inf and e[2] == 0.0 and e[3] == 1.0 and 0 < e[4] < 1e-320
    lg = O.vec(O.lib().oracle_log, np.array([np.nan, -1.0, 0.0, np.inf, 1.0, 5e-324]))
    assert np.isnan(lg[0]) and np.isnan(lg[1]) and lg[2] == -np.inf and lg[3] == np.inf and lg[4] == 0.0
    assert abs(lg[5] - np.log(5e-324)) < 1e-13


def test_pow4_matches_exact_rounding():
    """Julia's T^4 (pow_body) is the exactly rounded fourth power in the
    normal range; check against exact rational arithmetic."""
    from fractions import Fraction
    rng = np.random.default_rng(2)
    x = np.concatenate([rng.uniform(0, 3, 3000), np.exp(rng.uniform(-40, 40, 1000))])
    p = O.vec(O.lib().oracle_pow4, x)
    for xi, pi in zip(x[:800], p[:800]):
        assert pi == float(Fraction(float(xi)) ** 4)


def test_hypot():
    rng = np.random.default_rng(3)
    a, b = rng.normal(size=20000) * 10.0 ** rng.integers(-200, 200, 20000), rng.normal(size=20000)
    h = O.vec(O.lib().oracle_hypot, a, b)
    assert np.max(np.abs(h / np.hypot(a, b) - 1)) <= 2.3e-16


def test_besselkx_against_mpmath():
    rows = json.loads((GOLDEN / "besselkx.json").read_text())
    x = np.array([r["x"] for r in rows])
    for nu in (0, 1, 2, 3, 5):
        ref = np.array([float(r[str(nu)]) for r in rows])
        got = O.besselkx(nu, x)
        rel = np.abs(got / ref - 1)
        assert rel.max() < 2e-15, (nu, float(rel.max()), float(x[np.argmax(rel)]))


def test_besselkx_reference_branches():
    """safe_besselkx (src/eos.jl:27-34): 0 off the domain; the reference's own
    three-term asymptotic series from x = 1e4 (bit for bit)."""
    x = np.array([0.0, -1.0, np.nan, np.inf])
    assert np.all(O.besselkx(2, x) == 0.0)
    big = np.array([1e4, 3.7e5, 1.5e20])
    for nu in (1, 2):
        mu = 4.0 * nu * nu
        ix = 1.0 / (8.0 * big)
        s = 1.0 + (mu - 1.0) * ix * (1.0 + (mu - 9.0) * ix / 2.0 * (1.0 + (mu - 25.0) * ix / 3.0))
        assert np.array_equal(O.besselkx(nu, big), np.sqrt(np.pi / (2.0 * big)) * s)


@pytest.mark.parametrize("nu", [0, 1, 2])
def test_besselkx_continuity_at_branch_points(nu):
    for x0 in (1.0, 2.0, 1e4):
        xs = np.array([np.nextafter(x0, 0), x0])
        v = O.besselkx(nu, xs)
        assert abs(v[1] / v[0] - 1) < 1e-13


def _c_table(text, name):
    """The numbers of a C initialiser `name ... { a, b, ... }` in a source file."""
    m = re.search(re.escape(name) + r"[^{]*\{([^}]*)\}", text)
    assert m, name
    return [float(v) for v in m.group(1).replace("\\", " ").split(",") if v.strip()]


def test_bessel_tables_same_in_oracle_and_library():
    """The oracle and the CUDA library sum the same Chebyshev coefficients."""
    orc = (ROOT / "oracle" / "jlmath.h").read_text()
    lib = (ROOT / "fivohydro.jl_b200" / "csrc" / "fmath.cuh").read_text()
    for t in ("K0A", "K1A", "K0B", "K1B"):
        a, b = _c_table(orc, "O_CHEB_" + t), _c_table(lib, "#define FX_CHEB_" + t)
        assert a == b and len(a) >= 20, t
