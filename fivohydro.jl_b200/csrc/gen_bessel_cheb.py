"""Chebyshev coefficients of the scaled modified Bessel functions e^x K0, e^x K1.

Writes the coefficient tables used by fmath.cuh (device and host) for x in
[1, 1e4); the CPU oracle of the tests carries a copy of the same tables, and a
CPU test checks that both copies hold the same numbers.

  piece A, 1 <= x < 2:   e^x K_nu(x)            = sum_k a_k T_k(u),  u = 2x - 3
  piece B, 2 <= x < 1e4: sqrt(x) e^x K_nu(x)    = sum_k b_k T_k(u),  u = 4/x - 1

Coefficients are the discrete Chebyshev transform at Chebyshev–Gauss nodes
(N = degree + 24 nodes) of 50-digit mpmath values, rounded once to double.
Evaluated by Clenshaw's recurrence in double precision they are within
4e-16 relative of the exact functions on [1, 1e4).

    python gen_bessel_cheb.py        # prints the C initialisers
"""
import mpmath as mp

DEG_A = 21
DEG_B = 24


def _coeffs(func, n):
    N = n + 24
    us = [mp.cos(mp.pi * (j + mp.mpf(1) / 2) / N) for j in range(N)]
    fs = [func(u) for u in us]
    out = []
    for k in range(n + 1):
        s = mp.fsum(fs[j] * mp.cos(mp.pi * k * (j + mp.mpf(1) / 2) / N) for j in range(N))
        out.append(2 * s / N)
    out[0] /= 2
    return [float(v) for v in out]


def tables():
    mp.mp.dps = 50
    ka = lambda nu: (lambda u: mp.exp((u + 3) / 2) * mp.besselk(nu, (u + 3) / 2))
    kb = lambda nu: (lambda u: mp.sqrt(4 / (u + 1)) * mp.exp(4 / (u + 1)) * mp.besselk(nu, 4 / (u + 1)))
    return {"K0A": _coeffs(ka(0), DEG_A), "K1A": _coeffs(ka(1), DEG_A),
            "K0B": _coeffs(kb(0), DEG_B), "K1B": _coeffs(kb(1), DEG_B)}


def c_initialisers(prefix):
    lines = []
    for name, c in tables().items():
        body = ", ".join(repr(v) for v in c)
        lines.append(f"#define {prefix}{name} {{ {body} }}")
    return "\n".join(lines)


if __name__ == "__main__":
    print(c_initialisers("FX_CHEB_"))
