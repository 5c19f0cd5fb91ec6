/*
 * oracle/jlmath.h — scalar math for the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * The reference is Julia; its arithmetic runs on Julia's own exp/log, on
 * `Base.Math.pow_body` for float^integer, on NaN-propagating min/max and on
 * SpecialFunctions.jl (Amos) for scaled Bessel K. None of those libraries is
 * available here, so this file restates each one from a published method:
 *
 *   o_exp   Cody–Waite reduction x = k ln2 + r (ln2 split into a 32-bit head and
 *           a tail), degree-13 Taylor polynomial in Horner form with fma, and
 *           scaling by 2^k through the exponent bits.
 *   o_log   x = 2^e m, m in [1/sqrt2, sqrt2); log m = 2 atanh(s), s=(m-1)/(m+1),
 *           odd series to s^23; log x = e ln2 + log m.
 *   o_pow4  Julia's literal T^4 is `pow_body(T, 4)`: exponentiation by squaring
 *           carrying the low parts of each square (error-free products with
 *           fma), then one rounding of head + tail.
 *   o_min/o_max  Julia's Float64 min/max: NaN propagates, -0.0 < 0.0.
 *   o_clamp The reference's own clamp (src/utils.jl:6), NaN passes through.
 *   o_hypot Julia's hypot algorithm: order, early-out for widely varying
 *           operands, 2^+-563 rescaling, sqrt(fma(ax,ax,ay*ay)) and one
 *           fma-based correction step.
 *   o_besselkx  e^x K_nu(x), nu = 0, 1 (then upward recurrence):
 *           x < 1   power series of A&S 9.6.10-9.6.13 (K0, K1 via I0, I1 and
 *                   the digamma sums), times e^x;
 *           1 <= x < 2  Chebyshev series of e^x K_nu in u = 2x - 3;
 *           2 <= x < 1e4  Chebyshev series of sqrt(x) e^x K_nu in u = 4/x - 1;
 *                   both summed by Clenshaw's recurrence, coefficients from
 *                   50-digit mpmath values (the library's gen_bessel_cheb.py
 *                   writes the same tables);
 *           x >= 1e4  the reference's three-term asymptotic series
 *                   (safe_besselkx, src/eos.jl:27-34), verbatim in arithmetic.
 *           Checked against mpmath to <= 4e-16 relative (tests/test_oracle_math.py).
 *
 * The CUDA library implements the same algorithms with the same operation
 * order, and both are compiled without floating-point contraction, so the
 * oracle and the device produce identical bits.
 */
#ifndef FIVO_ORACLE_JLMATH_H
#define FIVO_ORACLE_JLMATH_H

#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

namespace orc {

static const double O_INF = std::numeric_limits<double>::infinity();
static const double O_NAN = std::numeric_limits<double>::quiet_NaN();
static const double O_PI = 3.141592653589793;

static inline uint64_t o_bits(double x) { uint64_t u; std::memcpy(&u, &x, 8); return u; }
static inline double o_from_bits(uint64_t u) { double x; std::memcpy(&x, &u, 8); return x; }
static inline bool o_isnan(double x) { return x != x; }
static inline bool o_isfinite(double x) { return std::isfinite(x); }
static inline bool o_signbit(double x) { return (o_bits(x) >> 63) != 0; }

/* Julia Base min/max for Float64 (NaN-propagating, -0.0 < 0.0). */
static inline double o_min(double x, double y) {
  bool take_y = (y < x) || (o_signbit(y) && !o_signbit(x));
  return take_y ? (o_isnan(x) ? x : y) : (o_isnan(y) ? y : x);
}
static inline double o_max(double x, double y) {
  bool take_y = (y > x) || (!o_signbit(y) && o_signbit(x));
  return take_y ? (o_isnan(x) ? x : y) : (o_isnan(y) ? y : x);
}
/* src/utils.jl:6 — `clamp(x, a, b) = x < a ? a : (x > b ? b : x)` */
static inline double o_clamp(double x, double a, double b) { return x < a ? a : (x > b ? b : x); }
/* Julia sign: NaN -> NaN, +-0 -> +-0, else +-1 */
static inline double o_sign(double x) {
  if (o_isnan(x)) return x;
  if (x == 0.0) return x;
  return x > 0.0 ? 1.0 : -1.0;
}

/* 2^k * p for p in [0.5, 2), k in [-1100, 1100] */
static inline double o_scale2(double p, int k) {
  if (k > 1023) { p = p * 8.98846567431158e307; k -= 1023; if (k > 1023) k = 1023; }  /* 2^1023 */
  if (k < -1022) {
    p = p * o_from_bits((uint64_t)(k + 1000 + 1023) << 52);
    return p * o_from_bits((uint64_t)(1023 - 1000) << 52);
  }
  return p * o_from_bits((uint64_t)(k + 1023) << 52);
}

static const double O_LN2_HI = 0.6931471803691238;     /* 32 leading bits of ln 2 */
static const double O_LN2_LO = 1.9082149292705877e-10; /* ln 2 - O_LN2_HI          */
static const double O_INV_LN2 = 1.4426950408889634;

static inline double o_exp(double x) {
  if (o_isnan(x)) return x;
  if (x > 709.782712893384) return O_INF;
  if (x < -745.1332191019412) return 0.0;
  double kd = std::nearbyint(x * O_INV_LN2);
  double r = std::fma(-kd, O_LN2_HI, x);
  r = std::fma(-kd, O_LN2_LO, r);
  double p = 1.6059043836821613e-10;            /* 1/13! */
  p = std::fma(p, r, 2.08767569878681e-09);      /* 1/12! */
  p = std::fma(p, r, 2.505210838544172e-08);
  p = std::fma(p, r, 2.755731922398589e-07);
  p = std::fma(p, r, 2.7557319223985893e-06);
  p = std::fma(p, r, 2.48015873015873e-05);
  p = std::fma(p, r, 0.0001984126984126984);
  p = std::fma(p, r, 0.001388888888888889);
  p = std::fma(p, r, 0.008333333333333333);
  p = std::fma(p, r, 0.041666666666666664);
  p = std::fma(p, r, 0.16666666666666666);
  p = std::fma(p, r, 0.5);
  p = std::fma(p, r, 1.0);
  p = std::fma(p, r, 1.0);
  return o_scale2(p, (int)kd);
}

static inline double o_log(double x) {
  if (o_isnan(x)) return x;
  if (x < 0.0) return O_NAN;
  if (x == 0.0) return -O_INF;
  if (x == O_INF) return x;
  int e = 0;
  if (x < 2.2250738585072014e-308) { x = x * 18014398509481984.0; e = -54; }  /* 2^54 */
  uint64_t u = o_bits(x);
  e += (int)((u >> 52) & 0x7ff) - 1023;
  double m = o_from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  double f = m - 1.0;
  double s = f / (2.0 + f);
  double z = s * s;
  double q = 0.043478260869565216;               /* 1/23 */
  q = std::fma(q, z, 0.047619047619047616);       /* 1/21 */
  q = std::fma(q, z, 0.05263157894736842);
  q = std::fma(q, z, 0.058823529411764705);
  q = std::fma(q, z, 0.06666666666666667);
  q = std::fma(q, z, 0.07692307692307693);
  q = std::fma(q, z, 0.09090909090909091);
  q = std::fma(q, z, 0.1111111111111111);
  q = std::fma(q, z, 0.14285714285714285);
  q = std::fma(q, z, 0.2);
  q = std::fma(q, z, 0.3333333333333333);
  double lm = std::fma(2.0 * s, z * q, 2.0 * s);
  double ed = (double)e;
  return std::fma(ed, O_LN2_HI, std::fma(ed, O_LN2_LO, lm));
}

/* Julia `x^4` for Float64 (literal_pow -> pow_body(x, 4)). */
static inline double o_pow4(double x) {
  double x2 = x * x;
  double e2 = std::fma(x, x, -x2);
  double err = (x2 * 2.0) * e2;
  double x4 = x2 * x2;
  double lo = std::fma(x2, x2, -x4) + err;
  if (o_isfinite(x4) && o_isfinite(lo)) return x4 + lo;
  return x4;
}

/* Julia `x^5` for Float64 (pow_body(x, 5)): the square and the fourth power carry
 * their low parts, the last product is fused. */
static inline double o_pow5(double x) {
  double x2 = x * x;
  double e2 = std::fma(x, x, -x2);
  double err = (x2 * 2.0) * e2;
  double x4 = x2 * x2;
  double lo = std::fma(x2, x2, -x4) + err;
  double err2 = x * lo;
  if (o_isfinite(x4) && o_isfinite(err2)) return std::fma(x4, x, err2);
  return x4 * x;
}

/* x^(3/2) as x sqrt(x) (both roundings IEEE). Julia's Float64^Float64 is a
 * double-double log/exp that can differ from this in the last bit. */
static inline double o_pow15(double x) { return x * std::sqrt(x); }

static inline double o_hypot(double x, double y) {
  if (std::isinf(x) || std::isinf(y)) return O_INF;
  double ax = std::fabs(x), ay = std::fabs(y);
  if (ay > ax) { double t = ax; ax = ay; ay = t; }
  if (ay <= ax * 1.0536712127723509e-08) return ax;      /* sqrt(eps/2) */
  double scale = 1.0;
  if (ax > 9.480751908109176e153) {                        /* sqrt(floatmax/2) */
    ax = ax * 3.312168642111238e-170; ay = ay * 3.312168642111238e-170;  /* 2^-563 */
    scale = 3.019169939857233e169;
  } else if (ay < 1.4916681462400413e-154) {               /* sqrt(floatmin) */
    ax = ax * 3.019169939857233e169; ay = ay * 3.019169939857233e169;
    scale = 3.312168642111238e-170;
  }
  double h = std::sqrt(std::fma(ax, ax, ay * ay));
  double hsq = h * h, axsq = ax * ax;
  h -= (std::fma(-ay, ay, hsq - axsq) + std::fma(h, h, -hsq) - std::fma(ax, ax, -axsq)) / (2.0 * h);
  return h * scale;
}

/* ---------------- scaled modified Bessel K ---------------- */

/* Chebyshev coefficients of e^x K_nu (piece A, u = 2x - 3, 1 <= x < 2) and of
 * sqrt(x) e^x K_nu (piece B, u = 4/x - 1, 2 <= x < 1e4), from 50-digit values */
static const double O_CHEB_K0A[] = {
  0.975293670703631, -0.14911366079770616, 0.01739593810625341, -0.0022865321321120587,
  0.00031902053048988584, -4.617742767921652e-05, 6.855099419473594e-06, -1.0367102847936046e-06,
  1.590358485499584e-07, -2.4674715067053715e-08, 3.863812252910323e-09, -6.096897833322557e-10,
  9.683069016813046e-11, -1.5464054179684872e-11, 2.481515505543579e-12, -3.9988227436440834e-13,
  6.467756230057925e-14, -1.0495481280269401e-14, 1.7081563652123322e-15, -2.7874138983949704e-16,
  4.5594687260393236e-17, -7.47431382282828e-18};
static const double O_CHEB_K1A[] = {
  1.287716931284971, -0.29355526501238677, 0.04578781607810882, -0.0075606314967654195,
  0.0012725129170005956, -0.0002159483044944044, 3.679893234585295e-05, -6.2852010326152186e-06,
  1.0749808007083846e-06, -1.8401830928999913e-07, 3.151902199740263e-08, -5.4007938898647565e-09,
  9.256899680411872e-10, -1.5869503264192334e-10, 2.7209976034987024e-11, -4.665992426162454e-12,
  8.002016298795233e-13, -1.3724164584124254e-13, 2.353949688583712e-14, -4.037647655524712e-15,
  6.925895800834045e-16, -1.1880559867658363e-16};
static const double O_CHEB_K0B[] = {
  1.2201515410329777, -0.0314481013119645, 0.0015698838857300533, -0.00012849549581627802,
  1.39498137188765e-05, -1.8317555227191195e-06, 2.766813639445015e-07, -4.660489897687948e-08,
  8.574034017414225e-09, -1.6975345093890614e-09, 3.5773972814003283e-10, -7.957489244477396e-11,
  1.8559491149549264e-11, -4.514597883374519e-12, 1.1403405882073441e-12, -2.9800969231481784e-13,
  8.032890775068375e-14, -2.2275133267462965e-14, 6.340076476276646e-15, -1.848593377920907e-15,
  5.5120559994043335e-16, -1.6782311257549006e-16, 5.2103917776435543e-17, -1.6475805939842632e-17,
  5.3004337711773354e-18};
static const double O_CHEB_K1B[] = {
  1.3603130952422213, 0.10392373657681724, -0.002857816859622779, 0.00019521551847135162,
  -1.936197974166083e-05, 2.406484947837217e-06, -3.5019606030878126e-07, 5.7410841254500495e-08,
  -1.0345762465678097e-08, 2.0150497551970347e-09, -4.1903547593419254e-10, 9.218315187605315e-11,
  -2.129967838427791e-11, 5.139639673482343e-12, -1.2891739609498229e-12, 3.348419666052243e-13,
  -8.976705182010146e-14, 2.4771544242195988e-14, -7.0198370892147685e-15, 2.038703166239861e-15,
  -6.057047270643018e-16, 1.8380935752430455e-16, -5.689462849193648e-17, 1.7940510478863572e-17,
  -5.7567444820733025e-18};
static const double O_EULER_GAMMA = 0.5772156649015329;

/* Clenshaw: b_k = fma(2u, b_{k+1}, c_k - b_{k+2}) for k = n-1..1;
 * sum = fma(u, b_1, c_0 - b_2) (one rounding per step on the dependency chain) */
static inline double o_clenshaw(const double* c, int n, double u) {
  double tu = 2.0 * u, b1 = 0.0, b2 = 0.0;
  for (int k = n - 1; k >= 1; --k) {
    double b = std::fma(tu, b1, c[k] - b2);
    b2 = b1; b1 = b;
  }
  return std::fma(u, b1, c[0] - b2);
}

/* e^x K0(x), e^x K1(x) for 0 < x < 1e4 */
static inline void o_k01x(double x, double* k0x, double* k1x) {
  if (x < 1.0) {
    double t = 0.25 * x * x;
    double term = 1.0, i0 = 1.0, s0 = 0.0, hk = 0.0;
    double term1 = 1.0, i1 = 1.0;
    double s1 = (-O_EULER_GAMMA) + (1.0 - O_EULER_GAMMA);
    for (int k = 1; k <= 15; ++k) {
      double kk = (double)k;
      term = term * (t / (kk * kk));
      hk = hk + 1.0 / kk;
      i0 = i0 + term;
      s0 = s0 + hk * term;
      term1 = term1 * (t / (kk * (kk + 1.0)));
      i1 = i1 + term1;
      s1 = s1 + (2.0 * (hk - O_EULER_GAMMA) + 1.0 / (kk + 1.0)) * term1;
    }
    double lx = o_log(0.5 * x);
    double k0 = -(lx + O_EULER_GAMMA) * i0 + s0;
    double I1 = 0.5 * x * i1;
    double k1 = 1.0 / x + lx * I1 - 0.25 * x * s1;
    double ex = o_exp(x);
    *k0x = k0 * ex;
    *k1x = k1 * ex;
    return;
  }
  const int na = (int)(sizeof(O_CHEB_K0A) / sizeof(double));
  const int nb = (int)(sizeof(O_CHEB_K0B) / sizeof(double));
  if (x < 2.0) {
    double u = (2.0 * x) - 3.0;
    *k0x = o_clenshaw(O_CHEB_K0A, na, u);
    *k1x = o_clenshaw(O_CHEB_K1A, na, u);
    return;
  }
  double u = (4.0 / x) - 1.0;
  double rs = 1.0 / std::sqrt(x);
  *k0x = o_clenshaw(O_CHEB_K0B, nb, u) * rs;
  *k1x = o_clenshaw(O_CHEB_K1B, nb, u) * rs;
}

/* safe_besselkx(nu, x), src/eos.jl:27-34: 0 for x <= 0 or non-finite, the
 * asymptotic series for x >= 1e4, else e^x K_nu(x) by upward recurrence. */
static inline double o_besselkx(int nu, double x) {
  if (!(o_isfinite(x) && x > 0.0)) return 0.0;
  if (x >= 1.0e4) {
    double mu = 4.0 * ((double)nu * (double)nu);
    double ix = 1.0 / (8.0 * x);
    double s = 1.0 + (mu - 1.0) * ix * (1.0 + (mu - 9.0) * ix / 2.0 * (1.0 + (mu - 25.0) * ix / 3.0));
    return std::sqrt(O_PI / (2.0 * x)) * s;
  }
  double k0, k1;
  o_k01x(x, &k0, &k1);
  if (nu == 0) return k0;
  if (nu == 1) return k1;
  double km = k0, kc = k1;
  for (int n = 1; n < nu; ++n) {
    double kn = km + ((2.0 * n) / x) * kc;
    km = kc; kc = kn;
  }
  return kc;
}

}  // namespace orc
#endif
