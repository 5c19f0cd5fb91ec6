/*
 * fmath.cuh — scalar FP64 math of the stage, identical in device and host code.
 *
 * The reference (Julia) evaluates exp/log with Julia's own implementations,
 * float^integer with Base.Math.pow_body, min/max with NaN propagation, and
 * scaled Bessel K with SpecialFunctions.jl. This file implements each from a
 * published method, chosen so that every operation is an IEEE-754 primitive
 * (+ - * / sqrt, fused multiply-add): compiled without contraction (-fmad=false)
 * the results are the same bits on the GPU and on any host.
 *
 *   fx_exp   Cody–Waite reduction x = k ln2 + r with a 32-bit head of ln 2,
 *            degree-13 Taylor polynomial in r (|r| <= ln2/2) by Horner/fma,
 *            2^k applied through the exponent field (two steps below 2^-1022).
 *   fx_log   x = 2^e m with m in [1/sqrt2, sqrt2); log m = 2 atanh(s),
 *            s = (m-1)/(m+1), odd series to s^23.
 *   fx_pow4  exponentiation by squaring with error-free squares (pow_body).
 *   fx_k01x  e^x K0(x), e^x K1(x): power series (A&S 9.6.10-9.6.13) for x < 1;
 *            Chebyshev series by Clenshaw's recurrence for 1 <= x < 1e4 (in
 *            u = 2x - 3 below 2, in u = 4/x - 1 for sqrt(x) e^x K above), with
 *            coefficients computed here from 50-digit values (gen_bessel_cheb.py);
 *            <= 4e-16 relative to 40-digit references.
 *   fx_besselkx  safe_besselkx (src/eos.jl:27-34): 0 for x <= 0, the reference's
 *            three-term asymptotic series for x >= 1e4, else recurrence.
 */
#ifndef FIVO_FMATH_CUH
#define FIVO_FMATH_CUH

#include <cstdint>
#include <cmath>

#ifdef __CUDACC__
#define FX_HD __host__ __device__ __forceinline__
#else
#define FX_HD inline
#endif

namespace fx {

#define FX_PI 3.141592653589793

FX_HD uint64_t bits(double x) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(x);
#else
  uint64_t u; __builtin_memcpy(&u, &x, 8); return u;
#endif
}
FX_HD double from_bits(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double x; __builtin_memcpy(&x, &u, 8); return x;
#endif
}
FX_HD bool isnan_(double x) { return x != x; }
FX_HD bool isfinite_(double x) { return (bits(x) & 0x7ff0000000000000ULL) != 0x7ff0000000000000ULL; }
FX_HD bool isinf_(double x) { return (bits(x) & 0x7fffffffffffffffULL) == 0x7ff0000000000000ULL; }
FX_HD bool signbit_(double x) { return (bits(x) >> 63) != 0; }
FX_HD double inf_() { return from_bits(0x7ff0000000000000ULL); }
FX_HD double nan_() { return from_bits(0x7ff8000000000000ULL); }
FX_HD double fabs_(double x) { return from_bits(bits(x) & 0x7fffffffffffffffULL); }
FX_HD double fma_(double a, double b, double c) {
#ifdef __CUDA_ARCH__
  return __fma_rn(a, b, c);
#else
  return std::fma(a, b, c);
#endif
}
FX_HD double sqrt_(double x) {
#ifdef __CUDA_ARCH__
  return __dsqrt_rn(x);
#else
  return std::sqrt(x);
#endif
}
FX_HD double rint_(double x) {
#ifdef __CUDA_ARCH__
  return rint(x);
#else
  return std::nearbyint(x);
#endif
}

/* Julia Float64 min/max: NaN propagates, -0.0 orders below 0.0 */
FX_HD double jmin(double x, double y) {
  bool ty = (y < x) || (signbit_(y) && !signbit_(x));
  return ty ? (isnan_(x) ? x : y) : (isnan_(y) ? y : x);
}
FX_HD double jmax(double x, double y) {
  bool ty = (y > x) || (!signbit_(y) && signbit_(x));
  return ty ? (isnan_(x) ? x : y) : (isnan_(y) ? y : x);
}
/* clamp of src/utils.jl:6 (NaN passes through) */
FX_HD double jclamp(double x, double a, double b) { return x < a ? a : (x > b ? b : x); }
FX_HD double jsign(double x) {
  if (isnan_(x)) return x;
  if (x == 0.0) return x;
  return x > 0.0 ? 1.0 : -1.0;
}

FX_HD double scale2(double p, int k) {
  /* p * 2^k in two exact power-of-two factors, without branches: the second
   * factor is 1.0 (an exact multiplication) in the normal range; above it the
   * first is 2^1023, below it 2^(k+1000) and the second 2^-1000 */
  const bool big = k > 1023, small = k < -1022;
  int k1 = big ? 1023 : (small ? k + 1000 : k);
  int k2 = big ? k - 1023 : (small ? -1000 : 0);
  k2 = k2 > 1023 ? 1023 : k2;
  double t = p * from_bits((uint64_t)(k1 + 1023) << 52);
  return t * from_bits((uint64_t)(k2 + 1023) << 52);
}

FX_HD double fx_exp(double x) {
  /* the special cases are selected at the end, so the body is straight-line
   * code that the scheduler can interleave with independent work */
  const bool nan = isnan_(x), over = x > 709.782712893384, under = x < -745.1332191019412;
  const double xs = (nan || over || under) ? 0.0 : x;
  double kd = rint_(xs * 1.4426950408889634);
  double r = fma_(-kd, 0.6931471803691238, xs);
  r = fma_(-kd, 1.9082149292705877e-10, r);
  double p = 1.6059043836821613e-10;
  p = fma_(p, r, 2.08767569878681e-09);
  p = fma_(p, r, 2.505210838544172e-08);
  p = fma_(p, r, 2.755731922398589e-07);
  p = fma_(p, r, 2.7557319223985893e-06);
  p = fma_(p, r, 2.48015873015873e-05);
  p = fma_(p, r, 0.0001984126984126984);
  p = fma_(p, r, 0.001388888888888889);
  p = fma_(p, r, 0.008333333333333333);
  p = fma_(p, r, 0.041666666666666664);
  p = fma_(p, r, 0.16666666666666666);
  p = fma_(p, r, 0.5);
  p = fma_(p, r, 1.0);
  p = fma_(p, r, 1.0);
  const double v = scale2(p, (int)kd);
  return nan ? x : (over ? inf_() : (under ? 0.0 : v));
}

FX_HD double fx_log(double x) {
  if (isnan_(x)) return x;
  if (x < 0.0) return nan_();
  if (x == 0.0) return -inf_();
  if (isinf_(x)) return x;
  int e = 0;
  if (x < 2.2250738585072014e-308) { x = x * 18014398509481984.0; e = -54; }
  uint64_t u = bits(x);
  e += (int)((u >> 52) & 0x7ff) - 1023;
  double m = from_bits((u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL);
  if (m > 1.4142135623730951) { m = m * 0.5; e += 1; }
  double f = m - 1.0;
  double s = f / (2.0 + f);
  double z = s * s;
  double q = 0.043478260869565216;
  q = fma_(q, z, 0.047619047619047616);
  q = fma_(q, z, 0.05263157894736842);
  q = fma_(q, z, 0.058823529411764705);
  q = fma_(q, z, 0.06666666666666667);
  q = fma_(q, z, 0.07692307692307693);
  q = fma_(q, z, 0.09090909090909091);
  q = fma_(q, z, 0.1111111111111111);
  q = fma_(q, z, 0.14285714285714285);
  q = fma_(q, z, 0.2);
  q = fma_(q, z, 0.3333333333333333);
  double lm = fma_(2.0 * s, z * q, 2.0 * s);
  double ed = (double)e;
  return fma_(ed, 0.6931471803691238, fma_(ed, 1.9082149292705877e-10, lm));
}

/* x^4 as Julia's pow_body(x, 4) */
FX_HD double fx_pow4(double x) {
  double x2 = x * x;
  double e2 = fma_(x, x, -x2);
  double err = (x2 * 2.0) * e2;
  double x4 = x2 * x2;
  double lo = fma_(x2, x2, -x4) + err;
  if (isfinite_(x4) && isfinite_(lo)) return x4 + lo;
  return x4;
}

/* x^5 as Julia's pow_body(x, 5) */
FX_HD double fx_pow5(double x) {
  double x2 = x * x;
  double e2 = fma_(x, x, -x2);
  double err = (x2 * 2.0) * e2;
  double x4 = x2 * x2;
  double lo = fma_(x2, x2, -x4) + err;
  double err2 = x * lo;
  if (isfinite_(x4) && isfinite_(err2)) return fma_(x4, x, err2);
  return x4 * x;
}

/* x^(3/2) as x sqrt(x) (IEEE square root and product) */
FX_HD double fx_pow15(double x) { return x * sqrt_(x); }

/* Julia's hypot (correctly rounded branch with fma) */
FX_HD double fx_hypot(double x, double y) {
  if (isinf_(x) || isinf_(y)) return inf_();
  double ax = fabs_(x), ay = fabs_(y);
  if (ay > ax) { double t = ax; ax = ay; ay = t; }
  if (ay <= ax * 1.0536712127723509e-08) return ax;
  double scale = 1.0;
  if (ax > 9.480751908109176e153) {
    ax = ax * 3.312168642111238e-170; ay = ay * 3.312168642111238e-170;
    scale = 3.019169939857233e169;
  } else if (ay < 1.4916681462400413e-154) {
    ax = ax * 3.019169939857233e169; ay = ay * 3.019169939857233e169;
    scale = 3.312168642111238e-170;
  }
  double h = sqrt_(fma_(ax, ax, ay * ay));
  double hsq = h * h, axsq = ax * ax;
  h -= (fma_(-ay, ay, hsq - axsq) + fma_(h, h, -hsq) - fma_(ax, ax, -axsq)) / (2.0 * h);
  return h * scale;
}

/* Chebyshev coefficients (gen_bessel_cheb.py: 50-digit mpmath, rounded once):
 * A: e^x K_nu(x) in u = 2x - 3 on [1, 2); B: sqrt(x) e^x K_nu(x) in u = 4/x - 1 on [2, 1e4). */
#define FX_CHEB_K0A { \
  0.975293670703631, -0.14911366079770616, 0.01739593810625341, -0.0022865321321120587, \
  0.00031902053048988584, -4.617742767921652e-05, 6.855099419473594e-06, -1.0367102847936046e-06, \
  1.590358485499584e-07, -2.4674715067053715e-08, 3.863812252910323e-09, -6.096897833322557e-10, \
  9.683069016813046e-11, -1.5464054179684872e-11, 2.481515505543579e-12, -3.9988227436440834e-13, \
  6.467756230057925e-14, -1.0495481280269401e-14, 1.7081563652123322e-15, -2.7874138983949704e-16, \
  4.5594687260393236e-17, -7.47431382282828e-18}
#define FX_CHEB_K1A { \
  1.287716931284971, -0.29355526501238677, 0.04578781607810882, -0.0075606314967654195, \
  0.0012725129170005956, -0.0002159483044944044, 3.679893234585295e-05, -6.2852010326152186e-06, \
  1.0749808007083846e-06, -1.8401830928999913e-07, 3.151902199740263e-08, -5.4007938898647565e-09, \
  9.256899680411872e-10, -1.5869503264192334e-10, 2.7209976034987024e-11, -4.665992426162454e-12, \
  8.002016298795233e-13, -1.3724164584124254e-13, 2.353949688583712e-14, -4.037647655524712e-15, \
  6.925895800834045e-16, -1.1880559867658363e-16}
#define FX_CHEB_K0B { \
  1.2201515410329777, -0.0314481013119645, 0.0015698838857300533, -0.00012849549581627802, \
  1.39498137188765e-05, -1.8317555227191195e-06, 2.766813639445015e-07, -4.660489897687948e-08, \
  8.574034017414225e-09, -1.6975345093890614e-09, 3.5773972814003283e-10, -7.957489244477396e-11, \
  1.8559491149549264e-11, -4.514597883374519e-12, 1.1403405882073441e-12, -2.9800969231481784e-13, \
  8.032890775068375e-14, -2.2275133267462965e-14, 6.340076476276646e-15, -1.848593377920907e-15, \
  5.5120559994043335e-16, -1.6782311257549006e-16, 5.2103917776435543e-17, -1.6475805939842632e-17, \
  5.3004337711773354e-18}
#define FX_CHEB_K1B { \
  1.3603130952422213, 0.10392373657681724, -0.002857816859622779, 0.00019521551847135162, \
  -1.936197974166083e-05, 2.406484947837217e-06, -3.5019606030878126e-07, 5.7410841254500495e-08, \
  -1.0345762465678097e-08, 2.0150497551970347e-09, -4.1903547593419254e-10, 9.218315187605315e-11, \
  -2.129967838427791e-11, 5.139639673482343e-12, -1.2891739609498229e-12, 3.348419666052243e-13, \
  -8.976705182010146e-14, 2.4771544242195988e-14, -7.0198370892147685e-15, 2.038703166239861e-15, \
  -6.057047270643018e-16, 1.8380935752430455e-16, -5.689462849193648e-17, 1.7940510478863572e-17, \
  -5.7567444820733025e-18}
#define FX_CHEB_NA 22
#define FX_CHEB_NB 25

#define FX_EULER_GAMMA 0.5772156649015329

#ifdef __CUDACC__
__constant__ double FX_K0A_DEV[FX_CHEB_NA] = FX_CHEB_K0A;
__constant__ double FX_K1A_DEV[FX_CHEB_NA] = FX_CHEB_K1A;
__constant__ double FX_K0B_DEV[FX_CHEB_NB] = FX_CHEB_K0B;
__constant__ double FX_K1B_DEV[FX_CHEB_NB] = FX_CHEB_K1B;
#endif
static const double FX_K0A_HOST[FX_CHEB_NA] = FX_CHEB_K0A;
static const double FX_K1A_HOST[FX_CHEB_NA] = FX_CHEB_K1A;
static const double FX_K0B_HOST[FX_CHEB_NB] = FX_CHEB_K0B;
static const double FX_K1B_HOST[FX_CHEB_NB] = FX_CHEB_K1B;

/* Clenshaw's recurrence for sum_k c_k T_k(u), two series at once:
 * b_k = fma(2u, b_{k+1}, c_k - b_{k+2}), sum = fma(u, b_1, c_0 - b_2): the
 * subtraction runs beside the chain, which is one fused multiply-add per term. */
template <int N>
FX_HD void fx_clenshaw2(const double* c0, const double* c1, double u, double* s0, double* s1) {
  const double tu = 2.0 * u;
  double p1 = 0.0, p2 = 0.0, q1 = 0.0, q2 = 0.0;
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
  for (int k = N - 1; k >= 1; --k) {
    double p = fma_(tu, p1, c0[k] - p2);
    double q = fma_(tu, q1, c1[k] - q2);
    p2 = p1; p1 = p; q2 = q1; q1 = q;
  }
  *s0 = fma_(u, p1, c0[0] - p2);
  *s1 = fma_(u, q1, c1[0] - q2);
}

/* e^x K0(x), e^x K1(x) for 2 <= x < 1e4 (piece B) */
FX_HD void fx_k01x_B(double x, double* k0x, double* k1x) {
  double g0, g1;
#ifdef __CUDA_ARCH__
  fx_clenshaw2<FX_CHEB_NB>(FX_K0B_DEV, FX_K1B_DEV, (4.0 / x) - 1.0, &g0, &g1);
#else
  fx_clenshaw2<FX_CHEB_NB>(FX_K0B_HOST, FX_K1B_HOST, (4.0 / x) - 1.0, &g0, &g1);
#endif
  double rs = 1.0 / sqrt_(x);
  *k0x = g0 * rs;
  *k1x = g1 * rs;
}

/* e^x K0(x), e^x K1(x) for 0 < x < 1e4 */
FX_HD void fx_k01x(double x, double* k0x, double* k1x) {
  if (x < 1.0) {
    double t = 0.25 * x * x;
    double term = 1.0, i0 = 1.0, s0 = 0.0, hk = 0.0;
    double term1 = 1.0, i1 = 1.0;
    double s1 = (-FX_EULER_GAMMA) + (1.0 - FX_EULER_GAMMA);
#ifdef __CUDA_ARCH__
#pragma unroll
#endif
    for (int k = 1; k <= 15; ++k) {
      double kk = (double)k;
      term = term * (t / (kk * kk));
      hk = hk + 1.0 / kk;
      i0 = i0 + term;
      s0 = s0 + hk * term;
      term1 = term1 * (t / (kk * (kk + 1.0)));
      i1 = i1 + term1;
      s1 = s1 + (2.0 * (hk - FX_EULER_GAMMA) + 1.0 / (kk + 1.0)) * term1;
    }
    double lx = fx_log(0.5 * x);
    double k0 = -(lx + FX_EULER_GAMMA) * i0 + s0;
    double I1 = 0.5 * x * i1;
    double k1 = 1.0 / x + lx * I1 - 0.25 * x * s1;
    double ex = fx_exp(x);
    *k0x = k0 * ex;
    *k1x = k1 * ex;
    return;
  }
  if (x < 2.0) {
#ifdef __CUDA_ARCH__
    fx_clenshaw2<FX_CHEB_NA>(FX_K0A_DEV, FX_K1A_DEV, (2.0 * x) - 3.0, k0x, k1x);
#else
    fx_clenshaw2<FX_CHEB_NA>(FX_K0A_HOST, FX_K1A_HOST, (2.0 * x) - 3.0, k0x, k1x);
#endif
    return;
  }
  fx_k01x_B(x, k0x, k1x);
}

/* the reference's asymptotic series (safe_besselkx, src/eos.jl:30-33) */
FX_HD double fx_besselkx_asym(int nu, double x) {
  double mu = 4.0 * ((double)nu * (double)nu);
  double ix = 1.0 / (8.0 * x);
  double s = 1.0 + (mu - 1.0) * ix * (1.0 + (mu - 9.0) * ix / 2.0 * (1.0 + (mu - 25.0) * ix / 3.0));
  return sqrt_(FX_PI / (2.0 * x)) * s;
}

FX_HD double fx_besselkx(int nu, double x) {
  if (!(isfinite_(x) && x > 0.0)) return 0.0;
  if (x >= 1.0e4) return fx_besselkx_asym(nu, x);
  double k0, k1;
  fx_k01x(x, &k0, &k1);
  if (nu == 0) return k0;
  if (nu == 1) return k1;
  double km = k0, kc = k1;
  for (int n = 1; n < nu; ++n) {
    double kn = km + ((2.0 * n) / x) * kc;
    km = kc; kc = kn;
  }
  return kc;
}

/* e^x K2(x) (same bits as fx_besselkx(2, x)) */
FX_HD double fx_besselk2x(double x) {
  if (!(isfinite_(x) && x > 0.0)) return 0.0;
  if (x >= 1.0e4) return fx_besselkx_asym(2, x);
  double k0, k1;
  fx_k01x(x, &k0, &k1);
  return k0 + (2.0 / x) * k1;
}

}  // namespace fx
#endif
