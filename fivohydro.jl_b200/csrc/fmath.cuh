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
 *            34-node trapezoidal rule (step 1/5) on DLMF 10.32.8 with t = s^2
 *            for x >= 1; <= 6e-16 relative to 40-digit references.
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
  if (k > 1023) { p = p * 8.98846567431158e307; k -= 1023; if (k > 1023) k = 1023; }
  if (k < -1022) {
    p = p * from_bits((uint64_t)(k + 1000 + 1023) << 52);
    return p * from_bits((uint64_t)(1023 - 1000) << 52);
  }
  return p * from_bits((uint64_t)(k + 1023) << 52);
}

FX_HD double fx_exp(double x) {
  if (isnan_(x)) return x;
  if (x > 709.782712893384) return inf_();
  if (x < -745.1332191019412) return 0.0;
  double kd = rint_(x * 1.4426950408889634);
  double r = fma_(-kd, 0.6931471803691238, x);
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
  return scale2(p, (int)kd);
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

/* trapezoid nodes s_k^2 = (k/5)^2 and weights (1/5) e^{-s_k^2}/sqrt(pi) (doubled for k > 0) */
#define FX_BESSEL_S2 { \
  0.0, 0.04, 0.16, 0.36, 0.64, 1.0, 1.44, 1.96, 2.56, 3.24, 4.0, 4.84, 5.76, 6.76, \
  7.84, 9.0, 10.24, 11.56, 12.96, 14.44, 16.0, 17.64, 19.36, 21.16, 23.04, 25.0, \
  27.04, 29.16, 31.36, 33.64, 36.0, 38.44, 40.96, 43.56}
#define FX_BESSEL_W { \
  0.11283791670955126, 0.21682695742097263, 0.19230825976786156, 0.15744868634285744, \
  0.11899715725149379, 0.08302149948411894, 0.05346886940070783, 0.03178834153545557, \
  0.017445811726789072, 0.008838344666402213, 0.004133397070818411, 0.001784431012983241, \
  0.0007111297361755495, 0.00026161000994465633, 8.884158884113332e-05, 2.785061038934957e-05, \
  8.059527106647123e-06, 2.1529842073361357e-06, 5.309193689433173e-07, 1.2085725786444936e-07, \
  2.5396469343733115e-08, 4.926408197336689e-09, 8.821529389366844e-10, 1.4581890004763904e-10, \
  2.225052137962172e-11, 3.134173306203467e-12, 4.075325146752109e-13, 4.89167914078347e-14, \
  5.420134984939562e-15, 5.543942072256747e-16, 5.2346024784985296e-17, 4.5625240909092945e-18, \
  3.670988941398298e-19, 2.726574842629012e-20}

#define FX_EULER_GAMMA 0.5772156649015329

#ifdef __CUDACC__
__constant__ double FX_S2_DEV[34] = FX_BESSEL_S2;
__constant__ double FX_W_DEV[34] = FX_BESSEL_W;
#endif
static const double FX_S2_HOST[34] = FX_BESSEL_S2;
static const double FX_W_HOST[34] = FX_BESSEL_W;

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
#ifdef __CUDA_ARCH__
  const double* S2 = FX_S2_DEV;
  const double* W = FX_W_DEV;
#else
  const double* S2 = FX_S2_HOST;
  const double* W = FX_W_HOST;
#endif
  double inv2x = 1.0 / (2.0 * x);
  double a0 = 0.0, a1 = 0.0;
#ifdef __CUDA_ARCH__
#pragma unroll 2
#endif
  for (int k = 33; k >= 0; --k) {
    double s2 = S2[k];
    double q = sqrt_(1.0 + s2 * inv2x);
    a0 = a0 + W[k] / q;
    a1 = a1 + (W[k] * s2) * q;
  }
  double pre = sqrt_(FX_PI / (2.0 * x));
  *k0x = pre * a0;
  *k1x = pre * (2.0 * a1);
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
