/*
 * oracle/referees.cpp — the semi-analytic referees of the reference's dissipative
 * gates, integrated in C++ so the gate tests finish in seconds. TEST
 * INFRASTRUCTURE ONLY (loaded by tests/ through ctypes, like the oracle).
 *
 * Each referee is a fixed-step RK4 of a 0+1D (or de Sitter) ODE system, written
 * from the reference's own test files, with the transport coefficients taken
 * from the oracle's cell-level functions (the same code the relaxation runs),
 * exactly as the reference's referees call the solver's own coefficient
 * functions:
 *
 *   oracle_ref_bjorken_bulk    G0b: test/test_bjorken_bulk2d.jl:50-78
 *   oracle_ref_bjorken_shear   G2c: test/test_dissipation2d.jl:118-155
 *   oracle_ref_bjorken_dnmr    Gd1: test/analytic_referees.jl:97-123 and the
 *                              coefficient closures of test/test_dnmr2d.jl:47-60
 *   oracle_ref_gubser_viscous  G1v: test/test_gubser_viscous2d.jl:78-102
 *                              (= gubser_viscous, test/analytic_referees.jl:141-152)
 *   oracle_ref_m2_rhs_1d       Gm1: the 1+1D second moment on its transported triad,
 *                              hq_consistent_m2_rhs (src/hq_consistent_m2.jl:138-252),
 *                              all terms on; the 2+1D tensor source must reduce to it
 *                              (test/test_consistent_m22d.jl:85-198)
 */
#include <cmath>
#include <vector>
#include "oracle_core.h"

using namespace orc;

namespace {

/* T from e by bisection on [lo, hi] at fixed alpha (mu = alpha T), `iters` halvings;
 * `mu_zero` evaluates the EOS at mu = 0 (G0b's form: the charm tracer does not
 * enter e). Ties go to the upper half, as `em < e_target ? lo = mid : hi = mid`. */
double T_of_e(double e_target, double alpha, const fivo_params& p, double lo, double hi, int iters,
              bool mu_zero) {
  for (int k = 0; k < iters; ++k) {
    double mid = 0.5 * (lo + hi);
    double P, n, em;
    eos_Pne(mid, mu_zero ? 0.0 : alpha * mid, p, &P, &n, &em);
    if (em < e_target) lo = mid; else hi = mid;
  }
  return 0.5 * (lo + hi);
}

}  // namespace

extern "C" {

/* G0b: de/dtau = -(e + P + Pi)/tau, dPi/dtau = (-Pi - zeta/tau)/tau_Pi, from
 * T0, alpha (u = 0, Pi = 0) at tau0 to tauf in n RK4 steps. out = (e, Pi, T). */
void oracle_ref_bjorken_bulk(const fivo_params* p, double T0, double alpha, double tau0, double tauf, int64_t n,
                             double* out) {
  double P0, n0, e0;
  eos_Pne(T0, alpha * T0, *p, &P0, &n0, &e0);
  const double h = (tauf - tau0) / (double)n;
  auto rhs = [&](double tau, double e, double Pi, double* de, double* dPi) {
    double T = T_of_e(e, alpha, *p, 1e-4, 5.0, 200, true);
    double P, nn, ee;
    eos_Pne(T, alpha * T, *p, &P, &nn, &ee);
    double zb[2];
    cell_bulk_coeffs(T, alpha * T, nn, ee, P, *p, zb);
    *de = -(e + P + Pi) / tau;
    *dPi = (-Pi - zb[0] / tau) / std::fmax(zb[1], 1e-12);
  };
  double e = e0, Pi = 0.0, tau = tau0;
  for (int64_t k = 0; k < n; ++k) {
    double a1, b1, a2, b2, a3, b3, a4, b4;
    rhs(tau, e, Pi, &a1, &b1);
    rhs(tau + h / 2, e + h / 2 * a1, Pi + h / 2 * b1, &a2, &b2);
    rhs(tau + h / 2, e + h / 2 * a2, Pi + h / 2 * b2, &a3, &b3);
    rhs(tau + h, e + h * a3, Pi + h * b3, &a4, &b4);
    e += h / 6 * (a1 + 2 * a2 + 2 * a3 + a4);
    Pi += h / 6 * (b1 + 2 * b2 + 2 * b3 + b4);
    tau += h;
  }
  out[0] = e;
  out[1] = Pi;
  out[2] = T_of_e(e, alpha, *p, 1e-4, 5.0, 200, true);
}

/* G2c: viscous Bjorken with shear only. y = (e, pi^xx), pieta = -2 pi^xx,
 * de = -(e + P + pieta)/tau, tau_pi dpi^xx = -pi^xx (1 + delta_pi theta) + pi_NS^xx,
 * pi_NS^xx = -2 eta (-theta/3), theta = 1/tau. out = (e, pi^xx, pieta). */
void oracle_ref_bjorken_shear(const fivo_params* p, double T0, double alpha, double tau0, double tauf, int64_t nsub,
                              double* out) {
  double P0, n0, e0;
  eos_Pne(T0, alpha * T0, *p, &P0, &n0, &e0);
  const double dtau = (tauf - tau0) / (double)nsub;
  auto rhs = [&](double tau, const double* y, double* f) {
    double e = y[0], pxx = y[1];
    double T = T_of_e(e, alpha, *p, 1e-4, 5.0, 60, false);
    double mu = alpha * T;
    double P, nn, ee;
    eos_Pne(T, mu, *p, &P, &nn, &ee);
    double sh[3];
    cell_shear_coeffs(T, mu, nn, e, P, *p, sh);
    double th = 1.0 / tau;
    double pieta = -2.0 * pxx;
    double nsxx = -2.0 * sh[0] * (-th / 3.0);
    f[0] = -(e + P + pieta) / tau;
    f[1] = sh[1] > 0 ? (-pxx * (1.0 + sh[2] * th) + nsxx) / sh[1] : 0.0;
  };
  double y[2] = {e0, 0.0}, tau = tau0;
  for (int64_t k = 0; k < nsub; ++k) {
    double k1[2], k2[2], k3[2], k4[2], t[2];
    rhs(tau, y, k1);
    for (int j = 0; j < 2; ++j) t[j] = y[j] + (dtau / 2) * k1[j];
    rhs(tau + dtau / 2, t, k2);
    for (int j = 0; j < 2; ++j) t[j] = y[j] + (dtau / 2) * k2[j];
    rhs(tau + dtau / 2, t, k3);
    for (int j = 0; j < 2; ++j) t[j] = y[j] + dtau * k3[j];
    rhs(tau + dtau, t, k4);
    for (int j = 0; j < 2; ++j) y[j] = y[j] + (dtau / 6) * (k1[j] + 2 * k2[j] + 2 * k3[j] + k4[j]);
    tau += dtau;
  }
  out[0] = y[0];
  out[1] = y[1];
  out[2] = -2.0 * y[1];
}

/* Gd1: the 0+1D DNMR set with phi = -pi^eta_eta,
 *   de/dtau = -(e + P + Pi - phi)/tau
 *   tau_pi dphi/dtau = -phi + (4/3) eta/tau - (d_pp + t_pp/3) tau_pi phi/tau + (2/3) l_pP tau_pi Pi/tau
 *   tau_Pi dPi/dtau = -Pi - zeta/tau - d_PP tau_Pi Pi/tau + l_Pp tau_Pi phi/tau
 * with the coefficients of model p at T = T(e) (alpha fixed) and the second-order
 * ratios ratios5 = (d_pp, t_pp, l_pP, d_PP, l_Pp). out = (e, phi, Pi) at tau1. */
void oracle_ref_bjorken_dnmr(const fivo_params* p, double T0, double alpha, double tau0, double tau1, int64_t n,
                             const double* ratios5, double* out) {
  const double dpp = ratios5[0], tpp = ratios5[1], lpP = ratios5[2], dPP = ratios5[3], lPp = ratios5[4];
  auto eos_eP = [&](double T, double* e, double* P) {
    double nn;
    eos_Pne(T, alpha * T, *p, P, &nn, e);
  };
  auto Tof_e = [&](double e) {
    double lo = 0.01, hi = 2.0;
    for (int k = 0; k < 100; ++k) {
      double mid = (lo + hi) / 2, em, Pm;
      eos_eP(mid, &em, &Pm);
      if (em < e) lo = mid; else hi = mid;
    }
    return (lo + hi) / 2;
  };
  auto f = [&](double tau, const double* y, double* d) {
    double e = y[0], phi = y[1], Pi = y[2];
    double T = Tof_e(e);
    double ee, P;
    eos_eP(T, &ee, &P);
    double P_, nn, e_;
    eos_Pne(T, alpha * T, *p, &P_, &nn, &e_);
    double sh[3], bu[2];
    cell_shear_coeffs(T, alpha * T, nn, e_, P_, *p, sh);
    cell_bulk_coeffs(T, alpha * T, nn, e_, P_, *p, bu);
    double eta = sh[0], tp = sh[1];
    double zeta = bu[0], tb = p->enable_bulk ? bu[1] : 1.0;
    d[0] = -(e + P + Pi - phi) / tau;
    d[1] = tp > 0 ? (-phi + (4.0 / 3.0) * eta / tau - (dpp + tpp / 3) * tp * phi / tau +
                     (2.0 / 3.0) * lpP * tp * Pi / tau) / tp
                  : 0.0;
    d[2] = (tb > 0 && zeta > 0) ? (-Pi - zeta / tau - dPP * tb * Pi / tau + lPp * tb * phi / tau) / tb : 0.0;
  };
  double e0, P0;
  eos_eP(T0, &e0, &P0);
  double y[3] = {e0, 0.0, 0.0};
  const double h = (tau1 - tau0) / (double)n;
  double t = tau0;
  for (int64_t i = 1; i <= n; ++i) {
    double k1[3], k2[3], k3[3], k4[3], z[3];
    f(t, y, k1);
    for (int j = 0; j < 3; ++j) z[j] = y[j] + (h / 2) * k1[j];
    f(t + h / 2, z, k2);
    for (int j = 0; j < 3; ++j) z[j] = y[j] + (h / 2) * k2[j];
    f(t + h / 2, z, k3);
    for (int j = 0; j < 3; ++j) z[j] = y[j] + h * k3[j];
    f(t + h, z, k4);
    for (int j = 0; j < 3; ++j) y[j] = y[j] + (h / 6) * (k1[j] + 2 * k2[j] + 2 * k3[j] + k4[j]);
    t = tau0 + (double)i * h;
  }
  out[0] = y[0];
  out[1] = y[1];
  out[2] = y[2];
}

/* G1v: the de Sitter system of viscous Gubser flow, forward in rho,
 *   dT/drho = -(2/3) T tanh rho + (1/3) T pibar tanh rho
 *   dpibar/drho = -(4/3) pibar^2 tanh rho - pibar/tau_pi + (4/15) tanh rho,  tau_pi = 5 (eta/s)/(T/hbar c)
 * from T(rhomin) = TH0 cosh(rhomin)^(-2/3), pibar(rhomin) = the Navier-Stokes value
 * (seed_ns) or 0. Th and pb receive the n+1 samples on the uniform rho grid. */
void oracle_ref_gubser_viscous(double etas, double TH0, double rhomin, double rhomax, int64_t n, int seed_ns,
                               double* Th, double* pb) {
  const double invfmGeV = 1.0 / 0.1973269804;
  const double h = (rhomax - rhomin) / (double)n;
  auto f = [&](double rho, double T, double q, double* dT, double* dq) {
    double th = std::tanh(rho);
    double tp = etas > 0 ? 5 * etas / (std::fmax(T, 1e-12) * invfmGeV) : 0.0;
    *dT = -(2.0 / 3.0) * T * th + (1.0 / 3.0) * T * q * th;
    *dq = etas > 0 ? -(4.0 / 3.0) * q * q * th - q / tp + (4.0 / 15.0) * th : 0.0;
  };
  Th[0] = TH0 * std::pow(std::cosh(rhomin), -2.0 / 3.0);
  pb[0] = (etas > 0 && seed_ns) ? (4.0 / 3.0) * etas * std::tanh(rhomin) / (Th[0] * invfmGeV) : 0.0;
  for (int64_t i = 0; i < n; ++i) {
    double rho = rhomin + (double)i * h;   /* range(rhomin, rhomax; length = n+1)[i+1] */
    double T = Th[i], q = pb[i];
    double a1, b1, a2, b2, a3, b3, a4, b4;
    f(rho, T, q, &a1, &b1);
    f(rho + h / 2, T + h / 2 * a1, q + h / 2 * b1, &a2, &b2);
    f(rho + h / 2, T + h / 2 * a2, q + h / 2 * b2, &a3, &b3);
    f(rho + h, T + h * a3, q + h * b3, &a4, &b4);
    Th[i + 1] = T + h / 6 * (a1 + 2 * a2 + 2 * a3 + a4);
    pb[i + 1] = q + h / 6 * (b1 + 2 * b2 + 2 * b3 + b4);
  }
}

/* ---- cell-level functions of the relaxation (the oracle's own code paths) ---- */
/* Gm1's referee. in[27] = (tau, r, ur, T, dtT, drT, drur, dtur, p_l, p_phi, PiQ, nu,
 * dtalpha, dralpha, dtnu, drnu, drp_l, drp_phi, drPiQ, n, tau_n, Ds, h, hp, tau_M, eta_M, m);
 * out[3] = (dp_l, dp_phi, dPiQ) / dtau. The coefficient closed forms are the 2+1D
 * ones (hq_m2_coeffs and hq_m2_coeffs_2d are the same expressions). */
void oracle_ref_m2_rhs_1d(const double* in, double* out) {
  const double tau = in[0], r = in[1], ur = in[2], T = in[3], dtT = in[4], drT = in[5], drur = in[6];
  const double dtur = in[7], pl = in[8], pf = in[9], PiQ = in[10], nu = in[11], dta = in[12], dra = in[13];
  const double dtnu = in[14], drnu = in[15], n = in[19], tn = in[20], Ds = in[21], h = in[22], hp = in[23];
  const double tM = in[24], etaM = in[25], m = in[26];
  const double Tm = std::fmax(T, 1e-20);
  const double ut = std::sqrt(1.0 + ur * ur);
  if (!(tM > 0.0 && r > 0.0)) { out[0] = out[1] = out[2] = 0.0; return; }
  const double peta = -(pl + pf);
  /* background kinematics on the triad (l, phi, eta) */
  const double Dlur = ur * dtur + ut * drur;
  const double thl = Dlur / ut, thf = ur / r, the = ut / tau;
  const double th = thl + thf + the;
  const double sl = thl - th / 3.0, sf = thf - th / 3.0, se = the - th / 3.0;
  const double al = (ut * dtur + ur * drur) / ut;
  const double nul = nu / ut;
  /* the current's gradient on the triad */
  const double Dlnu = ur * dtnu + ut * drnu;
  const double gll = Dlnu / ut - ur * nu * Dlur / (ut * ut * ut);
  const double gff = nu / r;
  const double anu = al * nul;
  const double thnu = (ur / ut) * dtnu + nu * dtur / (ut * ut * ut) + drnu + ur * nu / (ut * tau) + nu / r;
  const double trnu = thnu - anu;
  const double snl = gll - trnu / 3.0, snf = gff - trnu / 3.0;
  const double etaQ = etaM, zetaQ = (5.0 / 3.0) * etaQ;
  double cf[5];
  m2_coeffs(Tm, n, tn, Ds, h, m, cf);   /* dlnC, etabar, lambda_a, A, A/B */
  const double DlnT = (ut * dtT + ur * drT) / Tm;
  const double DlnC = cf[0] * DlnT;
  const double DlTh = (h + Tm * hp) * (ur * dtT + ut * drT);
  const double ps = pl * sl + pf * sf + peta * se;
  const double geo = tM * ((5.0 / 3.0) * th + DlnC);
  const double rank1 = 2.0 * cf[2] * al * nul + (Ds / Tm) * nul * DlTh;
  const double srcl = pl + 2.0 * etaQ * snl + geo * pl + 2.0 * tM * (pl * sl - ps / 3.0) + 2.0 * tM * PiQ * sl +
                      2.0 * cf[1] * sl + rank1 * (2.0 / 3.0);
  const double srcf = pf + 2.0 * etaQ * snf + geo * pf + 2.0 * tM * (pf * sf - ps / 3.0) + 2.0 * tM * PiQ * sf +
                      2.0 * cf[1] * sf + rank1 * (-1.0 / 3.0);
  double srcB = PiQ + zetaQ * thnu + geo * PiQ + (2.0 / 3.0) * tM * ps + cf[1] * (cf[4] * DlnT + (5.0 / 3.0) * th) +
                (Ds * cf[3] / (3.0 * Tm)) * anu + (5.0 / 6.0) * (Ds / Tm) * nul * DlTh;
  srcB += cf[1] * (ut * dta + ur * dra);
  const double den = tM * ut;
  out[0] = -(tM * ur * in[16] + srcl) / den;
  out[1] = -(tM * ur * in[17] + srcf) / den;
  out[2] = -(tM * ur * in[18] + srcB) / den;
}

void oracle_shear_coeffs(const fivo_params* p, double T, double mu, double n, double e, double P, double* out3) {
  cell_shear_coeffs(T, mu, n, e, P, *p, out3);
}
void oracle_bulk_coeffs(const fivo_params* p, double T, double mu, double n, double e, double P, double* out2) {
  cell_bulk_coeffs(T, mu, n, e, P, *p, out2);
}
void oracle_diff_tauN(const fivo_params* p, double T, double alpha, double DsT, double tauD, double* out2) {
  cell_diff_tauN(T, alpha, *p, DsT, tauD, &out2[0], &out2[1]);
}
double oracle_vacuum_weight(const fivo_params* p, double n) { return cell_vacuum_weight(n, *p); }
double oracle_entropy(double T, double mu, double n, double e, double P) { return cell_entropy(T, mu, n, e, P); }
/* k rows of (ux, uy, ut, tau, theta, ax, ay, dxux, dxuy, dyux, dyuy, eta) -> k rows of 4 */
void oracle_ns_shear_target(int64_t k, const double* in12, double* out4) {
  for (int64_t i = 0; i < k; ++i) cell_ns_shear_target(in12 + 12 * i, out4 + 4 * i);
}
/* k rows of (ux, uy, ut, pixx, pixy, piyy) -> k values */
void oracle_project_traceless(int64_t k, const double* in6, double* out) {
  for (int64_t i = 0; i < k; ++i) {
    const double* q = in6 + 6 * i;
    out[i] = cell_project_traceless(q[0], q[1], q[2], q[3], q[4], q[5]);
  }
}
/* k rows of (ux, uy, ut, dxa, dya, dta, kappa) -> k rows of 2 */
void oracle_ns_diffusion_target(int64_t k, const double* in7, double* out2) {
  for (int64_t i = 0; i < k; ++i) {
    const double* q = in7 + 7 * i;
    cell_ns_diffusion_target(q[0], q[1], q[2], q[3], q[4], q[5], q[6], out2 + 2 * i);
  }
}
/* k rows of (ux, uy, pxx, pxy, pyy, peta, sxx, sxy, syy, seta) -> k rows of (pi:sigma, cxx, cxy, cyy) */
void oracle_pi_sigma(int64_t k, const double* in10, double* out4) {
  for (int64_t i = 0; i < k; ++i) cell_pi_sigma(in10 + 10 * i, out4 + 4 * i);
}
/* k rows of (ux, uy, ut, tau, pixx, pixy, piyy, pieta) -> k rows of (tt, tx, ty, xx, xy, yy, etaeta) */
void oracle_shear_tensor(int64_t k, const double* in8, double* out7) {
  for (int64_t i = 0; i < k; ++i) {
    const double* q = in8 + 8 * i;
    cell_shear_tensor(q[0], q[1], q[2], q[3], q[4], q[5], q[6], q[7], out7 + 7 * i);
  }
}

}  /* extern "C" */
