/*
 * oracle/oracle_core.cpp — CPU restatement of the reference's 2+1D stage.
 * TEST INFRASTRUCTURE ONLY (see oracle_core.h). Every function follows the Julia
 * function named in its comment, with Julia's evaluation order.
 */
#include "oracle_core.h"

#include <algorithm>
#include <cstdio>
#include <cstring>

namespace orc {

/* ============================== EOS (src/eos.jl) ============================== */

static inline double hq_mass(const fivo_params& e) { return e.m_hq; }

/* ConformalHQEOS eos_Pne, src/eos.jl:53-84 */
static void conformal_Pne(double T, double mu, const fivo_params& e, double* P, double* n, double* en) {
  T = o_max(T, T_MIN);
  double aSB = (PI2 / 90.0) * e.g_eff;                 /* a_SB, src/eos.jl:50 */
  double Plight = (aSB * o_pow4(T)) * FMGEV3;
  double elight = 3.0 * Plight;
  double m = hq_mass(e), g = e.g_hq;
  double x = m / T;
  if (!o_isfinite(x) || x <= 0.0) { *P = Plight; *n = 0.0; *en = elight; return; }
  double A = (g * (m * m)) / (2.0 * PI2);
  double K2x = o_besselkx(2, x);
  double K1x = o_besselkx(1, x);
  double exp_arg = (mu - m) / T;
  double Efac = o_exp(exp_arg);
  double n_hq = ((A * T) * Efac) * K2x;
  double P_hq = ((A * (T * T)) * Efac) * K2x;
  double e_hq = ((A * (T * T)) * Efac) * ((3.0 * K2x) + (x * K1x));
  if (e.hq_times_fmGeV3) { n_hq *= FMGEV3; P_hq *= FMGEV3; e_hq *= FMGEV3; }
  *P = Plight + P_hq; *n = n_hq; *en = elight + e_hq;
}

static const double LK0 = 0.0005624486560000001, LK1 = 0.003652264, LK2 = 0.023716,
                    LK3 = 0.154, LK4 = 5.208957878352717;

/* light_P, src/eos.jl:357-377 */
static double light_P(double T, const fivo_params& e) {
  T = o_max(T, T_MIN);
  double A = 0.01 * (e.lhrg_d * e.lhrg_d);
  double B = 0.1 * (e.lhrg_c * e.lhrg_c);
  double E = (-(A / (T * T))) - (B / T);
  E = o_clamp(E, -700.0, 700.0);
  double expE = o_exp(E);
  double T2 = T * T, T3 = (T * T) * T, T4 = o_pow4(T);
  double N = ((((LK0 * e.lhrg_a[3]) + ((LK1 * e.lhrg_a[2]) * T)) + ((LK2 * e.lhrg_a[1]) * T2)) +
              ((LK3 * e.lhrg_a[0]) * T3)) + (LK4 * T4);
  double D = ((((LK0 * e.lhrg_b[3]) + ((LK1 * e.lhrg_b[2]) * T)) + ((LK2 * e.lhrg_b[1]) * T2)) +
              ((LK3 * e.lhrg_b[0]) * T3)) + T4;
  return ((FMGEV3 * expE) * T4) * (N / D);
}

/* light_dP_dT, src/eos.jl:379-412 */
static double light_dP_dT(double T, const fivo_params& e) {
  T = o_max(T, T_MIN);
  double A = 0.01 * (e.lhrg_d * e.lhrg_d);
  double B = 0.1 * (e.lhrg_c * e.lhrg_c);
  double E = (-(A / (T * T))) - (B / T);
  E = o_clamp(E, -700.0, 700.0);
  double expE = o_exp(E);
  double T2 = T * T, T3 = (T * T) * T, T4 = o_pow4(T);
  double Ep = ((2.0 * A) / T3) + (B / T2);
  double N = ((((LK0 * e.lhrg_a[3]) + ((LK1 * e.lhrg_a[2]) * T)) + ((LK2 * e.lhrg_a[1]) * T2)) +
              ((LK3 * e.lhrg_a[0]) * T3)) + (LK4 * T4);
  double D = ((((LK0 * e.lhrg_b[3]) + ((LK1 * e.lhrg_b[2]) * T)) + ((LK2 * e.lhrg_b[1]) * T2)) +
              ((LK3 * e.lhrg_b[0]) * T3)) + T4;
  double Np = (((LK1 * e.lhrg_a[2]) + (((2.0 * LK2) * e.lhrg_a[1]) * T)) +
               (((3.0 * LK3) * e.lhrg_a[0]) * T2)) + ((4.0 * LK4) * T3);
  double Dp = (((LK1 * e.lhrg_b[2]) + (((2.0 * LK2) * e.lhrg_b[1]) * T)) +
               (((3.0 * LK3) * e.lhrg_b[0]) * T2)) + (4.0 * T3);
  double G = T4 * N, H = D;
  double Gp = ((4.0 * T3) * N) + (T4 * Np);
  double Hp = Dp;
  double F = G / H;
  double Fp = ((Gp * H) - (G * Hp)) / (H * H);
  return (FMGEV3 * expE) * (Fp + (F * Ep));
}

/* light_d2P_dT2, src/eos.jl:414-463 */
static double light_d2P_dT2(double T, const fivo_params& e) {
  T = o_max(T, T_MIN);
  double A = 0.01 * (e.lhrg_d * e.lhrg_d);
  double B = 0.1 * (e.lhrg_c * e.lhrg_c);
  double E = (-(A / (T * T))) - (B / T);
  E = o_clamp(E, -700.0, 700.0);
  double expE = o_exp(E);
  double T2 = T * T, T3 = (T * T) * T, T4 = o_pow4(T);
  double Ep = ((2.0 * A) / T3) + (B / T2);
  double Epp = ((-6.0 * A) / T4) - ((2.0 * B) / T3);
  double N = ((((LK0 * e.lhrg_a[3]) + ((LK1 * e.lhrg_a[2]) * T)) + ((LK2 * e.lhrg_a[1]) * T2)) +
              ((LK3 * e.lhrg_a[0]) * T3)) + (LK4 * T4);
  double D = ((((LK0 * e.lhrg_b[3]) + ((LK1 * e.lhrg_b[2]) * T)) + ((LK2 * e.lhrg_b[1]) * T2)) +
              ((LK3 * e.lhrg_b[0]) * T3)) + T4;
  double Np = (((LK1 * e.lhrg_a[2]) + (((2.0 * LK2) * e.lhrg_a[1]) * T)) +
               (((3.0 * LK3) * e.lhrg_a[0]) * T2)) + ((4.0 * LK4) * T3);
  double Dp = (((LK1 * e.lhrg_b[2]) + (((2.0 * LK2) * e.lhrg_b[1]) * T)) +
               (((3.0 * LK3) * e.lhrg_b[0]) * T2)) + (4.0 * T3);
  double Npp = (((2.0 * LK2) * e.lhrg_a[1]) + (((6.0 * LK3) * e.lhrg_a[0]) * T)) + ((12.0 * LK4) * T2);
  double Dpp = (((2.0 * LK2) * e.lhrg_b[1]) + (((6.0 * LK3) * e.lhrg_b[0]) * T)) + (12.0 * T2);
  double G = T4 * N, H = D;
  double Gp = ((4.0 * T3) * N) + (T4 * Np);
  double Hp = Dp;
  double Gpp = (((12.0 * T2) * N) + ((8.0 * T3) * Np)) + (T4 * Npp);
  double Hpp = Dpp;
  double F = G / H;
  double Fp = ((Gp * H) - (G * Hp)) / (H * H);
  double Q = (Gp * H) - (G * Hp);
  double Qp = (Gpp * H) - (G * Hpp);
  double Fpp = ((Qp * H) - ((2.0 * Q) * Hp)) / ((H * H) * H);
  return (FMGEV3 * expE) * ((Fpp + ((2.0 * Fp) * Ep)) + (F * (Epp + (Ep * Ep))));
}

/* light_e, src/eos.jl:466-470 */
static double light_e(double T, const fivo_params& e) {
  double P = light_P(T, e);
  double dP = light_dP_dT(T, e);
  return (-P) + (T * dP);
}

/* _lhrg_assemble_2d, src2d/primrec2d.jl:134-154 */
static void lhrg_assemble(double T, double mu, const fivo_params& e, double x, double Pl,
                          double el, double K2x, double* P, double* n, double* en) {
  if (!o_isfinite(x) || x <= 0.0) { *P = Pl; *n = 0.0; *en = el; return; }
  double m = hq_mass(e), g = e.g_hq;
  double A = ((e.canon_factor * g) * (m * m)) / (2.0 * PI2);
  double z = (mu - m) / T;
  z = o_clamp(z, -700.0, 700.0);
  double Efac = o_exp(z);
  double n_hq = ((A * T) * Efac) * K2x;
  double P_hq = 0.0, e_hq = 0.0;
  if (e.hq_times_fmGeV3) { n_hq *= FMGEV3; P_hq *= FMGEV3; e_hq *= FMGEV3; }
  *P = Pl + P_hq; *n = n_hq; *en = el + e_hq;
}

static inline double lhrg_x(double T, const fivo_params& e) { return o_min(hq_mass(e) / T, 100000.0); }
static inline double lhrg_K2(double x) { return (!o_isfinite(x) || x <= 0.0) ? 0.0 : o_besselkx(2, x); }

/* eos_Pne (src/eos.jl:53-84, 483-519). With this file's Bessel K, the LatticeHRG
 * eos_Pne and eos_Pne_2d (src2d/primrec2d.jl:170-176) are the same arithmetic. */
void eos_Pne(double T, double mu, const fivo_params& e, double* P, double* n, double* en) {
  if (e.eos_kind == FIVO_EOS_CONFORMAL_HQ) { conformal_Pne(T, mu, e, P, n, en); return; }
  T = o_max(T, T_MIN);
  double Pl = light_P(T, e);
  double el = light_e(T, e);
  double x = lhrg_x(T, e);
  lhrg_assemble(T, mu, e, x, Pl, el, lhrg_K2(x), P, n, en);
}

/* eos_Pne_2d with the T-keyed memo, src2d/primrec2d.jl:178-197 */
static void eos_Pne_2d_cached(double T, double mu, const fivo_params& e, EOSCache* c,
                              double* P, double* n, double* en) {
  if (e.eos_kind != FIVO_EOS_LATTICE_HRG || c == nullptr) { eos_Pne(T, mu, e, P, n, en); return; }
  T = o_max(T, T_MIN);
  int k = -1;
  for (int j = 0; j < 4; ++j) if (c->T[j] == T) { k = j; break; }
  double x = lhrg_x(T, e);
  if (k < 0) {
    k = c->next;
    c->next = (k == 3) ? 0 : k + 1;
    double Pl = light_P(T, e);
    c->T[k] = T;
    c->Pl[k] = Pl;
    c->el[k] = (-Pl) + (T * light_dP_dT(T, e));
    c->K2[k] = lhrg_K2(x);
  }
  lhrg_assemble(T, mu, e, x, c->Pl[k], c->el[k], c->K2[k], P, n, en);
}

/* eos_Pe_2d, src2d/primrec2d.jl:209-231 */
static void eos_Pe_2d(double T, double mu, const fivo_params& e, double* P, double* en) {
  if (e.eos_kind != FIVO_EOS_LATTICE_HRG) { double n; eos_Pne(T, mu, e, P, &n, en); return; }
  T = o_max(T, T_MIN);
  double Pl = light_P(T, e);
  double el = (-Pl) + (T * light_dP_dT(T, e));
  double x = hq_mass(e) / T;
  x = o_min(x, 100000.0);
  if (!o_isfinite(x) || x <= 0.0) { *P = Pl; *en = el; return; }
  double P_hq = 0.0, e_hq = 0.0;
  if (e.hq_times_fmGeV3) { P_hq *= FMGEV3; e_hq *= FMGEV3; }
  *P = Pl + P_hq; *en = el + e_hq;
}

/* eos_cs2, src/eos.jl:51 and 473-478 */
double eos_cs2(double T, double mu, const fivo_params& e) {
  (void)mu;
  if (e.eos_kind == FIVO_EOS_CONFORMAL_HQ) return 1.0 / 3.0;
  T = o_max(T, T_MIN);
  double Pp = light_dP_dT(T, e);
  double Ppp = light_d2P_dT2(T, e);
  return (Ppp == 0.0) ? (1.0 / 3.0) : (Pp / (T * Ppp));
}

/* eos_has_charge_2d, src2d/primrec2d.jl:273-276 */
static inline bool eos_has_charge(const fivo_params& e) {
  return e.eos_kind == FIVO_EOS_CONFORMAL_HQ ? (e.g_hq > 0.0) : true;
}

/* eos_entropy, src/eos.jl:306-310 */
static inline double eos_entropy(double T, double mu, double n, double e, double P) {
  T = o_max(T, T_MIN);
  double s = ((e + P) - (mu * n)) / T;
  return o_max(s, 0.0);
}

/* ============================ shear algebra (src2d/shear2d.jl) ============================ */

struct PiC { double tt, tx, ty, xx, xy, yy, etaeta; };

/* shear_tensor_contravariant_2d, src2d/shear2d.jl:61-74 */
static inline PiC shear_tensor(double ux, double uy, double ut, double tau, double pixx,
                               double pixy, double piyy, double pieta) {
  double iu = safe_inv(ut);
  double tx = ((ux * pixx) + (uy * pixy)) * iu;
  double ty = ((ux * pixy) + (uy * piyy)) * iu;
  double tt = ((ux * tx) + (uy * ty)) * iu;
  PiC r{tt, tx, ty, pixx, pixy, piyy, pieta * safe_inv(tau * tau)};
  return r;
}

/* shear_constraint_residual_2d, src2d/shear2d.jl:88-101 */
static inline void shear_residual(double ux, double uy, double ut, double pixx, double pixy,
                                  double piyy, double pieta, double* R, double* rel) {
  double iu = safe_inv(ut);
  double tx = ((ux * pixx) + (uy * pixy)) * iu;
  double ty = ((ux * pixy) + (uy * piyy)) * iu;
  double tt = ((ux * tx) + (uy * ty)) * iu;
  double r = (((-tt) + pixx) + piyy) + pieta;
  double scale = o_max(o_max(o_max(o_max(std::fabs(tt), std::fabs(pixx)), std::fabs(piyy)),
                             std::fabs(pieta)), std::fabs(pixy));
  *R = r;
  *rel = scale > TINY ? std::fabs(r) / scale : 0.0;
}

/* project_shear_traceless_2d, src2d/shear2d.jl:131-142 */
static inline double project_traceless(double ux, double uy, double ut, double pixx, double pixy,
                                       double piyy) {
  double iu = safe_inv(ut);
  double tx = ((ux * pixx) + (uy * pixy)) * iu;
  double ty = ((ux * pixy) + (uy * piyy)) * iu;
  double tt = ((ux * tx) + (uy * ty)) * iu;
  return (tt - pixx) - piyy;
}

/* nu_tau_2d, src2d/shear2d.jl:180-181 */
static inline double nu_tau(double ux, double uy, double ut, double nux, double nuy) {
  return ((ux * nux) + (uy * nuy)) * safe_inv(ut);
}

/* ======================= primitive recovery (src2d/primrec2d.jl) ======================= */

/* solve_gauss_n!, src2d/primrec2d.jl:33-87. J row-major n x n; returns false on failure. */
static bool solve_gauss_n(double* delta, const double J[4][4], const double* F, int n) {
  double A[4][5];
  for (int r = 0; r < n; ++r) {
    for (int c = 0; c < n; ++c) A[r][c] = J[r][c];
    A[r][n] = -F[r];
  }
  double smax = 0.0;
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c) smax = o_max(smax, std::fabs(A[r][c]));
  if (!o_isfinite(smax) || smax == 0.0) return false;
  double pivtol = 1e-15 * smax;
  for (int k = 0; k < n; ++k) {
    int p = k;
    double amax = std::fabs(A[k][k]);
    for (int r = k + 1; r < n; ++r)
      if (std::fabs(A[r][k]) > amax) { amax = std::fabs(A[r][k]); p = r; }
    if (amax < pivtol) return false;
    if (p != k)
      for (int c = k; c <= n; ++c) { double t = A[k][c]; A[k][c] = A[p][c]; A[p][c] = t; }
    double invp = 1.0 / A[k][k];
    for (int r = k + 1; r < n; ++r) {
      double f = A[r][k] * invp;
      if (f == 0.0) continue;
      for (int c = k; c <= n; ++c) A[r][c] -= f * A[k][c];
    }
  }
  for (int r = n - 1; r >= 0; --r) {
    double s = A[r][n];
    for (int c = r + 1; c < n; ++c) s -= A[r][c] * delta[c];
    delta[r] = s / A[r][r];
  }
  for (int r = 0; r < n; ++r) if (!o_isfinite(delta[r])) return false;
  return true;
}

static double LOG_T_MIN() { static const double v = o_log(T_MIN); return v; }
static double LOG_T_SOLVE_MAX() { static const double v = o_log(T_SOLVE_MAX); return v; }
static double LOG_SEED_T() { static const double v = o_log(o_max(0.15, T_MIN)); return v; }

/* _invert_e_for_T, src2d/primrec2d.jl:300-314 */
static double invert_e_for_T(double e_target, double phi, const fivo_params& e) {
  double lo = LOG_T_MIN(), hi = LOG_T_SOLVE_MAX();
  if (e_target <= 0.0) return lo;
  for (int it = 0; it < 60; ++it) {
    double mid = 0.5 * (lo + hi);
    double Tm = o_exp(mid);
    double Pm, em;
    eos_Pe_2d(Tm, hq_mass(e) + (Tm * phi), e, &Pm, &em);
    if (!o_isfinite(em) || em > e_target) hi = mid; else lo = mid;
  }
  return 0.5 * (lo + hi);
}

/* seed_from_conserved_2d, src2d/primrec2d.jl:323-347 */
static void seed_from_conserved(double E, double Sx, double Sy, double phi, const fivo_params& e,
                                double* yT, double* ux, double* uy) {
  double M = std::sqrt((Sx * Sx) + (Sy * Sy));
  if (!o_isfinite(E) || E <= 0.0) { *yT = LOG_SEED_T(); *ux = 0.0; *uy = 0.0; return; }
  double P = E / 3.0;
  double y = LOG_SEED_T();
  double v = 0.0;
  for (int it = 0; it < 3; ++it) {
    double denom = E + P;
    v = denom > TINY ? o_min(M / denom, 0.999999) : 0.0;
    double ee = (denom * (1.0 - (v * v))) - P;
    if (ee <= 0.0) ee = o_max(E, TINY);
    y = invert_e_for_T(ee, phi, e);
    double T = o_exp(y);
    double Pn, en;
    eos_Pe_2d(T, hq_mass(e) + (T * phi), e, &Pn, &en);
    if (!o_isfinite(Pn)) break;
    P = Pn;
  }
  double gam = 1.0 / std::sqrt(o_max(1.0 - (v * v), 1e-16));
  double us = gam * v;
  double sx = M > TINY ? (us * Sx) / M : 0.0;
  double sy = M > TINY ? (us * Sy) / M : 0.0;
  *yT = y;
  *ux = o_clamp(sx, -U_CAP_2D, U_CAP_2D);
  *uy = o_clamp(sy, -U_CAP_2D, U_CAP_2D);
}

struct CellCons { double D, Sx, Sy, E, nux, nuy, Pi, pixx, pixy, piyy, pieta, tau; };

/* evalF_2d!, src2d/primrec2d.jl:360-390 */
static void evalF(double* F, const double* x, const CellCons& c, const fivo_params& e,
                  bool ncharge, EOSCache* cache) {
  double yT = x[0], phi = x[1], ux = x[2], uy = x[3];
  if (!(o_isfinite(yT) && o_isfinite(phi) && o_isfinite(ux) && o_isfinite(uy))) {
    F[0] = F[1] = F[2] = F[3] = O_INF; return;
  }
  double T = o_exp(yT);
  double mu = hq_mass(e) + (T * phi);
  double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
  double P, n, en;
  eos_Pne_2d_cached(T, mu, e, cache, &P, &n, &en);
  if (!(o_isfinite(P) && o_isfinite(n) && o_isfinite(en))) { F[0] = F[1] = F[2] = F[3] = O_INF; return; }
  double weff = (en + P) + c.Pi;
  double Ptot = P + c.Pi;
  PiC Pc = shear_tensor(ux, uy, ut, c.tau, c.pixx, c.pixy, c.piyy, c.pieta);
  F[0] = ncharge ? (((n * ut) + nu_tau(ux, uy, ut, c.nux, c.nuy)) - c.D) : 0.0;
  F[1] = (((weff * ut) * ux) + Pc.tx) - c.Sx;
  F[2] = (((weff * ut) * uy) + Pc.ty) - c.Sy;
  F[3] = ((((weff * ut) * ut) - Ptot) + Pc.tt) - c.E;
}

static inline bool all_finite4(const double* F) {
  return o_isfinite(F[0]) && o_isfinite(F[1]) && o_isfinite(F[2]) && o_isfinite(F[3]);
}

/* _solve_phi_bisect, src2d/primrec2d.jl:416-434 */
static void solve_phi_bisect(double D, double T, double ux, double uy, double nux, double nuy,
                             const fivo_params& e, EOSCache* c, double* phi, bool* ok) {
  double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
  double target = D - nu_tau(ux, uy, ut, nux, nuy);
  double m = hq_mass(e);
  if (!o_isfinite(target) || target <= 0.0) { *phi = -PHI_CAP; *ok = false; return; }
  double lo = -PHI_CAP, hi = PHI_CAP;
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    double P, nm, en;
    eos_Pne_2d_cached(T, m + (T * mid), e, c, &P, &nm, &en);
    if (o_isfinite(nm) && (nm * ut) > target) hi = mid; else lo = mid;
  }
  double f = 0.5 * (lo + hi);
  double P, nf, en;
  eos_Pne_2d_cached(T, m + (T * f), e, c, &P, &nf, &en);
  *phi = f; *ok = o_isfinite(nf);
}

/* _cons_to_prim_attempt_2d!, src2d/primrec2d.jl:511-742 */
static RecoveryOut cons_to_prim_attempt(const CellCons& c, const fivo_params& e, double yT0,
                                        double phi0, double ux0, double uy0, int maxit, double tol) {
  RecoveryOut out;
  const double yT_lo = LOG_T_MIN(), yT_hi = LOG_T_SOLVE_MAX();
  out.reason = PRR_UNSET; out.iters = 0; out.resnorm = O_NAN;
  const double D = c.D, Sx = c.Sx, Sy = c.Sy, E = c.E;
  if (!o_isfinite(E) || E <= E_VAC || !o_isfinite(D) || D < D_VAC) {
    out.reason = PRR_VACUUM; out.resnorm = 0.0;
    double T = T_MIN, mu = 0.0, P, n, en;
    eos_Pne(T, mu, e, &P, &n, &en);
    out.T = T; out.mu = mu; out.ux = 0.0; out.uy = 0.0; out.n = 0.0; out.e = o_max(E, 0.0);
    out.P = P; out.ok = false;
    return out;
  }
  const bool ncharge = eos_has_charge(e);
  EOSCache ec; ec.reset();
  const int n_unk = ncharge ? 4 : 3;
  double x[4], F[4], Fp[4], Fm[4], J[4][4], delta[4];
  x[1] = (ncharge && o_isfinite(phi0)) ? o_clamp(phi0, -PHI_CAP, PHI_CAP) : 0.0;
  if (o_isfinite(yT0) && o_isfinite(ux0) && o_isfinite(uy0)) {
    x[0] = o_clamp(yT0, yT_lo, yT_hi);
    x[2] = o_clamp(ux0, -U_CAP_2D, U_CAP_2D);
    x[3] = o_clamp(uy0, -U_CAP_2D, U_CAP_2D);
  } else {
    double sy, sx_, syy;
    seed_from_conserved(E, Sx, Sy, x[1], e, &sy, &sx_, &syy);
    x[0] = o_clamp(sy, yT_lo, yT_hi); x[2] = sx_; x[3] = syy;
  }
  const int slot3[4] = {0, 2, 3, 3}, slot4[4] = {0, 1, 2, 3};
  const int* slot = ncharge ? slot4 : slot3;

  evalF(F, x, c, e, ncharge, &ec);
  if (!all_finite4(F)) {
    out.reason = PRR_NONFINITE_INITIAL;
    double T = o_clamp(o_exp(x[0]), T_MIN, T_SOLVE_MAX), mu = hq_mass(e), P, n, en;
    eos_Pne(T, mu, e, &P, &n, &en);
    out.T = T; out.mu = mu; out.ux = 0.0; out.uy = 0.0; out.n = 0.0; out.e = o_max(en, 0.0);
    out.P = P; out.ok = false;
    return out;
  }
  double sD = o_max(std::fabs(D), 1e-12);
  double sS = o_max(o_max(o_max(std::fabs(Sx), std::fabs(Sy)), 1e-10 * std::fabs(E)), 1e-12);
  double sE = o_max(std::fabs(E), 1e-12);
  const double rs[4] = {1.0 / sD, 1.0 / sS, 1.0 / sS, 1.0 / sE};
  bool converged = false;
  double last_nrm = O_NAN;
  const int r_lo = ncharge ? 0 : 1;

  for (int it = 1; it <= maxit; ++it) {
    double nrm = 0.0;
    for (int r = r_lo; r < 4; ++r) nrm = o_max(nrm, std::fabs(F[r] * rs[r]));
    last_nrm = nrm;
    if (nrm < tol) { converged = true; out.reason = PRR_CONVERGED; out.iters = it - 1; break; }
    bool ok_jac = true;
    for (int k = 0; k < n_unk; ++k) {
      int s = slot[k];
      double h = 1e-6 * o_max(1.0, std::fabs(x[s]));
      double xs = x[s];
      x[s] = xs + h;
      evalF(Fp, x, c, e, ncharge, &ec);
      x[s] = xs - h;
      evalF(Fm, x, c, e, ncharge, &ec);
      x[s] = xs;
      if (!(all_finite4(Fp) && all_finite4(Fm))) { ok_jac = false; break; }
      double inv2h = 1.0 / (2.0 * h);
      for (int r = 0; r < n_unk; ++r) {
        int rr = ncharge ? r : r + 1;
        J[r][k] = ((Fp[rr] - Fm[rr]) * inv2h) * rs[rr];
      }
    }
    if (!ok_jac) { out.reason = PRR_NONFINITE_JACOBIAN; break; }
    double Fact[4];
    for (int r = 0; r < n_unk; ++r) {
      int rr = ncharge ? r : r + 1;
      delta[r] = 0.0;
      Fact[r] = F[rr] * rs[rr];
    }
    if (!solve_gauss_n(delta, J, Fact, n_unk)) { out.reason = PRR_LINSOLVE_FAILED; break; }
    double alpha = 1.0;
    for (int k = 0; k < n_unk; ++k) {
      double ad = std::fabs(delta[k]);
      if (ad > 1.0) alpha = o_min(alpha, 1.0 / ad);
    }
    double xs1 = x[0], xs2 = x[1], xs3 = x[2], xs4 = x[3];
    bool accepted = false;
    for (int ls = 0; ls < 12; ++ls) {
      x[0] = xs1; x[1] = xs2; x[2] = xs3; x[3] = xs4;
      for (int k = 0; k < n_unk; ++k) x[slot[k]] += alpha * delta[k];
      x[0] = o_clamp(x[0], yT_lo, yT_hi);
      if (ncharge) x[1] = o_clamp(x[1], -PHI_CAP, PHI_CAP);
      x[2] = o_clamp(x[2], -U_CAP_2D, U_CAP_2D);
      x[3] = o_clamp(x[3], -U_CAP_2D, U_CAP_2D);
      evalF(F, x, c, e, ncharge, &ec);
      if (all_finite4(F)) {
        double trial = 0.0;
        for (int r = r_lo; r < 4; ++r) trial = o_max(trial, std::fabs(F[r] * rs[r]));
        if (trial < nrm * (1.0 - (1e-4 * alpha))) { accepted = true; break; }
      }
      alpha *= 0.5;
    }
    if (!accepted) { out.reason = PRR_LINESEARCH_FAILED; break; }
  }
  out.resnorm = last_nrm;
  double T = o_clamp(o_exp(x[0]), T_MIN, T_SOLVE_MAX);
  double mu = ncharge ? (hq_mass(e) + (T * x[1])) : hq_mass(e);
  double ux = x[2], uy = x[3];
  double P, n, en;
  eos_Pne_2d_cached(T, mu, e, &ec, &P, &n, &en);
  if (!converged) out.reason = (out.reason == PRR_UNSET) ? PRR_MAXIT : out.reason;
  evalF(F, x, c, e, ncharge, &ec);
  double rows[4] = {0, 0, 0, 0};
  double resnorm = 0.0;
  for (int r = r_lo; r < 4; ++r) { rows[r] = std::fabs(F[r] * rs[r]); resnorm = o_max(resnorm, rows[r]); }
  out.resnorm = resnorm;
  out.T = T; out.mu = mu; out.ux = ux; out.uy = uy;
  if (!(o_isfinite(resnorm) && resnorm < tol)) {
    double hyd = o_max(o_max(rows[1], rows[2]), rows[3]);
    if (ncharge && o_isfinite(hyd) && hyd < tol) {
      double phb; bool okb;
      solve_phi_bisect(D, T, ux, uy, c.nux, c.nuy, e, &ec, &phb, &okb);
      x[1] = o_clamp(phb, -PHI_CAP, PHI_CAP);
      mu = hq_mass(e) + (T * x[1]);
      eos_Pne_2d_cached(T, mu, e, &ec, &P, &n, &en);
      out.reason = okb ? PRR_CONVERGED : PRR_RESIDUAL_TOO_LARGE;
      out.mu = mu; out.n = o_max(n, 0.0); out.e = o_max(en, 0.0); out.P = P; out.ok = true;
      return out;
    }
    out.reason = PRR_RESIDUAL_TOO_LARGE;
    out.n = n; out.e = o_max(en, 0.0); out.P = P; out.ok = false;
    return out;
  }
  out.reason = PRR_CONVERGED;
  out.n = n; out.e = o_max(en, 0.0); out.P = P; out.ok = true;
  return out;
}

/* cons_to_prim_2d!, src2d/primrec2d.jl:465-486 */
RecoveryOut cons_to_prim_2d(double D, double Sx, double Sy, double E, double nux, double nuy,
                            double Pi, double pixx, double pixy, double piyy, double pieta,
                            double tau, const fivo_params& e, double yT0, double phi0,
                            double ux0, double uy0, int maxit, double tol) {
  CellCons c{D, Sx, Sy, E, nux, nuy, Pi, pixx, pixy, piyy, pieta, tau};
  RecoveryOut r = cons_to_prim_attempt(c, e, yT0, phi0, ux0, uy0, maxit, tol);
  if (r.ok) return r;
  if (r.reason == PRR_VACUUM) return r;
  if (!(o_isfinite(yT0) && o_isfinite(ux0) && o_isfinite(uy0))) return r;
  return cons_to_prim_attempt(c, e, O_NAN, O_NAN, O_NAN, O_NAN, maxit, tol);
}

/* prim_to_cons_2d!, src2d/primrec2d.jl:753-796. Writes Ucol only on success. */
bool prim_to_cons_2d(double* Ucol, double T, double mu, double ux, double uy, double nux,
                     double nuy, double Pi, double pixx, double pixy, double piyy, double pieta,
                     double tau, const fivo_params& e, const Layout& L, Prim* out) {
  double Tc = o_max(T, T_MIN);
  double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
  double P, n, en;
  eos_Pne(Tc, mu, e, &P, &n, &en);   /* eos_Pne_2d without memo == eos_Pne here */
  if (!(o_isfinite(P) && o_isfinite(n) && o_isfinite(en)) || en <= 0.0) {
    if (out) *out = Prim{Tc, mu, 0.0, 0.0, 0.0, 0.0, 0.0, nux, nuy, Pi, pixx, pixy, piyy, pieta, false};
    return false;
  }
  double weff = (en + P) + Pi;
  double Ptot = P + Pi;
  PiC Pc = shear_tensor(ux, uy, ut, tau, pixx, pixy, piyy, pieta);
  double Jt = (n * ut) + nu_tau(ux, uy, ut, nux, nuy);
  Ucol[L.iDtau] = tau * Jt;
  Ucol[L.iSx] = ((weff * ut) * ux) + Pc.tx;
  Ucol[L.iSy] = ((weff * ut) * uy) + Pc.ty;
  Ucol[L.iE] = (((weff * ut) * ut) - Ptot) + Pc.tt;
  if (L.hasNu) { Ucol[L.iNux] = nux; Ucol[L.iNuy] = nuy; }
  if (L.hasPi) Ucol[L.iPi] = Pi;
  if (L.hasShear) { Ucol[L.iPixx] = pixx; Ucol[L.iPixy] = pixy; Ucol[L.iPiyy] = piyy; Ucol[L.iPieta] = pieta; }
  if (out) *out = Prim{Tc, mu, ux, uy, n, en, P, nux, nuy, Pi, pixx, pixy, piyy, pieta, true};
  return true;
}

/* =========================== model / grid / work =========================== */

bool make_model(const fivo_params& p, Model& m, const char** err) {
  m.p = p;
  Layout& L = m.L;
  int k = 0;
  L.iDtau = k++; L.iSx = k++; L.iSy = k++; L.iE = k++;
  L.hasNu = p.with_charge != 0; L.iNux = L.hasNu ? k++ : -1; L.iNuy = L.hasNu ? k++ : -1;
  L.hasPi = p.enable_bulk != 0; L.iPi = L.hasPi ? k++ : -1;
  L.hasShear = p.enable_shear != 0;
  L.iPixx = L.hasShear ? k++ : -1; L.iPixy = L.hasShear ? k++ : -1;
  L.iPiyy = L.hasShear ? k++ : -1; L.iPieta = L.hasShear ? k++ : -1;
  /* the charm second moment's rows follow the medium's (make_layout2d with_m2) */
  L.hasM2 = p.consistent_m2 != 0;
  L.iPQxx = L.hasM2 ? k++ : -1; L.iPQxy = L.hasM2 ? k++ : -1; L.iPQyy = L.hasM2 ? k++ : -1;
  L.iPQeta = L.hasM2 ? k++ : -1; L.iPiQ = L.hasM2 ? k++ : -1;
  L.nv = k;
  /* reject_unwired_knobs_2d, src2d/primitives2d.jl:263-269 */
  if (p.consistent_fm && p.tauN_coeff != 1.0) {
    if (err) *err = "tauN_coeff cannot be combined with consistent_fm = true";
    return false;
  }
  /* build_model_2d, main2D.jl:102-108 */
  if (p.E_vac_cut > 0.0) m.E_vac_cut = p.E_vac_cut;
  else { double P, n, en; eos_Pne(p.T_vac_cut, 0.0, p, &P, &n, &en); m.E_vac_cut = en; }
  return true;
}

void make_grid(int Nx, int Ny, int ng, double xmax, double ymax, Grid& g) {
  g.Nx = Nx; g.Ny = Ny; g.ng = ng;
  g.xmin = -xmax; g.xmax = xmax; g.ymin = -ymax; g.ymax = ymax;
  g.dx = (xmax - g.xmin) / Nx; g.dy = (ymax - g.ymin) / Ny;
  g.Nxtot = Nx + 2 * ng; g.Nytot = Ny + 2 * ng; g.Ntot = (int64_t)g.Nxtot * g.Nytot;
  g.xC.resize(g.Nxtot); g.yC.resize(g.Nytot);
  /* xC[i] = xmin + (i - nghost - 0.5)*dx for 1-based i, src2d/grid2d.jl:61-62 */
  for (int i = 0; i < g.Nxtot; ++i) g.xC[i] = g.xmin + (((double)(i + 1 - ng)) - 0.5) * g.dx;
  for (int j = 0; j < g.Nytot; ++j) g.yC[j] = g.ymin + (((double)(j + 1 - ng)) - 0.5) * g.dy;
}

void make_work(const Grid& g, const Model& m, Work& w) {
  size_t N = (size_t)g.Ntot, nv = (size_t)m.L.nv;
  auto vz = [&](std::vector<double>& v, size_t n) { v.assign(n, 0.0); };
  auto vn = [&](std::vector<double>& v) { v.assign(N, O_NAN); };
  vz(w.yT, N); vz(w.phi, N); vz(w.mu, N); vz(w.alpha, N); vz(w.ux, N); vz(w.uy, N);
  vz(w.P, N); vz(w.n, N); vz(w.e, N); w.ok.assign(N, 0);
  vn(w.x0_yT); vn(w.x0_phi); vn(w.x0_ux); vn(w.x0_uy);
  vn(w.ux_prev); vn(w.uy_prev); vn(w.alpha_prev); vn(w.T_prev); vn(w.nux_prev); vn(w.nuy_prev);
  vz(w.sigx, 4 * N); vz(w.sigy, 4 * N); vz(w.ULpx, 4 * N); vz(w.URpx, 4 * N); vz(w.ULpy, 4 * N); vz(w.URpy, 4 * N);
  vz(w.ULcx, nv * N); vz(w.URcx, nv * N); vz(w.ULcy, nv * N); vz(w.URcy, nv * N);
  vz(w.Fhx, nv * N); vz(w.Fhy, nv * N); vz(w.S, nv * N); vz(w.diss_snap, nv * N);
  vz(w.k, nv * N); vz(w.U1, nv * N); vz(w.U2, nv * N);
  w.bad.assign(N, 0); w.bad_tmp.assign(N, 0);
  vz(w.theta, N); vz(w.vxC, N); vz(w.vyC, N);
  vz(w.slope_tmp, N); vz(w.alphaFx, N); vz(w.alphaFy, N); vz(w.gradAx, N); vz(w.gradAy, N);
  vz(w.shear_res, N);
  w.nprimfail = 0; w.nvacuum = 0; w.primfail_i = -1; w.primfail_reason = 0; w.primfail_resnorm = 0;
  w.amax = 0.0; w.nmood = 0; w.nhalve = 0;
}

/* =========================== boundary conditions (src2d/bc2d.jl:14-65) =========================== */

void apply_bc_2d(double* U, const Grid& g, const Layout& L, int bc) {
  const int ng = g.ng, nv = L.nv;
  const int ix0 = ng, ix1 = ng + g.Nx - 1, iy0 = ng, iy1 = ng + g.Ny - 1;  /* 0-based interior ends */
  auto cp = [&](int64_t dst, int64_t src) {
    for (int a = 0; a < nv; ++a) U[dst * nv + a] = U[src * nv + a];
  };
  if (bc == FIVO_BC_PERIODIC) {
    for (int k = 1; k <= ng; ++k)
      for (int iy = 0; iy < g.Nytot; ++iy) {
        cp(g.lin(ng - k, iy), g.lin(ix1 + 1 - k, iy));
        cp(g.lin(ix1 + k, iy), g.lin(ix0 - 1 + k, iy));
      }
    for (int k = 1; k <= ng; ++k)
      for (int ix = 0; ix < g.Nxtot; ++ix) {
        cp(g.lin(ix, ng - k), g.lin(ix, iy1 + 1 - k));
        cp(g.lin(ix, iy1 + k), g.lin(ix, iy0 - 1 + k));
      }
    return;
  }
  for (int k = 1; k <= ng; ++k)
    for (int iy = 0; iy < g.Nytot; ++iy) {
      cp(g.lin(ng - k, iy), g.lin(ix0, iy));
      cp(g.lin(ix1 + k, iy), g.lin(ix1, iy));
    }
  for (int k = 1; k <= ng; ++k)
    for (int ix = 0; ix < g.Nxtot; ++ix) {
      cp(g.lin(ix, ng - k), g.lin(ix, iy0));
      cp(g.lin(ix, iy1 + k), g.lin(ix, iy1));
    }
}

/* =========================== rhs (src2d/rhs2d.jl) =========================== */

static inline void dissipatives_at(const double* U, int64_t i, const Layout& L, double* d) {
  const double* u = U + i * L.nv;
  d[0] = L.hasNu ? u[L.iNux] : 0.0;   d[1] = L.hasNu ? u[L.iNuy] : 0.0;
  d[2] = L.hasPi ? u[L.iPi] : 0.0;
  d[3] = L.hasShear ? u[L.iPixx] : 0.0; d[4] = L.hasShear ? u[L.iPixy] : 0.0;
  d[5] = L.hasShear ? u[L.iPiyy] : 0.0; d[6] = L.hasShear ? u[L.iPieta] : 0.0;
}

/* _primitive_pass!, src2d/rhs2d.jl:67-160 */
static void primitive_pass(const double* U, const Grid& g, double tau, const Model& m, Work& w) {
  const Layout& L = m.L;
  const fivo_params& e = m.p;
  int64_t nfail = 0, nvac = 0;
  int64_t rep_i = -1; int rep_reason = 0; double rep_res = 0.0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : nfail, nvac)
  for (int ix = 0; ix < g.Nxtot; ++ix) {
    for (int iy = 0; iy < g.Nytot; ++iy) {
      int64_t i = g.lin(ix, iy);
      const double* u = U + i * L.nv;
      double D = safe_div(u[L.iDtau], tau);
      double d[7];
      dissipatives_at(U, i, L, d);
      RecoveryOut r = cons_to_prim_2d(D, u[L.iSx], u[L.iSy], u[L.iE], d[0], d[1], d[2], d[3], d[4],
                                      d[5], d[6], tau, e, w.x0_yT[i], w.x0_phi[i], w.x0_ux[i],
                                      w.x0_uy[i], e.primrec_maxit, e.primrec_tol);
      double T = r.T, mu = r.mu, ux = r.ux, uy = r.uy, n = r.n, en = r.e, P = r.P;
      bool ok = r.ok;
      if (!ok) {
        if (r.reason == PRR_VACUUM) nvac += 1;
        else {
          nfail += 1;
#pragma omp critical
          {
            if (rep_i < 0 || i < rep_i) { rep_i = i; rep_reason = r.reason; rep_res = r.resnorm; }
          }
        }
        T = T_MIN; mu = 0.0; ux = 0.0; uy = 0.0;
        eos_Pne(T, mu, e, &P, &n, &en);
        en = o_max(en, 0.0); n = 0.0;
      }
      double Tm = o_max(T, T_MIN);
      w.yT[i] = o_log(Tm);
      w.phi[i] = o_clamp((mu - hq_mass(e)) / Tm, -PHI_CAP, PHI_CAP);
      w.mu[i] = mu;
      w.alpha[i] = mu / Tm;
      w.ux[i] = ux; w.uy[i] = uy;
      w.P[i] = P; w.n[i] = n; w.e[i] = en;
      w.ok[i] = ok ? 1 : 0;
      double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
      double iu = safe_inv(ut);
      w.vxC[i] = ux * iu;
      w.vyC[i] = uy * iu;
      if (ok) { w.x0_yT[i] = w.yT[i]; w.x0_phi[i] = w.phi[i]; w.x0_ux[i] = ux; w.x0_uy[i] = uy; }
      else { w.x0_yT[i] = O_NAN; w.x0_phi[i] = O_NAN; w.x0_ux[i] = O_NAN; w.x0_uy[i] = O_NAN; }
      if (L.hasShear) {
        double R, rel;
        shear_residual(ux, uy, ut, d[3], d[4], d[5], d[6], &R, &rel);
        w.shear_res[i] = rel;
      }
    }
  }
  w.nprimfail = nfail; w.nvacuum = nvac;
  w.primfail_i = rep_i; w.primfail_reason = rep_reason; w.primfail_resnorm = rep_res;
}

/* update_primitives_2d!, src2d/rhs2d.jl:57-65 */
int64_t update_primitives_2d(double* U, const Grid& g, double tau, const Model& m, Work& w, int bc) {
  apply_bc_2d(U, g, m.L, bc);
  primitive_pass(U, g, tau, m, w);
  return w.nprimfail;
}

/* mc_limiter, src/utils.jl:14-22 */
static inline double mc_limiter(double a, double b) {
  if (o_sign(a) != o_sign(b)) return 0.0;
  double s = o_sign(a);
  double aa = std::fabs(a), bb = std::fabs(b);
  return s * o_min(2.0 * aa, o_min(2.0 * bb, 0.5 * (aa + bb)));
}

/* reconstruct_muscl_2d!, src2d/reconstruction2d.jl:27-103 */
static void reconstruct_muscl(double* UL, double* UR, double* sig, const Work& w, const Grid& g, bool xdir) {
  const int64_t st = xdir ? g.Nytot : 1;
  const int ng = g.ng;
  const double* yT = w.yT.data(); const double* ph = w.phi.data();
  const double* ux = w.ux.data(); const double* uy = w.uy.data();
  std::fill(sig, sig + 4 * g.Ntot, 0.0);
  int ixlo = xdir ? 1 : 0, ixhi = xdir ? g.Nxtot - 2 : g.Nxtot - 1;
  int iylo = xdir ? 0 : 1, iyhi = xdir ? g.Nytot - 1 : g.Nytot - 2;
#pragma omp parallel for
  for (int ix = ixlo; ix <= ixhi; ++ix)
    for (int iy = iylo; iy <= iyhi; ++iy) {
      int64_t i = g.lin(ix, iy), im = i - st, ip = i + st;
      sig[4 * i + 0] = mc_limiter(yT[i] - yT[im], yT[ip] - yT[i]);
      sig[4 * i + 1] = mc_limiter(ph[i] - ph[im], ph[ip] - ph[i]);
      sig[4 * i + 2] = mc_limiter(ux[i] - ux[im], ux[ip] - ux[i]);
      sig[4 * i + 3] = mc_limiter(uy[i] - uy[im], uy[ip] - uy[i]);
    }
  int fxhi = xdir ? g.Nxtot - 2 : g.Nxtot - 1;
  int fyhi = xdir ? g.Nytot - 1 : g.Nytot - 2;
  const int kmax = xdir ? g.Nxtot : g.Nytot;
#pragma omp parallel for
  for (int ix = 0; ix <= fxhi; ++ix)
    for (int iy = 0; iy <= fyhi; ++iy) {
      int64_t i = g.lin(ix, iy), ip = i + st;
      int k = (xdir ? ix : iy) + 1;          /* 1-based index of the left cell along dir */
      double* l = UL + 4 * i; double* r = UR + 4 * i;
      if (k <= ng || k >= kmax - ng) {
        l[0] = yT[i]; l[1] = ph[i]; l[2] = ux[i]; l[3] = uy[i];
        r[0] = yT[ip]; r[1] = ph[ip]; r[2] = ux[ip]; r[3] = uy[ip];
        continue;
      }
      int64_t im = i - st, ipp = ip + st;
      const double* si = sig + 4 * i; const double* sp = sig + 4 * ip;
      l[0] = yT[i] + 0.5 * si[0]; l[1] = ph[i] + 0.5 * si[1];
      l[2] = ux[i] + 0.5 * si[2]; l[3] = uy[i] + 0.5 * si[3];
      r[0] = yT[ip] - 0.5 * sp[0]; r[1] = ph[ip] - 0.5 * sp[1];
      r[2] = ux[ip] - 0.5 * sp[2]; r[3] = uy[ip] - 0.5 * sp[3];
      const double* f[4] = {yT, ph, ux, uy};
      for (int q = 0; q < 4; ++q) {
        const double* v = f[q];
        l[q] = o_clamp(l[q], o_min(o_min(v[im], v[i]), v[ip]), o_max(o_max(v[im], v[i]), v[ip]));
      }
      for (int q = 0; q < 4; ++q) {
        const double* v = f[q];
        r[q] = o_clamp(r[q], o_min(o_min(v[i], v[ip]), v[ipp]), o_max(o_max(v[i], v[ip]), v[ipp]));
      }
    }
}

/* flux_cell_2d!, src2d/fluxes2d.jl:24-69 */
static void flux_cell(double* F, const Prim& p, double tau, bool xdir, const Model& m) {
  const Layout& L = m.L;
  for (int a = 0; a < L.nv; ++a) F[a] = 0.0;
  double ux = p.ux, uy = p.uy;
  double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
  double iu = safe_inv(ut);
  double vx = ux * iu, vy = uy * iu;
  double Ptot = p.P + p.Pi;
  double weff = (p.e + p.P) + p.Pi;
  PiC Pc = shear_tensor(ux, uy, ut, tau, p.pixx, p.pixy, p.piyy, p.pieta);
  double Jx = (p.n * ux) + p.nux, Jy = (p.n * uy) + p.nuy;
  double v;
  if (xdir) {
    F[L.iDtau] = tau * Jx;
    F[L.iSx] = (((weff * ux) * ux) + Ptot) + Pc.xx;
    F[L.iSy] = ((weff * ux) * uy) + Pc.xy;
    F[L.iE] = ((weff * ut) * ux) + Pc.tx;
    v = vx;
  } else {
    F[L.iDtau] = tau * Jy;
    F[L.iSx] = ((weff * ux) * uy) + Pc.xy;
    F[L.iSy] = (((weff * uy) * uy) + Ptot) + Pc.yy;
    F[L.iE] = ((weff * ut) * uy) + Pc.ty;
    v = vy;
  }
  if (L.hasNu && m.p.advect_nu) { F[L.iNux] = p.nux * v; F[L.iNuy] = p.nuy * v; }
  if (L.hasPi && m.p.advect_Pi) F[L.iPi] = p.Pi * v;
  if (L.hasShear && m.p.advect_pi) {
    F[L.iPixx] = p.pixx * v; F[L.iPixy] = p.pixy * v; F[L.iPiyy] = p.piyy * v; F[L.iPieta] = p.pieta * v;
  }
}

/* wavespeeds_2d, src2d/fluxes2d.jl:87-113 */
static void wavespeeds(const Prim& p, const fivo_params& e, bool xdir, double pinn, double* lm, double* lp) {
  double cs2 = o_clamp(eos_cs2(p.T, p.mu, e), 0.0, 0.999);
  double w = p.e + p.P;
  if (w > TINY) cs2 = o_min(cs2 + ((std::fabs(p.Pi) + std::fabs(pinn)) / w), 0.999);
  double ut = std::sqrt((1.0 + (p.ux * p.ux)) + (p.uy * p.uy));
  double iu = safe_inv(ut);
  double vx = p.ux * iu, vy = p.uy * iu;
  double v2 = (vx * vx) + (vy * vy);
  double vn = xdir ? vx : vy;
  double den = 1.0 - (v2 * cs2);
  if (den <= TINY) { *lm = -1.0; *lp = 1.0; return; }
  double cs = safe_sqrt(cs2);
  double rad = (1.0 - v2) * (den - ((vn * vn) * (1.0 - cs2)));
  double disc = cs * safe_sqrt(o_max(rad, 0.0));
  double a = ((vn * (1.0 - cs2)) - disc) / den;
  double b = ((vn * (1.0 - cs2)) + disc) / den;
  *lm = o_clamp(a, -1.0, 1.0);
  *lp = o_clamp(b, -1.0, 1.0);
}

/* _floor_prim_2d!, src2d/rhs2d.jl:259-268 */
static Prim floor_prim(double* Uc, const Layout& L, double Emin) {
  for (int a = 0; a < L.nv; ++a) Uc[a] = 0.0;
  Uc[L.iE] = Emin;
  return Prim{T_MIN, 0.0, 0.0, 0.0, 0.0, Emin, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, true};
}

/* _faces_2d! + hlle_flux_2d!, src2d/rhs2d.jl:282-371, src2d/fluxes2d.jl:121-157 */
static void faces(double* Fh, const double* ULp, const double* URp, double* ULc, double* URc,
                  const double* U, const Grid& g, double tau, const Model& m, const Work& w,
                  bool xdir, double Emin, const uint8_t* ffo, double* amax_out) {
  const Layout& L = m.L;
  const fivo_params& e = m.p;
  const int nv = L.nv;
  const int64_t st = xdir ? g.Nytot : 1;
  int fxhi = xdir ? g.Nxtot - 2 : g.Nxtot - 1;
  int fyhi = xdir ? g.Nytot - 1 : g.Nytot - 2;
  double amax = 0.0;
#pragma omp parallel for schedule(dynamic, 1) reduction(max : amax)
  for (int ix = 0; ix <= fxhi; ++ix) {
    double FL[16], FR[16];
    for (int iy = 0; iy <= fyhi; ++iy) {
      int64_t i = g.lin(ix, iy), ip = i + st;
      double dL[7], dR[7];
      dissipatives_at(U, i, L, dL);
      dissipatives_at(U, ip, L, dR);
      bool forced = ffo != nullptr && (ffo[i] || ffo[ip]);
      bool good = false;
      Prim pL, pR;
      double* lc = ULc + i * nv; double* rc = URc + i * nv;
      if (!forced) {
        const double* l = ULp + 4 * i; const double* r = URp + 4 * i;
        double TL = o_exp(l[0]); double muL = hq_mass(e) + (TL * l[1]);
        double TR = o_exp(r[0]); double muR = hq_mass(e) + (TR * r[1]);
        bool okL = prim_to_cons_2d(lc, TL, muL, l[2], l[3], dL[0], dL[1], dL[2], dL[3], dL[4], dL[5], dL[6], tau, e, L, &pL);
        bool okR = prim_to_cons_2d(rc, TR, muR, r[2], r[3], dR[0], dR[1], dR[2], dR[3], dR[4], dR[5], dR[6], tau, e, L, &pR);
        good = okL && okR && lc[L.iDtau] >= 0.0 && rc[L.iDtau] >= 0.0 && lc[L.iE] >= Emin && rc[L.iE] >= Emin;
      }
      if (!good) {
        double TLc = o_exp(w.yT[i]), muLc = w.mu[i];
        double TRc = o_exp(w.yT[ip]), muRc = w.mu[ip];
        bool okL = prim_to_cons_2d(lc, TLc, muLc, w.ux[i], w.uy[i], dL[0], dL[1], dL[2], dL[3], dL[4], dL[5], dL[6], tau, e, L, &pL);
        bool okR = prim_to_cons_2d(rc, TRc, muRc, w.ux[ip], w.uy[ip], dR[0], dR[1], dR[2], dR[3], dR[4], dR[5], dR[6], tau, e, L, &pR);
        if (!(okL && okR)) {
          if (!okL) pL = floor_prim(lc, L, Emin);
          if (!okR) pR = floor_prim(rc, L, Emin);
        }
      }
      flux_cell(FL, pL, tau, xdir, m);
      flux_cell(FR, pR, tau, xdir, m);
      double pinnL = xdir ? pL.pixx : pL.piyy;
      double pinnR = xdir ? pR.pixx : pR.piyy;
      double lmL, lpL, lmR, lpR;
      wavespeeds(pL, e, xdir, pinnL, &lmL, &lpL);
      wavespeeds(pR, e, xdir, pinnR, &lmR, &lpR);
      double sL = o_min(lmL, lmR), sR = o_max(lpL, lpR);
      double* fh = Fh + i * nv;
      if (sL >= 0) { for (int a = 0; a < nv; ++a) fh[a] = FL[a]; }
      else if (sR <= 0) { for (int a = 0; a < nv; ++a) fh[a] = FR[a]; }
      else {
        double inv = 1.0 / ((sR - sL) + TINY);
        for (int a = 0; a < nv; ++a)
          fh[a] = (((sR * FL[a]) - (sL * FR[a])) + ((sR * sL) * (rc[a] - lc[a]))) * inv;
      }
      double a = o_max(std::fabs(sL), std::fabs(sR));
      if (a > amax) amax = a;
    }
  }
  *amax_out = amax;
}

/* compute_divv_2d!, src2d/rhs2d.jl:29-41 */
static void compute_divv(Work& w, const Grid& g) {
  std::fill(w.theta.begin(), w.theta.end(), 0.0);
  double invdx = 1.0 / g.dx, invdy = 1.0 / g.dy;
  for (int ix = 1; ix <= g.Nxtot - 2; ++ix)
    for (int iy = 1; iy <= g.Nytot - 2; ++iy) {
      int64_t i = g.lin(ix, iy), ixm = i - g.Nytot, ixp = i + g.Nytot;
      w.theta[i] = ((0.5 * (w.vxC[ixp] - w.vxC[ixm])) * invdx) + ((0.5 * (w.vyC[i + 1] - w.vyC[i - 1])) * invdy);
    }
}

/* rhs_2d!, src2d/rhs2d.jl:169-249 */
void rhs_2d(double* dU, double* U, const Grid& g, double tau, const Model& m, Work& w, int bc,
            double Emin, const uint8_t* ffo) {
  const Layout& L = m.L;
  const int nv = L.nv, ng = g.ng;
  apply_bc_2d(U, g, L, bc);
  primitive_pass(U, g, tau, m, w);
  reconstruct_muscl(w.ULpx.data(), w.URpx.data(), w.sigx.data(), w, g, true);
  reconstruct_muscl(w.ULpy.data(), w.URpy.data(), w.sigy.data(), w, g, false);
  std::fill(w.Fhx.begin(), w.Fhx.end(), 0.0);
  std::fill(w.Fhy.begin(), w.Fhy.end(), 0.0);
  double ax = 0.0, ay = 0.0;
  faces(w.Fhx.data(), w.ULpx.data(), w.URpx.data(), w.ULcx.data(), w.URcx.data(), U, g, tau, m, w, true, Emin, ffo, &ax);
  faces(w.Fhy.data(), w.ULpy.data(), w.URpy.data(), w.ULcy.data(), w.URcy.data(), U, g, tau, m, w, false, Emin, ffo, &ay);
  w.amax = o_max(ax, ay);
  const fivo_params& p = m.p;
  bool need_div = (L.hasNu && p.advect_nu) || (L.hasPi && p.advect_Pi) || (L.hasShear && p.advect_pi);
  if (need_div) compute_divv(w, g); else std::fill(w.theta.begin(), w.theta.end(), 0.0);
  std::fill(w.S.begin(), w.S.end(), 0.0);
  double itau = safe_inv(tau);
  for (int ix = ng; ix < ng + g.Nx; ++ix)
    for (int iy = ng; iy < ng + g.Ny; ++iy) {
      int64_t i = g.lin(ix, iy);
      const double* u = U + i * nv;
      double d[7]; dissipatives_at(U, i, L, d);
      double* S = w.S.data() + i * nv;
      /* source_cell_2d!, src2d/fluxes2d.jl:166-177 */
      S[L.iSx] = (-u[L.iSx]) * itau;
      S[L.iSy] = (-u[L.iSy]) * itau;
      S[L.iE] = (-((u[L.iE] + (w.P[i] + d[2])) + d[6])) * itau;
      if (need_div) {
        double divv = w.theta[i];
        if (L.hasNu && p.advect_nu) { S[L.iNux] += u[L.iNux] * divv; S[L.iNuy] += u[L.iNuy] * divv; }
        if (L.hasPi && p.advect_Pi) S[L.iPi] += u[L.iPi] * divv;
        if (L.hasShear && p.advect_pi) {
          S[L.iPixx] += u[L.iPixx] * divv; S[L.iPixy] += u[L.iPixy] * divv;
          S[L.iPiyy] += u[L.iPiyy] * divv; S[L.iPieta] += u[L.iPieta] * divv;
        }
      }
    }
  std::fill(dU, dU + nv * g.Ntot, 0.0);
  double invdx = 1.0 / g.dx, invdy = 1.0 / g.dy;
  for (int ix = ng; ix < ng + g.Nx; ++ix)
    for (int iy = ng; iy < ng + g.Ny; ++iy) {
      int64_t i = g.lin(ix, iy), ixm = i - g.Nytot;
      for (int a = 0; a < nv; ++a)
        dU[i * nv + a] = (((-(w.Fhx[i * nv + a] - w.Fhx[ixm * nv + a])) * invdx) -
                          ((w.Fhy[i * nv + a] - w.Fhy[(i - 1) * nv + a]) * invdy)) + w.S[i * nv + a];
    }
}

/* =========================== floors (src2d/floors2d.jl) =========================== */

static inline void blank(double* u, const Layout& L) {
  u[L.iSx] = 0.0; u[L.iSy] = 0.0; u[L.iDtau] = 0.0;
  if (L.hasNu) { u[L.iNux] = 0.0; u[L.iNuy] = 0.0; }
  if (L.hasPi) u[L.iPi] = 0.0;
  if (L.hasShear) { u[L.iPixx] = 0.0; u[L.iPixy] = 0.0; u[L.iPiyy] = 0.0; u[L.iPieta] = 0.0; }
}

/* enforce_floors_2d!, src2d/floors2d.jl:24-104 */
static void enforce_floors(double* U, const Grid& g, const Model& m, double Emin) {
  const Layout& L = m.L;
  double Evac = o_max(Emin, m.E_vac_cut);
  double rdom = m.p.r_domain;
  double rdom2 = o_isfinite(rdom) ? rdom * rdom : O_INF;
  for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
    for (int iy = g.ng; iy < g.ng + g.Ny; ++iy) {
      double* u = U + g.lin(ix, iy) * L.nv;
      if (o_isfinite(rdom)) {
        double x = g.xC[ix], y = g.yC[iy];
        if ((x * x) + (y * y) > rdom2) { u[L.iE] = Emin; blank(u, L); continue; }
      }
      double Ei = u[L.iE];
      if (!o_isfinite(Ei)) { u[L.iE] = Emin; blank(u, L); continue; }
      if (Ei < Evac) { u[L.iE] = Emin; blank(u, L); continue; }
      if (Ei <= 1e6 * Emin) blank(u, L);
      double Di = u[L.iDtau];
      if (!o_isfinite(Di) || Di < 0.0) u[L.iDtau] = 0.0;
      if (!o_isfinite(u[L.iSx])) u[L.iSx] = 0.0;
      if (!o_isfinite(u[L.iSy])) u[L.iSy] = 0.0;
      if (L.hasNu) { if (!o_isfinite(u[L.iNux])) u[L.iNux] = 0.0; if (!o_isfinite(u[L.iNuy])) u[L.iNuy] = 0.0; }
      if (L.hasPi) { if (!o_isfinite(u[L.iPi])) u[L.iPi] = 0.0; }
      if (L.hasShear) {
        if (!o_isfinite(u[L.iPixx])) u[L.iPixx] = 0.0;
        if (!o_isfinite(u[L.iPixy])) u[L.iPixy] = 0.0;
        if (!o_isfinite(u[L.iPiyy])) u[L.iPiyy] = 0.0;
        if (!o_isfinite(u[L.iPieta])) u[L.iPieta] = 0.0;
      }
    }
}

static inline double peff_of(const double* u, const Layout& L, const double* Pw, int64_t i) {
  double Peff = 0.0;
  if (Pw) { double p = Pw[i]; if (o_isfinite(p)) Peff = o_max(p, 0.0); }
  if (L.hasPi) { double v = u[L.iPi]; if (o_isfinite(v)) Peff += std::fabs(v); }
  if (L.hasShear) {
    const int ks[4] = {L.iPixx, L.iPixy, L.iPiyy, L.iPieta};
    for (int q = 0; q < 4; ++q) { double v = u[ks[q]]; if (o_isfinite(v)) Peff += std::fabs(v); }
  }
  return Peff;
}

/* enforce_S_energy_constraint_2d!, src2d/floors2d.jl:118-157 */
static void enforce_S_energy(double* U, const Grid& g, const Model& m, double chi, const double* Pw) {
  const Layout& L = m.L;
  for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
    for (int iy = g.ng; iy < g.ng + g.Ny; ++iy) {
      int64_t i = g.lin(ix, iy);
      double* u = U + i * L.nv;
      double Ei = u[L.iE], Sx = u[L.iSx], Sy = u[L.iSy];
      if (!(o_isfinite(Ei) && o_isfinite(Sx) && o_isfinite(Sy))) continue;
      if (Ei <= 0) continue;
      double Peff = peff_of(u, L, Pw, i);
      double Smax = chi * (Ei + Peff);
      double aS = o_hypot(Sx, Sy);
      if (aS > Smax) {
        double sc = Smax / (aS + TINY);
        u[L.iSx] = Sx * sc; u[L.iSy] = Sy * sc;
      }
    }
}

/* enforce_nu_charge_constraint_2d!, src2d/floors2d.jl:177-210 */
static void enforce_nu_charge(double* U, const Grid& g, const Model& m, double tau, double chi) {
  const Layout& L = m.L;
  if (!L.hasNu) return;
  for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
    for (int iy = g.ng; iy < g.ng + g.Ny; ++iy) {
      double* u = U + g.lin(ix, iy) * L.nv;
      double Dt = u[L.iDtau] / tau;
      double nux = u[L.iNux], nuy = u[L.iNuy];
      if (!(o_isfinite(Dt) && o_isfinite(nux) && o_isfinite(nuy))) continue;
      if (Dt <= 0.0) { u[L.iNux] = 0.0; u[L.iNuy] = 0.0; continue; }
      double cap = chi * Dt;
      double an = o_hypot(nux, nuy);
      if (an > cap) {
        double sc = cap / (an + TINY);
        u[L.iNux] = nux * sc; u[L.iNuy] = nuy * sc;
      }
    }
}

/* sanitize_stage_2d!, src2d/floors2d.jl:218-227 */
static void sanitize_stage(double* U, const Grid& g, double tau, const Model& m, const Work& w, int bc) {
  enforce_floors(U, g, m, E_FLOOR);
  enforce_S_energy(U, g, m, CHI_SRE, w.P.data());
  enforce_nu_charge(U, g, m, tau, 0.999);
  apply_bc_2d(U, g, m.L, bc);
}

/* cell_admissible_2d, src2d/floors2d.jl:281-337 (work always present here) */
static bool cell_admissible(const double* U, int64_t i, double tau, const Model& m, const Work& w) {
  const Layout& L = m.L;
  const double* u = U + i * L.nv;
  const double Emin = E_FLOOR, chi = CHI_SRE, v_eps = 1e-12;
  double E = u[L.iE], Sx = u[L.iSx], Sy = u[L.iSy], Dt = u[L.iDtau];
  if (!(o_isfinite(E) && o_isfinite(Sx) && o_isfinite(Sy) && o_isfinite(Dt))) return false;
  if (!(E >= Emin)) return false;
  if (!(Dt >= 0.0)) return false;
  if (L.hasNu && !(o_isfinite(u[L.iNux]) && o_isfinite(u[L.iNuy]))) return false;
  if (L.hasPi && !o_isfinite(u[L.iPi])) return false;
  if (L.hasShear && !(o_isfinite(u[L.iPixx]) && o_isfinite(u[L.iPixy]) && o_isfinite(u[L.iPiyy]) && o_isfinite(u[L.iPieta]))) return false;
  if (E <= 1e6 * Emin) return true;
  if (w.ok[i]) {
    double vx = w.vxC[i], vy = w.vyC[i];
    if (!(o_isfinite(vx) && o_isfinite(vy))) return false;
    double lim = (1.0 - v_eps) * (1.0 - v_eps);
    if (!((vx * vx) + (vy * vy) < lim)) return false;
  }
  double Peff = peff_of(u, L, w.P.data(), i);
  if (o_hypot(Sx, Sy) <= ((SR_MARGIN_2D * chi) * (E + Peff))) return true;
  double d[7]; dissipatives_at(U, i, L, d);
  RecoveryOut r = cons_to_prim_2d(safe_div(Dt, tau), Sx, Sy, E, d[0], d[1], d[2], d[3], d[4], d[5], d[6],
                                  tau, m.p, O_NAN, O_NAN, O_NAN, O_NAN, 80, 1e-12);
  return r.ok || r.reason == PRR_VACUUM;
}

/* state_ok_2d, src2d/timestepper2d.jl:56-66 */
static bool state_ok(const double* U, const Grid& g, const Model& m, const Work& w, double tau) {
  for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
    for (int iy = g.ng; iy < g.ng + g.Ny; ++iy)
      if (!cell_admissible(U, g.lin(ix, iy), tau, m, w)) return false;
  return true;
}

/* mark_bad_2d!, src2d/floors2d.jl:350-365 */
static void mark_bad(uint8_t* bad, const double* U, const Grid& g, double tau, const Model& m, const Work& w) {
  std::fill(bad, bad + g.Ntot, 0);
  for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
    for (int iy = g.ng; iy < g.ng + g.Ny; ++iy) {
      int64_t i = g.lin(ix, iy);
      if (!cell_admissible(U, i, tau, m, w)) bad[i] = 1;
    }
}

/* expand_bad_2d!, src2d/floors2d.jl:369-383 */
static void expand_bad(uint8_t* bad, uint8_t* tmp, const Grid& g, int radius) {
  for (int it = 0; it < radius; ++it) {
    std::memcpy(tmp, bad, (size_t)g.Ntot);
    for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
      for (int iy = g.ng; iy < g.ng + g.Ny; ++iy) {
        int64_t i = g.lin(ix, iy);
        if (tmp[i]) continue;
        if (bad[i - 1] || bad[i + 1] || bad[i - g.Nytot] || bad[i + g.Nytot]) tmp[i] = 1;
      }
    std::memcpy(bad, tmp, (size_t)g.Ntot);
  }
}

/* ======================= timestepper (src2d/timestepper2d.jl) ======================= */

/* compute_dt_2d, src2d/timestepper2d.jl:37-47 */
double compute_dt_2d(const Work& w, const Grid& g, double tau, double CFL, double CFLtau) {
  double amax = 0.0;
  if (w.amax > amax) amax = w.amax;
  amax = o_max(amax, 1e-6);
  double dt_cfl = (CFL * o_min(g.dx, g.dy)) / amax;
  double dt_tau = CFLtau * tau;
  return o_min(dt_cfl, dt_tau);
}

/* _stage_2d!, src2d/timestepper2d.jl:113-140 */
static bool stage(double* Uout, const double* Uin, const double* Uold, double* Ubase, const Grid& g,
                  double tau, double tau_state, double dt, double wold, double wnew, const Model& m,
                  Work& w, int bc, int max_mood) {
  const int64_t NN = (int64_t)m.L.nv * g.Ntot;
  const uint8_t* mask = nullptr;
  for (int attempt = 0; attempt <= max_mood; ++attempt) {
    rhs_2d(w.k.data(), Ubase, g, tau, m, w, bc, E_FLOOR, mask);
    if (wnew == 0.0) {
      for (int64_t q = 0; q < NN; ++q) Uout[q] = Uin[q] + (dt * w.k[q]);
    } else {
      for (int64_t q = 0; q < NN; ++q) Uout[q] = (wold * Uold[q]) + (wnew * (Uin[q] + (dt * w.k[q])));
    }
    sanitize_stage(Uout, g, tau_state, m, w, bc);
    if (state_ok(Uout, g, m, w, tau_state)) return true;
    if (attempt == max_mood) return false;
    w.nmood += 1;
    mark_bad(w.bad.data(), Uout, g, tau_state, m, w);
    expand_bad(w.bad.data(), w.bad_tmp.data(), g, 1 + attempt);
    mask = w.bad.data();
  }
  return false;
}

/* step_ssprk2_2d!, src2d/timestepper2d.jl:74-103 */
bool step_ssprk2_2d(double* U, const Grid& g, double tau, double dtau, const Model& m, Work& w,
                    int bc, int max_halve, int max_mood, double* used) {
  const int64_t NN = (int64_t)m.L.nv * g.Ntot;
  double D = dtau;
  w.nmood = 0; w.nhalve = 0;
  for (int h = 0; h <= max_halve; ++h) {
    std::memcpy(w.U2.data(), U, NN * sizeof(double));
    bool ok1 = stage(w.U1.data(), U, w.U2.data(), U, g, tau, tau + D, D, 1.0, 0.0, m, w, bc, max_mood);
    if (ok1) {
      bool ok2 = stage(U, w.U1.data(), w.U2.data(), w.U1.data(), g, tau + D, tau + D, D, 0.5, 0.5, m, w, bc, max_mood);
      if (ok2) { *used = D; return true; }
    }
    std::memcpy(U, w.U2.data(), NN * sizeof(double));
    D *= 0.5;
    w.nhalve += 1;
  }
  *used = D;
  return false;
}

/* step_ssprk3_2d!, src2d/timestepper2d.jl:148-188 */
bool step_ssprk3_2d(double* U, const Grid& g, double tau, double dtau, const Model& m, Work& w,
                    int bc, int max_halve, double* used) {
  const int64_t NN = (int64_t)m.L.nv * g.Ntot;
  double D = dtau;
  double* U1 = w.U1.data(); double* U2 = w.U2.data(); double* k = w.k.data();
  w.nmood = 0; w.nhalve = 0;
  for (int h = 0; h <= max_halve; ++h) {
    std::memcpy(U2, U, NN * sizeof(double));
    rhs_2d(k, U, g, tau, m, w, bc, E_FLOOR, nullptr);
    for (int64_t q = 0; q < NN; ++q) U1[q] = U[q] + (D * k[q]);
    sanitize_stage(U1, g, tau + D, m, w, bc);
    if (!state_ok(U1, g, m, w, tau + D)) { std::memcpy(U, U2, NN * sizeof(double)); D *= 0.5; w.nhalve += 1; continue; }
    rhs_2d(k, U1, g, tau + D, m, w, bc, E_FLOOR, nullptr);
    for (int64_t q = 0; q < NN; ++q) U1[q] = (0.75 * U2[q]) + (0.25 * (U1[q] + (D * k[q])));
    sanitize_stage(U1, g, tau + D, m, w, bc);
    if (!state_ok(U1, g, m, w, tau + D)) { std::memcpy(U, U2, NN * sizeof(double)); D *= 0.5; w.nhalve += 1; continue; }
    rhs_2d(k, U1, g, tau + (0.5 * D), m, w, bc, E_FLOOR, nullptr);
    for (int64_t q = 0; q < NN; ++q) U[q] = (U2[q] + (2.0 * (U1[q] + (D * k[q])))) / 3.0;
    sanitize_stage(U, g, tau + D, m, w, bc);
    if (state_ok(U, g, m, w, tau + D)) { *used = D; return true; }
    std::memcpy(U, U2, NN * sizeof(double));
    D *= 0.5;
    w.nhalve += 1;
  }
  *used = D;
  return false;
}

/* ======================= transport coefficients ======================= */

/* _fluidum_single_hadron_normalization_2d, src2d/transport2d.jl:19-26 */
static double fluidum_norm(double T, double alpha, const fivo_params& e) {
  double Tm = o_max(T, T_MIN);
  double m = hq_mass(e);
  double z = m / Tm;
  double b2 = o_besselkx(2, z);
  double ex = o_exp(o_clamp(alpha - z, -700.0, 700.0));
  return ((((e.g_hq * (Tm / (2.0 * PI2))) * (m * m)) * ex) * b2) * FMGEV3;
}

/* _diff_tauN_impl_2d, src2d/transport2d.jl:28-123 */
static double diff_tauN(double Tm, double alpha, const fivo_params& e, double DsT, double tauD) {
  double m = hq_mass(e);
  double z = m / Tm;
  if (e.eos_kind == FIVO_EOS_LATTICE_HRG) {
    if (z <= 0.0) return 0.0;
    double b1 = o_besselkx(1, z);
    double b2 = o_besselkx(2, z);
    double b3 = b1 + ((4.0 / z) * b2);
    double b4 = b2 + ((6.0 / z) * b3);
    double b5 = b3 + ((8.0 / z) * b4);
    double ex = o_exp(o_clamp(alpha - z, -700.0, 700.0));
    double tauq = (((e.g_hq * (DsT / ((96.0 * PI2) * ((Tm * Tm) * Tm)))) * o_pow5(m)) * ex) *
                  (((2.0 * b1) - (3.0 * b3)) + b5);
    double norm = fluidum_norm(Tm, alpha, e);
    if (std::fabs(norm) <= TINY) return 0.0;
    double tn = (tauq / norm) * (FMGEV * FMGEV);
    if (!o_isfinite(tn)) return 0.0;
    return o_max(tn, 0.0) * tauD;
  }
  if (z <= 0) return 0.0;
  if (z > 50.0) {
    double K2a = o_besselkx(2, z), K3a = o_besselkx(3, z);
    double tg = std::fabs(K2a) > TINY ? (((DsT * z) * (K3a / K2a)) / Tm) : ((DsT * z) / Tm);
    return o_min((tg / FMGEV) * tauD, 1e20);
  }
  double K1x = o_besselkx(1, z), K2x = o_besselkx(2, z), K3x = o_besselkx(3, z), K5x = o_besselkx(5, z);
  double numerator = ((2.0 * K1x) - (3.0 * K3x)) + K5x;
  double denominator = o_max(std::fabs(K2x), TINY);
  double ratio = (numerator / denominator) * o_sign(K2x == 0 ? 1.0 : K2x);
  double z3 = ((z * z) * z) / Tm;
  if (!o_isfinite(z3) || z3 > 1e50) z3 = 1e50;
  double tg = ((DsT / 48.0) * z3) * ratio;
  if (!o_isfinite(tg) || std::fabs(tg) > 1e50) return 1e50 * o_sign(tg);
  return (tg / FMGEV) * tauD;
}

/* viscosity / τ_shear (QGPViscosity), src/primitives.jl:56-65 */
static void shear_coeffs(double T, double mu, double n, double en, double P, const fivo_params& p,
                         double* eta, double* taupi, double* dpi) {
  if (!p.enable_shear) { *eta = 0; *taupi = 0; *dpi = 0; return; }
  double s = eos_entropy(T, mu, n, en, P);
  if (p.shear_kind != FIVO_SHEAR_QGP) { *eta = 0.0; *taupi = 0.0; *dpi = p.deltaShear_factor * 0.0; return; }
  double h = (o_max(p.eta_over_s, 0.0) * o_max(s, 0.0)) * INVFMGEV;
  double Ts = posden(T) * posden(s);
  double tp = safe_div(h, (Ts * posden(p.tauShear_coeff)));
  *eta = h; *taupi = tp; *dpi = p.deltaShear_factor * tp;
}

/* bulk_viscosity / τ_bulk, src/primitives.jl:98-108 (+ the Gaussian subtype) */
static void bulk_coeffs(double T, double mu, double n, double en, double P, const fivo_params& p,
                        double* zeta, double* tauPi) {
  if (!p.enable_bulk) { *zeta = 0.0; *tauPi = 0.0; return; }
  double s = eos_entropy(T, mu, n, en, P);
  double cs2 = eos_cs2(T, mu, p);
  if (p.bulk_kind == FIVO_BULK_ZERO) { *zeta = 0.0; *tauPi = 0.0; return; }
  double peak;
  if (p.bulk_kind == FIVO_BULK_LORENTZ) {
    double q = (T - 0.175) / 0.024;
    peak = p.zeta_over_s / (1.0 + (q * q));
  } else {
    double q = (T - p.bulk_T0) / p.bulk_width;
    peak = p.zeta_over_s * o_exp(-0.5 * (q * q));
  }
  double z = (peak * INVFMGEV) * o_max(s, 0.0);
  double sp = posden(s);
  double Dl = o_max(std::fabs((1.0 / 3.0) - cs2), 1e-8);
  *zeta = z;
  *tauPi = (safe_div(z, ((posden(T) * sp) * posden(p.tauPi_coeff))) * (1.0 / (Dl * Dl))) + 0.1;
}

/* diff_coeffs_2d, src2d/transport2d.jl:131-141 */
static void diff_coeffs(double T, double mu, double n, const fivo_params& p, double* kappa,
                        double* taun, double* dN) {
  if (!p.enable_diff) { *kappa = 0; *taun = 0; *dN = 0; return; }
  double Tm = posden(T);
  double alpha = mu / Tm;
  double DsT = p.kappa_coeff;
  *kappa = (safe_div(DsT, Tm) * o_max(n, 0.0)) / FMGEV;
  *taun = diff_tauN(Tm, alpha, p, DsT, p.tauN_coeff);
  *dN = p.deltaN_factor * (*taun);
}

/* vacuum_weight_2d, src2d/transport2d.jl:149-155 */
static inline double vacuum_weight(double n, const fivo_params& p) {
  double lo = p.vacuum_n_lo, hi = p.vacuum_n_hi;
  if (hi <= lo) return 1.0;
  if (n <= lo) return 0.0;
  if (n >= hi) return 1.0;
  return (n - lo) / (hi - lo);
}

/* ======================= relaxation (src2d/dissipation2d.jl) ======================= */

struct Kin { double th, ax, ay, at, dxux, dxuy, dyux, dyuy; };

/* kinematics_2d, src2d/dissipation2d.jl:141-167 */
static Kin kinematics(const Work& w, const Grid& g, int64_t i, double D, double tau) {
  double invdx = 1.0 / (2.0 * g.dx), invdy = 1.0 / (2.0 * g.dy);
  int64_t ixm = i - g.Nytot, ixp = i + g.Nytot;
  Kin k;
  k.dxux = (w.ux[ixp] - w.ux[ixm]) * invdx;
  k.dxuy = (w.uy[ixp] - w.uy[ixm]) * invdx;
  k.dyux = (w.ux[i + 1] - w.ux[i - 1]) * invdy;
  k.dyuy = (w.uy[i + 1] - w.uy[i - 1]) * invdy;
  double ux = w.ux[i], uy = w.uy[i];
  double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
  double uxp = w.ux_prev[i], uyp = w.uy_prev[i];
  bool have_prev = o_isfinite(uxp) && o_isfinite(uyp);
  double dtux = have_prev ? (ux - uxp) / D : 0.0;
  double dtuy = have_prev ? (uy - uyp) / D : 0.0;
  double dtut = ((ux * dtux) + (uy * dtuy)) * safe_inv(ut);
  k.th = ((dtut + k.dxux) + k.dyuy) + (ut * safe_inv(tau));
  k.ax = ((ut * dtux) + (ux * k.dxux)) + (uy * k.dyux);
  k.ay = ((ut * dtuy) + (ux * k.dxuy)) + (uy * k.dyuy);
  k.at = ((ux * k.ax) + (uy * k.ay)) * safe_inv(ut);
  return k;
}

/* ns_shear_target_2d, src2d/dissipation2d.jl:181-192 */
static void ns_shear_target(double ux, double uy, double ut, double tau, const Kin& k, double eta,
                            double* xx, double* xy, double* yy, double* et) {
  double third = k.th / 3.0;
  double sxx = (k.dxux + (ux * k.ax)) - (third * (1.0 + (ux * ux)));
  double syy = (k.dyuy + (uy * k.ay)) - (third * (1.0 + (uy * uy)));
  double sxy = ((0.5 * (k.dxuy + k.dyux)) + (0.5 * ((ux * k.ay) + (uy * k.ax)))) - (third * (ux * uy));
  double seta = (ut * safe_inv(tau)) - third;
  double m2 = -2.0 * eta;
  *xx = m2 * sxx; *xy = m2 * sxy; *yy = m2 * syy; *et = m2 * seta;
}

/* ns_diffusion_target_2d, src2d/dissipation2d.jl:204-209:
 * nu_NS^i = -kappa (d_i alpha + u^i D alpha), D alpha = u^tau d_tau alpha + u^k d_k alpha */
static inline void ns_diffusion_target(double ux, double uy, double ut, double dxa, double dya, double dta,
                                       double kappa, double* nsx, double* nsy) {
  double Da = ((ut * dta) + (ux * dxa)) + (uy * dya);
  *nsx = (-kappa) * (dxa + (ux * Da));
  *nsy = (-kappa) * (dya + (uy * Da));
}

/* pi_sigma_contractions_2d, src2d/hq_consistent_m2_2d.jl:201-210 */
static void pi_sigma(double ux, double uy, double pxx, double pxy, double pyy, double peta,
                     double sxx, double sxy, double syy, double seta,
                     double* ps, double* cxx, double* cxy, double* cyy) {
  double ux2 = ux * ux, uy2 = uy * uy, ux3 = (ux * ux) * ux, uy3 = (uy * uy) * uy, ux4 = o_pow4(ux);
  double opuy2 = 1.0 + uy2;
  double u2 = (1.0 + ux2) + uy2;
  double num = ((((((((((((((((2.0 * pxy) * sxy) + (pyy * syy)) + (((2.0 * pxy) * sxy) * ux2)) +
      (((2.0 * pyy) * syy) * ux2)) + ((pyy * syy) * ux4)) - ((((2.0 * pxy) * sxx) * ux) * uy)) -
      ((((2.0 * pyy) * sxy) * ux) * uy)) - ((((2.0 * pxy) * syy) * ux) * uy)) -
      ((((2.0 * pyy) * sxy) * ux3) * uy)) - ((((2.0 * pxy) * syy) * ux3) * uy)) +
      (((2.0 * pxy) * sxy) * uy2)) + (((pyy * sxx) * ux2) * uy2)) + ((((4.0 * pxy) * sxy) * ux2) * uy2)) -
      ((((2.0 * pxy) * sxx) * ux) * uy3)) + ((pxx * sxx) * (opuy2 * opuy2))) +
      ((peta * seta) * (u2 * u2));
  num = num + (((pxx * ux) * uy) * (((syy * ux) * uy) - ((2.0 * sxy) * opuy2)));
  *ps = num / (u2 * u2);
  *cxx = ((pxx * sxx) + (pxy * sxy)) - ((((pxx * ux) + (pxy * uy)) * ((sxx * ux) + (sxy * uy))) / u2);
  *cyy = ((pxy * sxy) + (pyy * syy)) - ((((pxy * ux) + (pyy * uy)) * ((sxy * ux) + (syy * uy))) / u2);
  double t1 = pyy * ((sxy + (sxy * ux2)) - ((sxx * ux) * uy));
  double t2 = pxy * ((((sxx + syy) + (syy * ux2)) - (((2.0 * sxy) * ux) * uy)) + (sxx * uy2));
  double t3 = pxx * ((sxy - ((syy * ux) * uy)) + (sxy * uy2));
  *cxy = ((t1 + t2) + t3) / (2.0 * u2);
}

/* vorticity_coupling_2d, src2d/hq_consistent_m2_2d.jl:442-468 */
static void vorticity_coupling(double ux, double uy, double ut, double tau, double pxx, double pxy,
                               double pyy, double peta, double ax, double ay, double dtux, double dtuy,
                               double dxux, double dxuy, double dyux, double dyuy,
                               double* wxx, double* wxy, double* wyy) {
  double iu = safe_inv(ut);
  double at = ((ux * ax) + (uy * ay)) * iu;
  double dxut = ((ux * dxux) + (uy * dxuy)) * iu;
  double dyut = ((ux * dyux) + (uy * dyuy)) * iu;
  double Atx = (-dtux) + (ut * ax), Axt = dxut + (ux * at);
  double Aty = (-dtuy) + (ut * ay), Ayt = dyut + (uy * at);
  double Axy = dxuy + (ux * ay), Ayx = dyux + (uy * ax);
  double wtx = 0.5 * (Atx - Axt), wty = 0.5 * (Aty - Ayt), wxy_ = 0.5 * (Axy - Ayx);
  PiC Pc = shear_tensor(ux, uy, ut, tau, pxx, pxy, pyy, peta);
  double Mxx = ((-Pc.tx) * wtx) - (Pc.xy * wxy_);
  double Mxy = ((-Pc.tx) * wty) + (Pc.xx * wxy_);
  double Myx = ((-Pc.ty) * wtx) - (Pc.yy * wxy_);
  double Myy = ((-Pc.ty) * wty) + (Pc.xy * wxy_);
  *wxx = 2.0 * Mxx; *wxy = Mxy + Myx; *wyy = 2.0 * Myy;
}

/* compute_alpha_grad_fv_2d!, src2d/dissipation2d.jl:225-260 */
static void compute_alpha_grad(Work& w, const Grid& g) {
  const int ng = g.ng;
  const double* a = w.alpha.data();
  for (int d = 0; d < 2; ++d) {
    bool xdir = d == 0;
    int64_t st = xdir ? g.Nytot : 1;
    double* face = xdir ? w.alphaFx.data() : w.alphaFy.data();
    double* grad = xdir ? w.gradAx.data() : w.gradAy.data();
    double invd = xdir ? 1.0 / g.dx : 1.0 / g.dy;
    double* sl = w.slope_tmp.data();
    std::fill(sl, sl + g.Ntot, 0.0); std::fill(face, face + g.Ntot, 0.0); std::fill(grad, grad + g.Ntot, 0.0);
    int lo = xdir ? 1 : 0, hi = xdir ? g.Nxtot - 2 : g.Nxtot - 1;
    int ylo = xdir ? 0 : 1, yhi = xdir ? g.Nytot - 1 : g.Nytot - 2;
    for (int ix = lo; ix <= hi; ++ix)
      for (int iy = ylo; iy <= yhi; ++iy) {
        int64_t i = g.lin(ix, iy);
        sl[i] = mc_limiter(a[i] - a[i - st], a[i + st] - a[i]);
      }
    int fhi = xdir ? g.Nxtot - 2 : g.Nxtot - 1;
    int gyhi = xdir ? g.Nytot - 1 : g.Nytot - 2;
    int kmax = xdir ? g.Nxtot : g.Nytot;
    for (int ix = 0; ix <= fhi; ++ix)
      for (int iy = 0; iy <= gyhi; ++iy) {
        int64_t i = g.lin(ix, iy), ip = i + st;
        int k = (xdir ? ix : iy) + 1;
        if (k <= ng || k >= kmax - ng) face[i] = 0.5 * (a[i] + a[ip]);
        else face[i] = 0.5 * ((a[i] + (0.5 * sl[i])) + (a[ip] - (0.5 * sl[ip])));
      }
    for (int ix = ng; ix < ng + g.Nx; ++ix)
      for (int iy = ng; iy < ng + g.Ny; ++iy) {
        int64_t i = g.lin(ix, iy);
        grad[i] = (face[i] - face[i - st]) * invd;
      }
  }
}

/* ---- the consistent charm first moment, src2d/hq_consistent_firstmoment2d.jl ---- */

/* hq_h_hprime_2d, :145-160: h = m K3/K2 and dh/dT (scaled Bessel functions) */
static void hq_h_hprime(double T, const fivo_params& p, double* h, double* hp) {
  double Tm = o_max(T, T_MIN);
  double m = p.m_hq;
  double z = m / Tm;
  *h = 0.0; *hp = 0.0;
  if (z <= 0.0) return;
  double K1 = o_besselkx(1, z), K2 = o_besselkx(2, z), K3 = o_besselkx(3, z), K4 = o_besselkx(4, z);
  if (std::fabs(K2) <= TINY) return;
  double hv = (m * K3) / K2;
  double hpv = ((m * z) / Tm) * ((((K2 + K4) * K2) - ((K1 + K3) * K3))) / ((2.0 * K2) * K2);
  *h = o_isfinite(hv) ? hv : 0.0;
  *hp = o_isfinite(hpv) ? hpv : 0.0;
}

/* hq_dn_dT_2d, :172-182: dn/dT at fixed alpha = (n/T)(3 + z K1/K2) */
static double hq_dn_dT(double T, double n, const fivo_params& p) {
  double Tm = o_max(T, T_MIN);
  double z = p.m_hq / Tm;
  if (z <= 0.0) return 0.0;
  double K1 = o_besselkx(1, z), K2 = o_besselkx(2, z);
  if (std::fabs(K2) <= TINY) return 0.0;
  double v = (n / Tm) * (3.0 + ((z * K1) / K2));
  return o_isfinite(v) ? v : 0.0;
}

/* consistent_fm_source_2d, :218-282: the sources s^i, SOURCE-ON-THE-LHS */
static void consistent_fm_source(double ux, double uy, double ut, double T, double dxT, double dyT, double dtT,
                                 double nux, double nuy, double n, double dn_dT, double tn, double Ds, double hp,
                                 const Kin& k, uint32_t terms, double* sx, double* sy) {
  double Tm = o_max(T, T_MIN);
  double DT = ((ut * dtT) + (ux * dxT)) + (uy * dyT);
  double gTx = dxT + (ux * DT);
  double gTy = dyT + (uy * DT);
  double nut = nu_tau(ux, uy, ut, nux, nuy);
  double dtux = ((k.ax - (ux * k.dxux)) - (uy * k.dyux)) * safe_inv(ut);
  double dtuy = ((k.ay - (ux * k.dxuy)) - (uy * k.dyuy)) * safe_inv(ut);
  double ngux = ((nut * dtux) + (nux * k.dxux)) + (nuy * k.dyux);
  double nguy = ((nut * dtuy) + (nux * k.dxuy)) + (nuy * k.dyuy);
  double expansion = (terms & FIVO_TERM_FM_EXPANSION) ? tn * k.th : 0.0;
  double dlnh = (terms & FIVO_TERM_FM_DLNH) ? ((Ds / Tm) * hp) * DT : 0.0;
  double br = expansion + dlnh;
  double pref = (Ds / Tm) * (n + (Tm * dn_dT));
  *sx = ((((terms & FIVO_TERM_FM_GRADT) ? pref * gTx : 0.0) + ((terms & FIVO_TERM_FM_INERTIAL) ? (tn * n) * k.ax : 0.0)) +
         ((terms & FIVO_TERM_FM_NU_GRADU) ? tn * ngux : 0.0)) + (nux * br);
  *sy = ((((terms & FIVO_TERM_FM_GRADT) ? pref * gTy : 0.0) + ((terms & FIVO_TERM_FM_INERTIAL) ? (tn * n) * k.ay : 0.0)) +
         ((terms & FIVO_TERM_FM_NU_GRADU) ? tn * nguy : 0.0)) + (nuy * br);
}

/* the closure's pieces with plain arguments, for the gate tests */
void cfm_h_hprime(double T, const fivo_params& p, double* h, double* hp) { hq_h_hprime(T, p, h, hp); }
double cfm_dn_dT(double T, double n, const fivo_params& p) { return hq_dn_dT(T, n, p); }
void cfm_diff_coeffs(double T, double mu, double n, const fivo_params& p, double* kappa, double* taun,
                     double* dN) {
  diff_coeffs(T, mu, n, p, kappa, taun, dN);
}
void cfm_source(double ux, double uy, double ut, double T, double dxT, double dyT, double dtT, double nux,
                double nuy, double n, double dn_dT, double tn, double Ds, double hp, double th, double ax,
                double ay, double dxux, double dxuy, double dyux, double dyuy, uint32_t terms, double* sx,
                double* sy) {
  const Kin k{th, ax, ay, 0.0, dxux, dxuy, dyux, dyuy};
  consistent_fm_source(ux, uy, ut, T, dxT, dyT, dtT, nux, nuy, n, dn_dT, tn, Ds, hp, k, terms, sx, sy);
}

/* ---- the consistent charm second moment, src2d/hq_consistent_m2_2d.jl ---- */

/* hq_m2_coeffs_2d, src2d/hq_consistent_m2_2d.jl:125-142: dlnC/dlnT, eta_bar, lambda_a, A, A/B */
struct M2Coeffs { double dlnC, etabar, lama, Aco, ABr; };
static M2Coeffs hq_m2_coeffs(double T, double n, double tn, double Ds, double h, double m) {
  double Tm = o_max(T, T_MIN);
  double z = m / Tm;
  double K2 = o_besselkx(2, z), K3 = o_besselkx(3, z), K4 = o_besselkx(4, z);
  double K5 = K3 + ((8.0 * K4) / z);
  double dl = (std::fabs(K4) > TINY && std::fabs(K3) > TINY)
                  ? z * (((K3 + K5) / (2.0 * K4)) - ((K2 + K4) / (2.0 * K3))) : 0.0;
  M2Coeffs c;
  c.etabar = ((tn * n) * Tm) / 2.0;
  c.lama = (Ds * ((m * m) + ((6.0 * Tm) * h))) / (2.0 * Tm);
  c.Aco = (m * m) + ((5.0 * Tm) * h);
  double abr = std::fabs(K3) > TINY ? 5.0 + ((z * K2) / K3) : 5.0;
  c.dlnC = o_isfinite(dl) ? dl : 0.0;
  c.ABr = o_isfinite(abr) ? abr : 5.0;
  return c;
}

/* tauM_charm_2d, src2d/transport2d.jl:177-184: tau_M = tau_n K4 K2 / (2 K3^2) */
static double tauM_charm(double T, double tn, double m) {
  double Tm = o_max(T, T_MIN), z = m / Tm;
  double K2 = o_besselkx(2, z), K3 = o_besselkx(3, z), K4 = o_besselkx(4, z);
  if (std::fabs(K3) <= TINY) return 0.0;
  double v = ((tn * K4) * K2) / ((2.0 * K3) * K3);
  return (o_isfinite(v) && v > 0) ? v : 0.0;
}

/* etaM_charm_2d, src2d/transport2d.jl:186 */
static inline double etaM_charm(double T, double tn) { return (o_max(T, T_MIN) * tn) / 2.0; }

/* sigma_nu_2d, src2d/hq_consistent_m2_2d.jl:171-182: the transverse-projected
 * traceless gradient of the current (the generated closed forms, in their order) */
static void sigma_nu(double uxv, double uyv, double uT, double tau, double nux, double nuy, double dtnx,
                     double dxnx, double dynx, double dtny, double dxny, double dyny, double dtux, double dxux,
                     double dyux, double dtuy, double dxuy, double dyuy, double* oxx, double* oxy, double* oyy,
                     double* oeta) {
  const double sxx = (((((tau * ((1.0 + (uxv * uxv)) + (uyv * uyv))) * (((((((2.0 * dtnx) * ((uxv * uxv) * uxv)) - (dtny * uyv)) + ((2.0 * dxnx) * uT)) - (dyny * uT)) - ((uxv * uxv) * (((dtny * uyv) - ((2.0 * dxnx) * uT)) + (dyny * uT)))) + (uxv * (((2.0 * dtnx) + ((3.0 * dtnx) * (uyv * uyv))) + (((3.0 * dynx) * uyv) * uT))))) + (nuy * ((((((((-1.0) - ((dtux * tau) * uxv)) - (uxv * uxv)) + (((2.0 * dtux) * tau) * ((uxv * uxv) * uxv))) * ((uyv * uyv) * uyv)) - ((((2.0 * tau) * uxv) * ((1.0 + (uxv * uxv)) * (1.0 + (uxv * uxv)))) * ((dtuy * uxv) + (dxuy * uT)))) - (((tau * ((-1.0) + (2.0 * (uxv * uxv)))) * (uyv * uyv)) * ((dtuy + (dtuy * (uxv * uxv))) - ((dyux * uxv) * uT)))) + (((1.0 + (uxv * uxv)) * uyv) * ((((-1.0) + (((2.0 * dtux) * tau) * ((uxv * uxv) * uxv))) + ((dyuy * tau) * uT)) + ((uxv * uxv) * (((-1.0) + (((2.0 * dxux) * tau) * uT)) - (((2.0 * dyuy) * tau) * uT)))))))) + (nux * ((((((o_pow5(uxv) * ((-1.0) + (((2.0 * dtuy) * tau) * uyv))) + (((tau * uyv) * (1.0 + (uyv * uyv))) * ((dtux * uyv) + (dyux * uT)))) + (((2.0 * tau) * o_pow4(uxv)) * (((-dtux) - (dtux * (uyv * uyv))) + ((dxuy * uyv) * uT)))) - (((2.0 * tau) * (uxv * uxv)) * ((((dtux + ((2.0 * dtux) * (uyv * uyv))) + (dtux * o_pow4(uyv))) + ((((-dxuy) + dyux) * uyv) * uT)) + ((dyux * ((uyv * uyv) * uyv)) * uT)))) - (uxv * (((1.0 + ((dtuy * tau) * ((uyv * uyv) * uyv))) + (((2.0 * dxux) * tau) * uT)) + ((uyv * uyv) * ((1.0 + (((2.0 * dxux) * tau) * uT)) + ((dyuy * tau) * uT)))))) + (((uxv * uxv) * uxv) * ((((((2.0 * dtuy) * tau) * uyv) + (((2.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) - (2.0 * (1.0 + ((dxux * tau) * uT)))) + ((uyv * uyv) * (((-1.0) - (((2.0 * dxux) * tau) * uT)) + (((2.0 * dyuy) * tau) * uT)))))))) / ((3.0 * tau) * o_pow15(((1.0 + (uxv * uxv)) + (uyv * uyv)))));
  const double sxy = (((((tau * ((1.0 + (uxv * uxv)) + (uyv * uyv))) * ((((((3.0 * dtny) * ((uxv * uxv) * uxv)) + (((3.0 * dynx) * (1.0 + (uyv * uyv))) * uT)) + (3.0 * (((dtnx * uyv) * (1.0 + (uyv * uyv))) + (dxny * uT)))) + ((uxv * uxv) * ((dtnx * uyv) + ((3.0 * dxny) * uT)))) + (uxv * (((3.0 * dtny) + (dtny * (uyv * uyv))) + (((dxnx + dyny) * uyv) * uT))))) - (nuy * (((((((((4.0 * dtuy) * tau) * o_pow5(uxv)) * uyv) + ((((3.0 * dxuy) * tau) * uyv) * uT)) + ((((4.0 * tau) * o_pow4(uxv)) * uyv) * ((-(dtux * uyv)) + (dxuy * uT)))) - (((tau * (uxv * uxv)) * uyv) * (((((-7.0) * dxuy) * uT) + (((2.0 * dtux) * uyv) * (3.0 + (2.0 * (uyv * uyv))))) + ((dyux * uT) * (3.0 + (4.0 * (uyv * uyv))))))) + (((uxv * uxv) * uxv) * ((((((10.0 * dtuy) * tau) * uyv) + (((4.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) + (((3.0 * dyuy) * tau) * uT)) + ((uyv * uyv) * ((2.0 - (((4.0 * dxux) * tau) * uT)) + (((4.0 * dyuy) * tau) * uT)))))) + (uxv * (((((((6.0 * dtuy) * tau) * uyv) + (((4.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) + (2.0 * o_pow4(uyv))) + (((3.0 * dyuy) * tau) * uT)) + ((uyv * uyv) * ((2.0 - (((3.0 * dxux) * tau) * uT)) + (((4.0 * dyuy) * tau) * uT)))))))) + (nux * (((((((2.0 * o_pow4(uxv)) * uyv) * ((-1.0) + (((2.0 * dtuy) * tau) * uyv))) - (((((3.0 * dxux) * tau) * uyv) * (1.0 + (uyv * uyv))) * uT)) - ((((4.0 * tau) * ((uxv * uxv) * uxv)) * uyv) * ((dtux + (dtux * (uyv * uyv))) - ((dxuy * uyv) * uT)))) + (((uxv * uxv) * uyv) * ((((((-2.0) + (((6.0 * dtuy) * tau) * uyv)) + (((4.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) - (((4.0 * dxux) * tau) * uT)) + (((3.0 * dyuy) * tau) * uT)) + ((uyv * uyv) * (((-2.0) - (((4.0 * dxux) * tau) * uT)) + (((4.0 * dyuy) * tau) * uT)))))) - ((tau * uxv) * (((dyux * uT) * ((3.0 + (7.0 * (uyv * uyv))) + (4.0 * o_pow4(uyv)))) + (uyv * ((((6.0 * dtux) + ((10.0 * dtux) * (uyv * uyv))) + ((4.0 * dtux) * o_pow4(uyv))) - (((3.0 * dxuy) * uyv) * uT)))))))) / ((6.0 * tau) * o_pow15(((1.0 + (uxv * uxv)) + (uyv * uyv)))));
  const double syy = (((((tau * ((1.0 + (uxv * uxv)) + (uyv * uyv))) * ((((((((-(dtnx * uxv)) + ((2.0 * dtny) * uyv)) + (((3.0 * dtny) * (uxv * uxv)) * uyv)) - ((dtnx * uxv) * (uyv * uyv))) + ((2.0 * dtny) * ((uyv * uyv) * uyv))) + ((((3.0 * dxny) * uxv) * uyv) * uT)) - ((dxnx * (1.0 + (uyv * uyv))) * uT)) + (((2.0 * dyny) * (1.0 + (uyv * uyv))) * uT))) + (nux * ((((((uxv * uxv) * uxv) * ((((-1.0) - ((dtuy * tau) * uyv)) - (uyv * uyv)) + (((2.0 * dtuy) * tau) * ((uyv * uyv) * uyv)))) - ((((2.0 * tau) * uyv) * ((1.0 + (uyv * uyv)) * (1.0 + (uyv * uyv)))) * ((dtux * uyv) + (dyux * uT)))) - (((tau * (uxv * uxv)) * ((-1.0) + (2.0 * (uyv * uyv)))) * ((dtux + (dtux * (uyv * uyv))) - ((dxuy * uyv) * uT)))) + ((uxv * (1.0 + (uyv * uyv))) * ((((-1.0) + (((2.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) + ((dxux * tau) * uT)) + ((uyv * uyv) * (((-1.0) - (((2.0 * dxux) * tau) * uT)) + (((2.0 * dyuy) * tau) * uT)))))))) + (nuy * ((((((((-1.0) + (((2.0 * dtux) * tau) * uxv)) * o_pow5(uyv)) + (((tau * uxv) * (1.0 + (uxv * uxv))) * ((dtuy * uxv) + (dxuy * uT)))) + (((2.0 * tau) * o_pow4(uyv)) * (((-dtuy) - (dtuy * (uxv * uxv))) + ((dyux * uxv) * uT)))) - (((2.0 * tau) * (uyv * uyv)) * ((((dtuy + ((2.0 * dtuy) * (uxv * uxv))) + (dtuy * o_pow4(uxv))) + (((dxuy - dyux) * uxv) * uT)) + ((dxuy * ((uxv * uxv) * uxv)) * uT)))) + (((uyv * uyv) * uyv) * ((((((2.0 * dtux) * tau) * uxv) + (((2.0 * dtux) * tau) * ((uxv * uxv) * uxv))) + ((uxv * uxv) * (((-1.0) + (((2.0 * dxux) * tau) * uT)) - (((2.0 * dyuy) * tau) * uT)))) - (2.0 * (1.0 + ((dyuy * tau) * uT)))))) - (uyv * (((1.0 + ((dtux * tau) * ((uxv * uxv) * uxv))) + (((2.0 * dyuy) * tau) * uT)) + ((uxv * uxv) * ((1.0 + ((dxux * tau) * uT)) + (((2.0 * dyuy) * tau) * uT)))))))) / ((3.0 * tau) * o_pow15(((1.0 + (uxv * uxv)) + (uyv * uyv)))));
  const double seta = (((((((((-dxnx) - dyny) + ((((dtux * uxv) + (dtuy * uyv)) * ((nux * uxv) + (nuy * uyv))) / o_pow15(((1.0 + (uxv * uxv)) + (uyv * uyv))))) - (((((dtux * nux) + (dtuy * nuy)) + (dtnx * uxv)) + (dtny * uyv)) / uT)) + ((2.0 * ((nux * uxv) + (nuy * uyv))) / (tau * uT))) + (nux * (((dxux * uxv) + (dyux * uyv)) + (dtux * uT)))) + (nuy * (((dxuy * uxv) + (dyuy * uyv)) + (dtuy * uT)))) - ((((nux * uxv) + (nuy * uyv)) * (((dxux * (uxv * uxv)) + (uxv * (((dxuy + dyux) * uyv) + (dtux * uT)))) + (uyv * ((dyuy * uyv) + (dtuy * uT))))) / ((1.0 + (uxv * uxv)) + (uyv * uyv)))) / 3.0);
  *oxx = sxx; *oxy = sxy; *oyy = syy; *oeta = seta;
}

/* rank1_traceless_2d, src2d/hq_consistent_m2_2d.jl:225-234: A^<i B^j> for two u-orthogonal transverse vectors */
static void rank1_traceless(double Ax, double Ay, double Bx, double By, double ux, double uy, double ut,
                            double* qxx, double* qxy, double* qyy) {
  double u2 = ut * ut;
  double tr = ((Ay * ((By + (By * (ux * ux))) - ((Bx * ux) * uy))) + (Ax * ((Bx - ((By * ux) * uy)) + (Bx * (uy * uy))))) / u2;
  *qxx = (Ax * Bx) - (((1.0 + (ux * ux)) * tr) / 3.0);
  *qyy = (Ay * By) - (((1.0 + (uy * uy)) * tr) / 3.0);
  *qxy = (((Ay * Bx) + (Ax * By)) / 2.0) - (((ux * uy) * tr) / 3.0);
}

/* consistent_m2_source_2d, src2d/hq_consistent_m2_2d.jl:247-404: d_tau of (pQxx, pQxy, pQyy, PiQ) and geo, each
 * term behind its Terms switch. a[] holds the 44 positional arguments in order. */
enum {
  M2_UX, M2_UY, M2_UT, M2_TAU, M2_T, M2_DXT, M2_DYT, M2_DTT, M2_NUX, M2_NUY, M2_PXX, M2_PXY, M2_PYY, M2_PETA,
  M2_PIQ, M2_DTA, M2_DXA, M2_DYA, M2_THNU, M2_ANUX, M2_ANUY, M2_DTNUX, M2_DTNUY, M2_DXNUX, M2_DXNUY, M2_DYNUX,
  M2_DYNUY, M2_TH, M2_AX, M2_AY, M2_DTUX, M2_DTUY, M2_DXUX, M2_DXUY, M2_DYUX, M2_DYUY, M2_N, M2_TN, M2_DS, M2_H,
  M2_HP, M2_TM, M2_ETAM, M2_M, M2_NARG
};
static void consistent_m2_source(const double* a, uint32_t t, double* out) {
  const double ux = a[M2_UX], uy = a[M2_UY], ut = a[M2_UT], tau = a[M2_TAU];
  const double Tm = o_max(a[M2_T], T_MIN);
  const double tM = a[M2_TM];
  if (!(tM > 0.0)) { for (int j = 0; j < 5; ++j) out[j] = 0.0; return; }
  const double nux = a[M2_NUX], nuy = a[M2_NUY];
  const double pxx = a[M2_PXX], pxy = a[M2_PXY], pyy = a[M2_PYY], peta = a[M2_PETA], PiQ = a[M2_PIQ];
  const double th = a[M2_TH], ax = a[M2_AX], ay = a[M2_AY];
  const double Ds = a[M2_DS], h = a[M2_H], hp = a[M2_HP];
  const double etaQ = a[M2_ETAM];
  const double zetaQ = (5.0 / 3.0) * etaQ;
  const M2Coeffs cf = hq_m2_coeffs(Tm, a[M2_N], a[M2_TN], Ds, h, a[M2_M]);
  /* the medium's shear at unit viscosity: ns_shear_target_2d(..., -1/2) */
  const Kin k{th, ax, ay, 0.0, a[M2_DXUX], a[M2_DXUY], a[M2_DYUX], a[M2_DYUY]};
  double sxx_, sxy_, syy_, seta_;
  ns_shear_target(ux, uy, ut, tau, k, -0.5, &sxx_, &sxy_, &syy_, &seta_);
  const double anudot = ((ax * nux) + (ay * nuy)) - ((((ax * ux) + (ay * uy)) * ((nux * ux) + (nuy * uy))) / (ut * ut));
  double snxx, snxy, snyy, sneta;
  sigma_nu(ux, uy, ut, tau, nux, nuy, a[M2_DTNUX], a[M2_DXNUX], a[M2_DYNUX], a[M2_DTNUY], a[M2_DXNUY],
           a[M2_DYNUY], a[M2_DTUX], a[M2_DXUX], a[M2_DYUX], a[M2_DTUY], a[M2_DXUY], a[M2_DYUY], &snxx, &snxy,
           &snyy, &sneta);
  const double DT = ((ut * a[M2_DTT]) + (ux * a[M2_DXT])) + (uy * a[M2_DYT]);
  const double DlnT = DT / Tm;
  const double DlnC = cf.dlnC * DlnT;
  const double Da = ((ut * a[M2_DTA]) + (ux * a[M2_DXA])) + (uy * a[M2_DYA]);
  const double geo = (t & FIVO_TERM_M2_EXPANSION) ? tM * (((5.0 / 3.0) * th) + DlnC) : 0.0;
  double ps, cxx, cxy, cyy;
  pi_sigma(ux, uy, pxx, pxy, pyy, peta, sxx_, sxy_, syy_, seta_, &ps, &cxx, &cxy, &cyy);
  const double gTx = (h + (Tm * hp)) * (a[M2_DXT] + (ux * DT));
  const double gTy = (h + (Tm * hp)) * (a[M2_DYT] + (uy * DT));
  double qaxx, qaxy, qayy, qgxx, qgxy, qgyy;
  rank1_traceless(ax, ay, nux, nuy, ux, uy, ut, &qaxx, &qaxy, &qayy);
  rank1_traceless(nux, nuy, gTx, gTy, ux, uy, ut, &qgxx, &qgxy, &qgyy);
  const bool ia = t & FIVO_TERM_M2_ACCEL_NU, ig = t & FIVO_TERM_M2_NU_GRADTH;
  const double qxx = (ia ? (2.0 * cf.lama) * qaxx : 0.0) + (ig ? (Ds / Tm) * qgxx : 0.0);
  const double qyy = (ia ? (2.0 * cf.lama) * qayy : 0.0) + (ig ? (Ds / Tm) * qgyy : 0.0);
  const double qxy = (ia ? (2.0 * cf.lama) * qaxy : 0.0) + (ig ? (Ds / Tm) * qgxy : 0.0);
  const bool i1 = t & FIVO_TERM_M2_NU_GRADIENT, i2 = t & FIVO_TERM_M2_BG_GRADU;
  const bool i3 = t & FIVO_TERM_M2_PI_SIGMA, i4 = t & FIVO_TERM_M2_PIQ_SIGMA;
  double sxx = ((((((pxx + (i1 ? (2.0 * etaQ) * snxx : 0.0)) + (geo * pxx)) +
                  (i3 ? (2.0 * tM) * (cxx - (((1.0 + (ux * ux)) * ps) / 3.0)) : 0.0)) +
                 (i4 ? ((2.0 * tM) * PiQ) * sxx_ : 0.0)) + (i2 ? (2.0 * cf.etabar) * sxx_ : 0.0)) + qxx);
  double syy = ((((((pyy + (i1 ? (2.0 * etaQ) * snyy : 0.0)) + (geo * pyy)) +
                  (i3 ? (2.0 * tM) * (cyy - (((1.0 + (uy * uy)) * ps) / 3.0)) : 0.0)) +
                 (i4 ? ((2.0 * tM) * PiQ) * syy_ : 0.0)) + (i2 ? (2.0 * cf.etabar) * syy_ : 0.0)) + qyy);
  double sxy = ((((((pxy + (i1 ? (2.0 * etaQ) * snxy : 0.0)) + (geo * pxy)) +
                  (i3 ? (2.0 * tM) * (cxy - (((ux * uy) * ps) / 3.0)) : 0.0)) +
                 (i4 ? ((2.0 * tM) * PiQ) * sxy_ : 0.0)) + (i2 ? (2.0 * cf.etabar) * sxy_ : 0.0)) + qxy);
  if (t & FIVO_TERM_M2_VORTICITY) {
    double wxx, wxy, wyy;
    vorticity_coupling(ux, uy, ut, tau, pxx, pxy, pyy, peta, ax, ay, a[M2_DTUX], a[M2_DTUY], a[M2_DXUX],
                       a[M2_DXUY], a[M2_DYUX], a[M2_DYUY], &wxx, &wxy, &wyy);
    sxx += tM * wxx; sxy += tM * wxy; syy += tM * wyy;
  }
  if (t & FIVO_TERM_M2_PROJECTOR) {
    const double at = ((ux * ax) + (uy * ay)) / ut;
    const PiC Q = shear_tensor(ux, uy, ut, tau, pxx, pxy, pyy, peta);
    const double cx = (((-Q.tx) * at) + (Q.xx * ax)) + (Q.xy * ay);
    const double cy = (((-Q.ty) * at) + (Q.xy * ax)) + (Q.yy * ay);
    sxx -= tM * ((2.0 * ux) * cx);
    sxy -= tM * ((ux * cy) + (uy * cx));
    syy -= tM * ((2.0 * uy) * cy);
  }
  const double sB =
      (((((((PiQ + (i1 ? zetaQ * a[M2_THNU] : 0.0)) + (geo * PiQ)) + (i3 ? ((2.0 / 3.0) * tM) * ps : 0.0)) +
          (cf.etabar * (((t & FIVO_TERM_M2_BG_DLNT) ? cf.ABr * DlnT : 0.0) + (i2 ? (5.0 / 3.0) * th : 0.0)))) +
         (ia ? ((Ds * cf.Aco) / (3.0 * Tm)) * anudot : 0.0)) +
        (ig ? ((5.0 / 6.0) * (Ds / Tm)) *
                  (((nux * gTx) + (nuy * gTy)) - ((((nux * ux) + (nuy * uy)) * ((gTx * ux) + (gTy * uy))) / (ut * ut)))
            : 0.0)) +
       ((t & FIVO_TERM_M2_BG_DALPHA) ? cf.etabar * Da : 0.0));
  const double den = tM * ut;
  out[0] = (-sxx) / den; out[1] = (-sxy) / den; out[2] = (-syy) / den; out[3] = (-sB) / den; out[4] = geo;
}

/* the second moment's pieces with plain arguments, for the gate tests */
void m2_source(const double* in44, uint32_t terms, double* out5) { consistent_m2_source(in44, terms, out5); }
void m2_coeffs(double T, double n, double tn, double Ds, double h, double m, double* out5) {
  M2Coeffs c = hq_m2_coeffs(T, n, tn, Ds, h, m);
  out5[0] = c.dlnC; out5[1] = c.etabar; out5[2] = c.lama; out5[3] = c.Aco; out5[4] = c.ABr;
}
double m2_tauM(double T, double tn, double m) { return tauM_charm(T, tn, m); }
void m2_sigma_nu(const double* a, double* out4) {
  sigma_nu(a[0], a[1], a[2], a[3], a[4], a[5], a[6], a[7], a[8], a[9], a[10], a[11], a[12], a[13], a[14], a[15],
           a[16], a[17], &out4[0], &out4[1], &out4[2], &out4[3]);
}
void m2_rank1_traceless(const double* a, double* out3) {
  rank1_traceless(a[0], a[1], a[2], a[3], a[4], a[5], a[6], &out3[0], &out3[1], &out3[2]);
}

/* relax_dissipative_2d! and the per-cell sector updates, src2d/dissipation2d.jl:293-705 */
int64_t relax_dissipative_2d(double* U, const Grid& g, double tau, double D, const Model& m, Work& w) {
  const Layout& L = m.L;
  const fivo_params& p = m.p;
  if (!(p.enable_shear || p.enable_bulk || p.enable_diff)) return 0;
  const int nv = L.nv, ng = g.ng;
  std::memcpy(w.diss_snap.data(), U, sizeof(double) * nv * g.Ntot);
  const double* Q = w.diss_snap.data();
  if (p.enable_diff) compute_alpha_grad(w, g);
  const double invdx = 1.0 / g.dx, invdy = 1.0 / g.dy;
  auto upw = [&](int a, int64_t i, double ux, double uy) {
    double dqx = ux >= 0 ? (Q[i * nv + a] - Q[(i - g.Nytot) * nv + a]) * invdx
                         : (Q[(i + g.Nytot) * nv + a] - Q[i * nv + a]) * invdx;
    double dqy = uy >= 0 ? (Q[i * nv + a] - Q[(i - 1) * nv + a]) * invdy
                         : (Q[(i + 1) * nv + a] - Q[i * nv + a]) * invdy;
    return (ux * dqx) + (uy * dqy);
  };
#pragma omp parallel for schedule(dynamic, 1)
  for (int ix = ng; ix < ng + g.Nx; ++ix)
    for (int iy = ng; iy < ng + g.Ny; ++iy) {
      int64_t i = g.lin(ix, iy);
      if (!w.ok[i]) continue;
      double* u = U + i * nv;
      double ux = w.ux[i], uy = w.uy[i];
      double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
      Kin k = kinematics(w, g, i, D, tau);
      double T = o_exp(w.yT[i]), mu = w.mu[i], n = w.n[i], en = w.e[i], P = w.P[i];
      /* ---- bulk: relax_bulk_cell_2d!, :377-416 ---- */
      if (p.enable_bulk && L.hasPi) {
        double Pin = u[L.iPi];
        double zeta, tPi;
        bulk_coeffs(T, mu, n, en, P, p, &zeta, &tPi);
        double PiNS = (-zeta) * k.th;
        double A = safe_div(tPi * ut, D);
        double adv = p.relax_advect_Pi ? (-tPi) * upw(L.iPi, i, ux, uy) : 0.0;
        double dPi = p.deltaPi_factor * tPi;
        if (p.lambda_Pi_pi_factor != 0.0 && p.enable_shear && L.hasShear) {
          double sxx, sxy, syy, se, ps, c1, c2, c3;
          ns_shear_target(ux, uy, ut, tau, k, -0.5, &sxx, &sxy, &syy, &se);
          pi_sigma(ux, uy, u[L.iPixx], u[L.iPixy], u[L.iPiyy], u[L.iPieta], sxx, sxy, syy, se, &ps, &c1, &c2, &c3);
          adv = adv - ((p.lambda_Pi_pi_factor * tPi) * ps);
        }
        double num = ((A * Pin) + PiNS) + adv;
        Pin = dPi == 0.0 ? num / (A + 1.0) : num / o_max((A + 1.0) + (dPi * k.th), 0.5 * (A + 1.0));
        Pin = o_max(Pin, -0.99 * o_max(P, 0.0));
        if (p.Pi_clip_factor > 0) { double cap = p.Pi_clip_factor * std::fabs(P); Pin = o_clamp(Pin, -cap, cap); }
        u[L.iPi] = Pin;
      }
      /* ---- shear: relax_shear_cell_2d!, :432-534 ---- */
      if (p.enable_shear && L.hasShear) {
        double eta, tpi, dpi;
        shear_coeffs(T, mu, n, en, P, p, &eta, &tpi, &dpi);
        double pixx = u[L.iPixx], pixy = u[L.iPixy], piyy = u[L.iPiyy], pieta = u[L.iPieta];
        double nsxx, nsxy, nsyy, nse;
        ns_shear_target(ux, uy, ut, tau, k, eta, &nsxx, &nsxy, &nsyy, &nse);
        PiC Pc = shear_tensor(ux, uy, ut, tau, pixx, pixy, piyy, pieta);
        double cx = (((-Pc.tx) * k.at) + (Pc.xx * k.ax)) + (Pc.xy * k.ay);
        double cy = (((-Pc.ty) * k.at) + (Pc.xy * k.ax)) + (Pc.yy * k.ay);
        double A = safe_div(tpi * ut, D);
        double den = o_max((A + 1.0) + (dpi * k.th), 0.5 * (A + 1.0));
        double pd = p.shear_projected_deriv ? tpi : 0.0;
        bool ra = p.relax_advect_pi != 0;
        double axx = ra ? (-tpi) * upw(L.iPixx, i, ux, uy) : 0.0;
        double axy = ra ? (-tpi) * upw(L.iPixy, i, ux, uy) : 0.0;
        double ayy = ra ? (-tpi) * upw(L.iPiyy, i, ux, uy) : 0.0;
        if (p.terms & FIVO_TERM_SHEAR_VORTICITY) {
          double iu = safe_inv(ut);
          double dtux = ((k.ax - (ux * k.dxux)) - (uy * k.dyux)) * iu;
          double dtuy = ((k.ay - (ux * k.dxuy)) - (uy * k.dyuy)) * iu;
          double wxx, wxy, wyy;
          vorticity_coupling(ux, uy, ut, tau, pixx, pixy, piyy, pieta, k.ax, k.ay, dtux, dtuy,
                             k.dxux, k.dxuy, k.dyux, k.dyuy, &wxx, &wxy, &wyy);
          axx -= tpi * wxx; axy -= tpi * wxy; ayy -= tpi * wyy;
        }
        if (p.taupi_pi_factor != 0.0 || p.lambda_pi_Pi_factor != 0.0) {
          double sxx, sxy, syy, se;
          ns_shear_target(ux, uy, ut, tau, k, -0.5, &sxx, &sxy, &syy, &se);
          if (p.taupi_pi_factor != 0.0) {
            double tpp = p.taupi_pi_factor * tpi;
            double ps, cxx, cxy, cyy;
            pi_sigma(ux, uy, pixx, pixy, piyy, pieta, sxx, sxy, syy, se, &ps, &cxx, &cxy, &cyy);
            axx -= tpp * (cxx - (((1.0 + (ux * ux)) * ps) / 3.0));
            axy -= tpp * (cxy - (((ux * uy) * ps) / 3.0));
            ayy -= tpp * (cyy - (((1.0 + (uy * uy)) * ps) / 3.0));
          }
          if (p.lambda_pi_Pi_factor != 0.0 && p.enable_bulk && L.hasPi) {
            double lP = (p.lambda_pi_Pi_factor * tpi) * u[L.iPi];
            axx -= lP * sxx; axy -= lP * sxy; ayy -= lP * syy;
          }
        }
        pixx = ((((A * pixx) + nsxx) + (pd * ((2.0 * ux) * cx))) + axx) / den;
        pixy = ((((A * pixy) + nsxy) + (pd * ((ux * cy) + (uy * cx)))) + axy) / den;
        piyy = ((((A * piyy) + nsyy) + (pd * ((2.0 * uy) * cy))) + ayy) / den;
        if (p.pi_clip_factor > 0) {
          double cap = p.pi_clip_factor * std::fabs(P);
          pixx = o_clamp(pixx, -cap, cap); pixy = o_clamp(pixy, -cap, cap); piyy = o_clamp(piyy, -cap, cap);
        }
        double pe = project_traceless(ux, uy, ut, pixx, pixy, piyy);
        u[L.iPixx] = pixx; u[L.iPixy] = pixy; u[L.iPiyy] = piyy; u[L.iPieta] = pe;
      }
      /* ---- charge: relax_charge_cell_2d!, :552-705 ---- */
      if (p.enable_diff && L.hasNu) {
        double wv = vacuum_weight(n, p);
        if (wv <= 0.0) { u[L.iNux] = 0.0; u[L.iNuy] = 0.0; continue; }
        double kappa, tn, dN;
        diff_coeffs(T, mu, n, p, &kappa, &tn, &dN);
        double nux = u[L.iNux], nuy = u[L.iNuy];
        double dxa = w.gradAx[i], dya = w.gradAy[i];
        double ap = w.alpha_prev[i];
        double dta = o_isfinite(ap) ? (w.alpha[i] - ap) / D : 0.0;
        double nsx = 0.0, nsy = 0.0;
        if (p.terms & FIVO_TERM_NU_GRADALPHA) ns_diffusion_target(ux, uy, ut, dxa, dya, dta, kappa, &nsx, &nsy);
        /* the consistent first moment, src2d/dissipation2d.jl:589-623: subtracted
         * (the source is written on the left-hand side of the row) */
        if (p.consistent_fm) {
          double Tp = w.T_prev[i];
          double dtT = o_isfinite(Tp) ? (T - Tp) / D : 0.0;
          double dxT = (o_exp(w.yT[i + g.Nytot]) - o_exp(w.yT[i - g.Nytot])) / (2.0 * g.dx);
          double dyT = (o_exp(w.yT[i + 1]) - o_exp(w.yT[i - 1])) / (2.0 * g.dy);
          double hh, hp;
          hq_h_hprime(T, p, &hh, &hp);
          double dn_dT = hq_dn_dT(T, n, p);
          double Ds = safe_div(p.kappa_coeff, T) / FMGEV;
          double csx, csy;
          consistent_fm_source(ux, uy, ut, T, dxT, dyT, dtT, nux, nuy, n, dn_dT, tn, Ds, hp, k, p.terms, &csx, &csy);
          nsx -= csx; nsy -= csy;
        }
        nsx *= wv; nsy *= wv;
        if (p.vacuum_ramp_relax) { tn = wv * tn; dN = wv * dN; }
        double nut = nu_tau(ux, uy, ut, nux, nuy);
        double nua = (((-nut) * k.at) + (nux * k.ax)) + (nuy * k.ay);
        double A = safe_div(tn * ut, D);
        double den = o_max((A + 1.0) + (dN * k.th), 0.5 * (A + 1.0));
        double pdn = p.diff_projected_deriv ? tn : 0.0;
        double anx = p.relax_advect_nu ? (-tn) * upw(L.iNux, i, ux, uy) : 0.0;
        double any_ = p.relax_advect_nu ? (-tn) * upw(L.iNuy, i, ux, uy) : 0.0;
        nux = ((((A * nux) + nsx) + ((pdn * ux) * nua)) + anx) / den;
        nuy = ((((A * nuy) + nsy) + ((pdn * uy) * nua)) + any_) / den;
        if (p.nu_clip_factor > 0) {
          double cap = (p.nu_clip_factor * o_max(n, 0.0)) * ut;
          double mag = o_hypot(nux, nuy);
          if (mag > cap && mag > TINY) { double sc = cap / mag; nux *= sc; nuy *= sc; }
        }
        u[L.iNux] = nux; u[L.iNuy] = nuy;
        /* ---- the charm second moment: relax_charm_m2_cell_2d!, :722-888 (given the
         * ramped tau_n and the relaxed current of this cell) ---- */
        if (p.consistent_m2 && L.hasM2) {
          double pQxx = u[L.iPQxx], pQxy = u[L.iPQxy], pQyy = u[L.iPQyy], pQeta = u[L.iPQeta];
          double PiQv = u[L.iPiQ];
          const double mq = p.transport_mass > 0.0 ? p.transport_mass : p.m_hq;
          const double tMq = tauM_charm(T, tn, mq);
          const bool have_hist = o_isfinite(w.alpha_prev[i]) && o_isfinite(w.T_prev[i]);
          if (tMq > 0.0 && have_hist) {
            const double dtnx = o_isfinite(w.nux_prev[i]) ? (nux - w.nux_prev[i]) / D : 0.0;
            const double dtny = o_isfinite(w.nuy_prev[i]) ? (nuy - w.nuy_prev[i]) / D : 0.0;
            const int64_t ixm = i - g.Nytot, ixp = i + g.Nytot;
            const double dxnx = ((Q[ixp * nv + L.iNux] - Q[ixm * nv + L.iNux]) * 0.5) * invdx;
            const double dxny = ((Q[ixp * nv + L.iNuy] - Q[ixm * nv + L.iNuy]) * 0.5) * invdx;
            const double dynx = ((Q[(i + 1) * nv + L.iNux] - Q[(i - 1) * nv + L.iNux]) * 0.5) * invdy;
            const double dyny = ((Q[(i + 1) * nv + L.iNuy] - Q[(i - 1) * nv + L.iNuy]) * 0.5) * invdy;
            const double dtux2 = o_isfinite(w.ux_prev[i]) ? (ux - w.ux_prev[i]) / D : 0.0;
            const double dtuy2 = o_isfinite(w.uy_prev[i]) ? (uy - w.uy_prev[i]) / D : 0.0;
            const double anx = ((ut * dtnx) + (ux * dxnx)) + (uy * dynx);
            const double any2 = ((ut * dtny) + (ux * dxny)) + (uy * dyny);
            const double nut2 = nu_tau(ux, uy, ut, nux, nuy);
            const double thnu = ((((((((ux * dtnx) + (uy * dtny)) + (nux * dtux2)) + (nuy * dtuy2)) * safe_inv(ut)) -
                                   ((nut2 * ((ux * dtux2) + (uy * dtuy2))) * safe_inv(ut * ut))) + dxnx) + dyny) +
                                (nut2 * safe_inv(tau));
            const double Tp2 = w.T_prev[i];
            const double dtT2 = o_isfinite(Tp2) ? (T - Tp2) / D : 0.0;
            const double dxT2 = ((o_exp(w.yT[ixp]) - o_exp(w.yT[ixm])) * 0.5) * invdx;
            const double dyT2 = ((o_exp(w.yT[i + 1]) - o_exp(w.yT[i - 1])) * 0.5) * invdy;
            double h2, hp2;
            hq_h_hprime(T, p, &h2, &hp2);
            const double Ds2 = safe_div(p.kappa_coeff, T) / FMGEV;
            double a[M2_NARG] = {ux, uy, ut, tau, T, dxT2, dyT2, dtT2, nux, nuy, pQxx, pQxy, pQyy, pQeta, PiQv,
                                 dta, dxa, dya, thnu, anx, any2, dtnx, dtny, dxnx, dxny, dynx, dyny,
                                 k.th, k.ax, k.ay, dtux2, dtuy2, k.dxux, k.dxuy, k.dyux, k.dyuy,
                                 n, tn, Ds2, h2, hp2, tMq, etaM_charm(T, tn), mq};
            double s0[5], s1[5];
            consistent_m2_source(a, p.terms, s0);
            const double A2 = safe_div(tMq * ut, D);
            const double dp = 1e-7 * o_max(o_max(o_max(o_max(1.0, std::fabs(pQxx)), std::fabs(pQxy)), std::fabs(pQyy)),
                                           std::fabs(PiQv));
            /* one perturbed evaluation per channel: the slope of each row in its own field */
            double c[4];
            const int slot[4] = {M2_PXX, M2_PXY, M2_PYY, M2_PIQ};
            for (int j = 0; j < 4; ++j) {
              const double keep = a[slot[j]];
              a[slot[j]] = keep + dp;
              consistent_m2_source(a, p.terms, s1);
              a[slot[j]] = keep;
              c[j] = (((-(s1[j] - s0[j])) / dp) * tMq) * ut;
            }
            auto dn = [&](double cc) { return o_max(A2 + cc, 0.5 * (A2 + 1.0)); };
            const bool ram = p.relax_advect_m2 != 0;
            const double amxx = ram ? (-tMq) * upw(L.iPQxx, i, ux, uy) : 0.0;
            const double amxy = ram ? (-tMq) * upw(L.iPQxy, i, ux, uy) : 0.0;
            const double amyy = ram ? (-tMq) * upw(L.iPQyy, i, ux, uy) : 0.0;
            const double amB = ram ? (-tMq) * upw(L.iPiQ, i, ux, uy) : 0.0;
            const double Rxx = ((((-tMq) * ut) * s0[0]) - (c[0] * pQxx)) - amxx;
            const double Rxy = ((((-tMq) * ut) * s0[1]) - (c[1] * pQxy)) - amxy;
            const double Ryy = ((((-tMq) * ut) * s0[2]) - (c[2] * pQyy)) - amyy;
            const double RB = ((((-tMq) * ut) * s0[3]) - (c[3] * PiQv)) - amB;
            pQxx = ((A2 * pQxx) - Rxx) / dn(c[0]);
            pQxy = ((A2 * pQxy) - Rxy) / dn(c[1]);
            pQyy = ((A2 * pQyy) - Ryy) / dn(c[2]);
            PiQv = ((A2 * PiQv) - RB) / dn(c[3]);
            pQeta = project_traceless(ux, uy, ut, pQxx, pQxy, pQyy);
            u[L.iPQxx] = pQxx; u[L.iPQxy] = pQxy; u[L.iPQyy] = pQyy; u[L.iPQeta] = pQeta; u[L.iPiQ] = PiQv;
          }
        }
      }
    }
  w.ux_prev = w.ux;
  w.uy_prev = w.uy;
  /* the current's history for the second moment's d_tau nu, :354-359 */
  if (p.consistent_m2 && L.hasNu)
    for (int64_t j = 0; j < g.Ntot; ++j) { w.nux_prev[j] = U[j * nv + L.iNux]; w.nuy_prev[j] = U[j * nv + L.iNuy]; }
  return (int64_t)g.Nx * g.Ny;
}

/* project_shear!, main2D.jl:332-358 */
void project_shear(double* U, const Grid& g, const Work& w, const Model& m, double* maxr, double* meanr) {
  const Layout& L = m.L;
  *maxr = 0.0; *meanr = 0.0;
  if (!L.hasShear) return;
  bool correct = m.p.shear_constraint_project != 0;
  double mx = 0.0, sum = 0.0; int64_t cnt = 0;
  for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
    for (int iy = g.ng; iy < g.ng + g.Ny; ++iy) {
      int64_t i = g.lin(ix, iy);
      double ux = w.ux[i], uy = w.uy[i];
      double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
      double* u = U + i * L.nv;
      double R, rel;
      shear_residual(ux, uy, ut, u[L.iPixx], u[L.iPixy], u[L.iPiyy], u[L.iPieta], &R, &rel);
      mx = o_max(mx, rel); sum += rel; cnt += 1;
      if (correct) u[L.iPieta] = project_traceless(ux, uy, ut, u[L.iPixx], u[L.iPixy], u[L.iPiyy]);
    }
  *maxr = mx; *meanr = cnt > 0 ? sum / cnt : 0.0;
}

/* finalize_ic!, main2D.jl:164-171 */
void finalize_ic(double* U, const Grid& g, const Model& m, int bc, double Emin, double tau0) {
  enforce_floors(U, g, m, Emin);
  enforce_S_energy(U, g, m, CHI_SRE, nullptr);
  enforce_nu_charge(U, g, m, tau0, 0.999);
  apply_bc_2d(U, g, m.L, bc);
}

/* run_sim_2d!'s while loop (main2D.jl:436-513), from tau; nsteps_run is the
 * count of accepted steps since the run began (run_sim_2d!'s local nsteps) */
void advance_sim_2d(double* U, const Grid& g, const Model& m, Work& w, double tau, double taufinal,
                    double CFL, double CFLtau, int integrator, int bc, int64_t max_steps,
                    int64_t* nsteps_run, fivo_run_result* res) {
  const Layout& L = m.L;
  const fivo_params& p = m.p;
  int64_t nsteps = 0, nprimfail = 0, nvacuum = 0;
  double max_shear_res = 0.0;
  bool any_sector = p.enable_shear || p.enable_bulk || p.enable_diff;
  res->ok = 1;
  while (tau < taufinal && nsteps < max_steps) {
    double D = compute_dt_2d(w, g, tau, CFL, CFLtau);
    D = o_min(D, taufinal - tau);
    if (D <= 0) break;
    if (o_isfinite(w.alpha_prev[0]) || *nsteps_run > 0) {
      w.alpha_prev = w.alpha;
      for (int64_t j = 0; j < g.Ntot; ++j) w.T_prev[j] = o_exp(w.yT[j]);
    }
    double used = 0.0;
    bool ok = integrator == FIVO_SSPRK3
                  ? step_ssprk3_2d(U, g, tau, D, m, w, bc, 12, &used)
                  : step_ssprk2_2d(U, g, tau, D, m, w, bc, 12, 2, &used);
    if (!ok) { res->ok = 0; break; }
    tau += used;
    nsteps += 1;
    *nsteps_run += 1;
    if (any_sector) {
      update_primitives_2d(U, g, tau, m, w, bc);
      relax_dissipative_2d(U, g, tau, used, m, w);
    }
    nprimfail += w.nprimfail;
    nvacuum += w.nvacuum;
    if (L.hasShear) {
      double r, mr;
      project_shear(U, g, w, m, &r, &mr);
      max_shear_res = o_max(max_shear_res, r);
    }
  }
  res->tau = tau; res->nsteps = nsteps; res->nprimfail = nprimfail; res->nvacuum = nvacuum;
  res->max_shear_res = max_shear_res;
}

/* run_sim_2d!, main2D.jl:371-561 (no dumps) */
void run_sim_2d(double* U, const Grid& g, const Model& m, Work& w, double tau0, double taufinal,
                double CFL, double CFLtau, int integrator, int bc, bool reset_history,
                int64_t max_steps, fivo_run_result* res) {
  const Layout& L = m.L;
  if (reset_history) {
    std::fill(w.x0_yT.begin(), w.x0_yT.end(), O_NAN); std::fill(w.x0_phi.begin(), w.x0_phi.end(), O_NAN);
    std::fill(w.x0_ux.begin(), w.x0_ux.end(), O_NAN); std::fill(w.x0_uy.begin(), w.x0_uy.end(), O_NAN);
    std::fill(w.ux_prev.begin(), w.ux_prev.end(), O_NAN); std::fill(w.uy_prev.begin(), w.uy_prev.end(), O_NAN);
    std::fill(w.alpha_prev.begin(), w.alpha_prev.end(), O_NAN); std::fill(w.T_prev.begin(), w.T_prev.end(), O_NAN);
    std::fill(w.nux_prev.begin(), w.nux_prev.end(), O_NAN); std::fill(w.nuy_prev.begin(), w.nuy_prev.end(), O_NAN);
  }
  rhs_2d(w.k.data(), U, g, tau0, m, w, bc, E_FLOOR, nullptr);
  double Qin = 0.0;
  for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
    for (int iy = g.ng; iy < g.ng + g.Ny; ++iy) Qin += U[g.lin(ix, iy) * L.nv + L.iDtau];
  int64_t nsteps_run = 0;
  advance_sim_2d(U, g, m, w, tau0, taufinal, CFL, CFLtau, integrator, bc, max_steps, &nsteps_run, res);
  res->Q0 = Qin;
  if (!res->ok) {
    res->maxu = O_NAN; res->dQ = O_NAN; res->Q1 = O_NAN; res->minPtot = O_NAN;
    return;
  }
  double minPtot = O_INF, maxu = 0.0, Qout = 0.0;
  for (int ix = g.ng; ix < g.ng + g.Nx; ++ix)
    for (int iy = g.ng; iy < g.ng + g.Ny; ++iy) {
      int64_t i = g.lin(ix, iy);
      Qout += U[i * L.nv + L.iDtau];
      double uu = o_hypot(w.ux[i], w.uy[i]);
      if (uu > maxu) maxu = uu;
      if (w.P[i] > 0) {
        double pt = w.P[i] + (L.hasPi ? U[i * L.nv + L.iPi] : 0.0);
        if (pt < minPtot) minPtot = pt;
      }
    }
  res->maxu = maxu;
  res->dQ = std::fabs(Qin) > 0 ? std::fabs(Qout - Qin) / std::fabs(Qin) : 0.0;
  res->Q1 = Qout;
  res->minPtot = minPtot;
}

/* ---- cell-level functions for the gate tests (same code the solver runs) ---- */
void cell_shear_coeffs(double T, double mu, double n, double en, double P, const fivo_params& p, double* out3) {
  shear_coeffs(T, mu, n, en, P, p, &out3[0], &out3[1], &out3[2]);
}
void cell_bulk_coeffs(double T, double mu, double n, double en, double P, const fivo_params& p, double* out2) {
  bulk_coeffs(T, mu, n, en, P, p, &out2[0], &out2[1]);
}
void cell_diff_tauN(double T, double alpha, const fivo_params& p, double DsT, double tauD, double* taun,
                    double* norm) {
  *taun = diff_tauN(o_max(T, T_MIN), alpha, p, DsT, tauD);
  *norm = fluidum_norm(T, alpha, p);
}
double cell_vacuum_weight(double n, const fivo_params& p) { return vacuum_weight(n, p); }
double cell_entropy(double T, double mu, double n, double en, double P) { return eos_entropy(T, mu, n, en, P); }
void cell_ns_shear_target(const double* kin12, double* out4) {
  /* kin12 = (ux, uy, ut, tau, theta, ax, ay, dxux, dxuy, dyux, dyuy, eta) */
  Kin k;
  k.th = kin12[4]; k.ax = kin12[5]; k.ay = kin12[6]; k.at = 0.0;
  k.dxux = kin12[7]; k.dxuy = kin12[8]; k.dyux = kin12[9]; k.dyuy = kin12[10];
  ns_shear_target(kin12[0], kin12[1], kin12[2], kin12[3], k, kin12[11], &out4[0], &out4[1], &out4[2], &out4[3]);
}
double cell_project_traceless(double ux, double uy, double ut, double pixx, double pixy, double piyy) {
  return project_traceless(ux, uy, ut, pixx, pixy, piyy);
}
void cell_ns_diffusion_target(double ux, double uy, double ut, double dxa, double dya, double dta, double kappa,
                              double* out2) {
  ns_diffusion_target(ux, uy, ut, dxa, dya, dta, kappa, &out2[0], &out2[1]);
}
void cell_pi_sigma(const double* in10, double* out4) {
  pi_sigma(in10[0], in10[1], in10[2], in10[3], in10[4], in10[5], in10[6], in10[7], in10[8], in10[9],
           &out4[0], &out4[1], &out4[2], &out4[3]);
}
void cell_shear_tensor(double ux, double uy, double ut, double tau, double pixx, double pixy, double piyy,
                       double pieta, double* out7) {
  PiC c = shear_tensor(ux, uy, ut, tau, pixx, pixy, piyy, pieta);
  out7[0] = c.tt; out7[1] = c.tx; out7[2] = c.ty; out7[3] = c.xx; out7[4] = c.xy; out7[5] = c.yy;
  out7[6] = c.etaeta;
}

}  // namespace orc
