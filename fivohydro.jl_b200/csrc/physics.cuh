/*
 * physics.cuh — per-cell physics of the 2+1D stage, as device functions.
 *
 * Each function follows the reference function named in its comment with the
 * same evaluation order (Julia folds n-ary + and * to the left), so results
 * are the bits of the CPU restatement. Where this file is faster than a literal
 * transcription it only shares common subexpressions (the light-sector EOS
 * evaluates P, dP/dT and d2P/dT2 from one exponential) or skips work whose
 * result is multiplied by an exact zero; neither changes a rounding.
 */
#ifndef FIVO_PHYSICS_CUH
#define FIVO_PHYSICS_CUH

#include "fmath.cuh"
#include "../../include/fivo2d.h"

namespace fv {

using namespace fx;

/* src/constants.jl:11-44 */
#define FV_FMGEV (1.0 / 0.1973269804)
#define FV_INVFMGEV 0.1973269804
#define FV_T_MIN 1e-20
#define FV_T_SOLVE_MAX 10.0
#define FV_PHI_CAP 10000.0
#define FV_E_VAC 1e-20
#define FV_D_VAC 0.0
#define FV_E_FLOOR 1e-20
#define FV_CHI_SRE 0.99999999
#define FV_TINY 1e-300
#define FV_EPS_POS 1e-50
#define FV_U_CAP 1.0e4
#define FV_SR_MARGIN 0.98

enum : uint8_t {
  PRR_UNSET = 0, PRR_VACUUM = 1, PRR_CONVERGED = 2, PRR_NONFINITE_INITIAL = 3,
  PRR_NONFINITE_JACOBIAN = 4, PRR_LINSOLVE_FAILED = 5, PRR_LINESEARCH_FAILED = 6,
  PRR_EOS_INVALID = 7, PRR_RESIDUAL_TOO_LARGE = 8, PRR_MAXIT = 9
};

/* Everything a kernel needs about the model and the grid, passed by value. */
struct DevParams {
  fivo_params p;
  int nv, iDtau, iSx, iSy, iE, iNux, iNuy, iPi, iPixx, iPixy, iPiyy, iPieta;
  int hasNu, hasPi, hasShear, ncharge;
  /* nv counts every state row; the first nvf take part in the fluxes, floors and
   * admissibility, the charm second moment's five rows (hasM2) come after them */
  int nvf, hasM2, iPQxx, iPQxy, iPQyy, iPQeta, iPiQ;
  int Nx, Ny, ng, Nxtot, Nytot;
  long long Ntot;
  double dx, dy, xmin, ymin;
  double E_vac_cut;
  double fmgev3, pi2;
  double log_T_min, log_T_solve_max, log_seed_T;
  double aSB, A_conf, A_lhrg, lA, lB;
};

FX_HD double posden(double x) { return x > FV_EPS_POS ? x : FV_EPS_POS; }
FX_HD double safe_inv(double x) { return 1.0 / posden(x); }
FX_HD double safe_div(double a, double b) { return a / posden(b); }
FX_HD double safe_sqrt(double x) { return x <= 0 ? 0.0 : sqrt_(x); }

/* ================================ EOS ================================ */

#define LK0 0.0005624486560000001
#define LK1 0.003652264
#define LK2 0.023716
#define LK3 0.154
#define LK4 5.208957878352717

/* light_P / light_dP_dT / light_d2P_dT2 (src/eos.jl:357-463) from one exp.
 * want: 1 = P, 2 = dP, 4 = d2P (bitmask). T is already max(T, T_MIN). */
template <int WANT>
FX_HD void light_eos(double T, const DevParams& d, double* P, double* dP, double* d2P) {
  const fivo_params& e = d.p;
  double A = d.lA, B = d.lB;
  double T2 = T * T, T3 = (T * T) * T, T4 = fx_pow4(T);
  double E = (-(A / T2)) - (B / T);
  E = jclamp(E, -700.0, 700.0);
  double expE = fx_exp(E);
  double N = ((((LK0 * e.lhrg_a[3]) + ((LK1 * e.lhrg_a[2]) * T)) + ((LK2 * e.lhrg_a[1]) * T2)) +
              ((LK3 * e.lhrg_a[0]) * T3)) + (LK4 * T4);
  double D = ((((LK0 * e.lhrg_b[3]) + ((LK1 * e.lhrg_b[2]) * T)) + ((LK2 * e.lhrg_b[1]) * T2)) +
              ((LK3 * e.lhrg_b[0]) * T3)) + T4;
  double C = d.fmgev3 * expE;
  if (WANT & 1) *P = (C * T4) * (N / D);
  if (WANT & 6) {
    double Ep = ((2.0 * A) / T3) + (B / T2);
    double Np = (((LK1 * e.lhrg_a[2]) + (((2.0 * LK2) * e.lhrg_a[1]) * T)) +
                 (((3.0 * LK3) * e.lhrg_a[0]) * T2)) + ((4.0 * LK4) * T3);
    double Dp = (((LK1 * e.lhrg_b[2]) + (((2.0 * LK2) * e.lhrg_b[1]) * T)) +
                 (((3.0 * LK3) * e.lhrg_b[0]) * T2)) + (4.0 * T3);
    double G = T4 * N, H = D;
    double Gp = ((4.0 * T3) * N) + (T4 * Np);
    double Hp = Dp;
    double F = G / H;
    double Fp = ((Gp * H) - (G * Hp)) / (H * H);
    if (WANT & 2) *dP = C * (Fp + (F * Ep));
    if (WANT & 4) {
      double Epp = ((-6.0 * A) / T4) - ((2.0 * B) / T3);
      double Npp = (((2.0 * LK2) * e.lhrg_a[1]) + (((6.0 * LK3) * e.lhrg_a[0]) * T)) + ((12.0 * LK4) * T2);
      double Dpp = (((2.0 * LK2) * e.lhrg_b[1]) + (((6.0 * LK3) * e.lhrg_b[0]) * T)) + (12.0 * T2);
      double Gpp = (((12.0 * T2) * N) + ((8.0 * T3) * Np)) + (T4 * Npp);
      double Hpp = Dpp;
      double Q = (Gp * H) - (G * Hp);
      double Qp = (Gpp * H) - (G * Hpp);
      double Fpp = ((Qp * H) - ((2.0 * Q) * Hp)) / ((H * H) * H);
      *d2P = C * ((Fpp + ((2.0 * Fp) * Ep)) + (F * (Epp + (Ep * Ep))));
    }
  }
}

/* _lhrg_assemble_2d, src2d/primrec2d.jl:134-154 */
FX_HD void lhrg_assemble(double T, double mu, const DevParams& d, double x, double Pl, double el,
                         double K2x, double* P, double* n, double* en) {
  /* computed unconditionally and selected, so it has no branch */
  const bool off = !isfinite_(x) || x <= 0.0;
  double m = d.p.m_hq;
  double z = (mu - m) / T;
  z = jclamp(z, -700.0, 700.0);
  double Efac = fx_exp(z);
  double n_hq = ((d.A_lhrg * T) * Efac) * K2x;
  double P_hq = 0.0, e_hq = 0.0;
  if (d.p.hq_times_fmGeV3) { n_hq *= d.fmgev3; P_hq *= d.fmgev3; e_hq *= d.fmgev3; }
  *P = off ? Pl : Pl + P_hq;
  *n = off ? 0.0 : n_hq;
  *en = off ? el : el + e_hq;
}

FX_HD double lhrg_x(double T, const DevParams& d) { return jmin(d.p.m_hq / T, 100000.0); }
/* e^x K2(x) as the LatticeHRG charm density uses it (0 off the domain). The
 * usual range 2 <= x < 1e4 (0.15 < T < 750 MeV) is straight-line code on a
 * clamped argument, so it interleaves with the light-sector EOS; the rest of
 * the domain goes through the general function. Same bits either way. */
FX_HD double lhrg_K2(double x) {
  const bool common = x >= 2.0 && x < 1.0e4;
  const double xc = common ? x : 2.0;
  double k0, k1;
  fx_k01x_B(xc, &k0, &k1);
  double v = k0 + (2.0 / xc) * k1;
  if (!common) v = (!isfinite_(x) || x <= 0.0) ? 0.0 : fx_besselk2x(x);
  return v;
}

/* ConformalHQEOS eos_Pne, src/eos.jl:53-84. A == 0 (g_hq = 0) skips the Bessel
 * functions: the HQ terms are then 0 * (finite) or NaN when exp overflows. */
FX_HD void conformal_Pne(double T, double mu, const DevParams& d, double* P, double* n, double* en) {
  T = jmax(T, FV_T_MIN);
  double Plight = (d.aSB * fx_pow4(T)) * d.fmgev3;
  double elight = 3.0 * Plight;
  double m = d.p.m_hq;
  double x = m / T;
  if (!isfinite_(x) || x <= 0.0) { *P = Plight; *n = 0.0; *en = elight; return; }
  double A = d.A_conf;
  double exp_arg = (mu - m) / T;
  double Efac = fx_exp(exp_arg);
  double n_hq, P_hq, e_hq;
  if (A == 0.0) {
    double z = isinf_(Efac) ? nan_() : 0.0;
    n_hq = z; P_hq = z; e_hq = z;
  } else {
    double k0, k1, K2x, K1x;
    if (x >= 1.0e4) { K2x = fx_besselkx_asym(2, x); K1x = fx_besselkx_asym(1, x); }
    else { fx_k01x(x, &k0, &k1); K1x = k1; K2x = k0 + (2.0 / x) * k1; }
    n_hq = ((A * T) * Efac) * K2x;
    P_hq = ((A * (T * T)) * Efac) * K2x;
    e_hq = ((A * (T * T)) * Efac) * ((3.0 * K2x) + (x * K1x));
  }
  if (d.p.hq_times_fmGeV3) { n_hq *= d.fmgev3; P_hq *= d.fmgev3; e_hq *= d.fmgev3; }
  *P = Plight + P_hq; *n = n_hq; *en = elight + e_hq;
}

/* eos_Pne (src/eos.jl) == eos_Pne_2d without memo (src2d/primrec2d.jl:170-176) */
template <int EOS>
FX_HD void eos_Pne(double T, double mu, const DevParams& d, double* P, double* n, double* en) {
  if (EOS == FIVO_EOS_CONFORMAL_HQ) { conformal_Pne(T, mu, d, P, n, en); return; }
  T = jmax(T, FV_T_MIN);
  double Pl, dP;
  light_eos<3>(T, d, &Pl, &dP, nullptr);
  double el = (-Pl) + (T * dP);
  double x = lhrg_x(T, d);
  lhrg_assemble(T, mu, d, x, Pl, el, lhrg_K2(x), P, n, en);
}

/* eos_cs2, src/eos.jl:51, 473-478 */
template <int EOS>
FX_HD double eos_cs2(double T, const DevParams& d) {
  if (EOS == FIVO_EOS_CONFORMAL_HQ) return 1.0 / 3.0;
  T = jmax(T, FV_T_MIN);
  double Pp, Ppp;
  light_eos<6>(T, d, nullptr, &Pp, &Ppp);
  return (Ppp == 0.0) ? (1.0 / 3.0) : (Pp / (T * Ppp));
}

/* eos_Pne plus cs2 at the same T (faces: prim_to_cons and wavespeeds) */
template <int EOS>
FX_HD void eos_Pne_cs2(double T, double mu, const DevParams& d, double* P, double* n, double* en,
                       double* cs2) {
  if (EOS == FIVO_EOS_CONFORMAL_HQ) { conformal_Pne(T, mu, d, P, n, en); *cs2 = 1.0 / 3.0; return; }
  T = jmax(T, FV_T_MIN);
  double Pl, dP, d2P;
  light_eos<7>(T, d, &Pl, &dP, &d2P);
  double el = (-Pl) + (T * dP);
  double x = lhrg_x(T, d);
  lhrg_assemble(T, mu, d, x, Pl, el, lhrg_K2(x), P, n, en);
  *cs2 = (d2P == 0.0) ? (1.0 / 3.0) : (dP / (T * d2P));
}

/* eos_Pe_2d, src2d/primrec2d.jl:209-231 */
template <int EOS>
FX_HD void eos_Pe_2d(double T, double mu, const DevParams& d, double* P, double* en) {
  if (EOS != FIVO_EOS_LATTICE_HRG) { double n; eos_Pne<EOS>(T, mu, d, P, &n, en); return; }
  T = jmax(T, FV_T_MIN);
  double Pl, dP;
  light_eos<3>(T, d, &Pl, &dP, nullptr);
  double el = (-Pl) + (T * dP);
  double x = d.p.m_hq / T;
  x = jmin(x, 100000.0);
  if (!isfinite_(x) || x <= 0.0) { *P = Pl; *en = el; return; }
  double P_hq = 0.0, e_hq = 0.0;
  if (d.p.hq_times_fmGeV3) { P_hq *= d.fmgev3; e_hq *= d.fmgev3; }
  *P = Pl + P_hq; *en = el + e_hq;
}

/* EOSCache2D (src2d/primrec2d.jl:115-197): a T-keyed memo of the T-only part of
 * the LatticeHRG EOS inside one Newton solve. A hit returns the same bits as a
 * fresh evaluation, so the memo only changes the cost. Four slots, round robin. */
struct EosMemo {
  double T[4], Pl[4], el[4], K2[4];
  int next;
  FX_HD void reset() { T[0] = T[1] = T[2] = T[3] = nan_(); next = 0; }
};

template <int EOS>
FX_HD void eos_Pne_memo(double T, double mu, const DevParams& d, EosMemo& c, double* P, double* n,
                        double* en) {
  if (EOS != FIVO_EOS_LATTICE_HRG) { eos_Pne<EOS>(T, mu, d, P, n, en); return; }
  T = jmax(T, FV_T_MIN);
  double x = lhrg_x(T, d);
  double Pl, el, K2;
  if (c.T[0] == T) { Pl = c.Pl[0]; el = c.el[0]; K2 = c.K2[0]; }
  else if (c.T[1] == T) { Pl = c.Pl[1]; el = c.el[1]; K2 = c.K2[1]; }
  else if (c.T[2] == T) { Pl = c.Pl[2]; el = c.el[2]; K2 = c.K2[2]; }
  else if (c.T[3] == T) { Pl = c.Pl[3]; el = c.el[3]; K2 = c.K2[3]; }
  else {
    double dP;
    light_eos<3>(T, d, &Pl, &dP, nullptr);
    el = (-Pl) + (T * dP);
    K2 = lhrg_K2(x);
    int k = c.next;
    c.next = (k == 3) ? 0 : k + 1;
    /* unrolled store keeps the memo in registers */
    if (k == 0) { c.T[0] = T; c.Pl[0] = Pl; c.el[0] = el; c.K2[0] = K2; }
    else if (k == 1) { c.T[1] = T; c.Pl[1] = Pl; c.el[1] = el; c.K2[1] = K2; }
    else if (k == 2) { c.T[2] = T; c.Pl[2] = Pl; c.el[2] = el; c.K2[2] = K2; }
    else { c.T[3] = T; c.Pl[3] = Pl; c.el[3] = el; c.K2[3] = K2; }
  }
  lhrg_assemble(T, mu, d, x, Pl, el, K2, P, n, en);
}

/* eos_entropy, src/eos.jl:306-310 */
FX_HD double eos_entropy(double T, double mu, double n, double e, double P) {
  T = jmax(T, FV_T_MIN);
  double s = ((e + P) - (mu * n)) / T;
  return jmax(s, 0.0);
}

/* ============================ shear algebra (src2d/shear2d.jl) ============================ */

struct PiC { double tt, tx, ty, xx, xy, yy; };

FX_HD PiC shear_tensor(double ux, double uy, double ut, double pixx, double pixy, double piyy) {
  double iu = safe_inv(ut);
  double tx = ((ux * pixx) + (uy * pixy)) * iu;
  double ty = ((ux * pixy) + (uy * piyy)) * iu;
  double tt = ((ux * tx) + (uy * ty)) * iu;
  PiC r; r.tt = tt; r.tx = tx; r.ty = ty; r.xx = pixx; r.xy = pixy; r.yy = piyy;
  return r;
}

/* shear_constraint_residual_2d, src2d/shear2d.jl:88-101 (relative residual) */
FX_HD double shear_residual_rel(double ux, double uy, double ut, double pixx, double pixy,
                                double piyy, double pieta) {
  PiC c = shear_tensor(ux, uy, ut, pixx, pixy, piyy);
  double r = (((-c.tt) + pixx) + piyy) + pieta;
  double scale = jmax(jmax(jmax(jmax(fabs_(c.tt), fabs_(pixx)), fabs_(piyy)), fabs_(pieta)), fabs_(pixy));
  return scale > FV_TINY ? fabs_(r) / scale : 0.0;
}

/* project_shear_traceless_2d, src2d/shear2d.jl:131-142 */
FX_HD double project_traceless(double ux, double uy, double ut, double pixx, double pixy, double piyy) {
  PiC c = shear_tensor(ux, uy, ut, pixx, pixy, piyy);
  return (c.tt - pixx) - piyy;
}

FX_HD double nu_tau(double ux, double uy, double ut, double nux, double nuy) {
  return ((ux * nux) + (uy * nuy)) * safe_inv(ut);
}

FX_HD double utau(double ux, double uy) { return sqrt_((1.0 + (ux * ux)) + (uy * uy)); }

/* ======================= primitive recovery (src2d/primrec2d.jl) ======================= */

struct CellCons { double D, Sx, Sy, E, nux, nuy, Pi, pixx, pixy, piyy, pieta; };

struct Recovery {
  double T, mu, ux, uy, n, e, P, resnorm;
  uint8_t ok, reason;
};

/* the residual rows of evalF_2d! from the EOS values (src2d/primrec2d.jl:375-389);
 * a non-finite EOS value makes every row inf (selected, not branched) */
template <bool NCH>
FX_HD void evalF_rows(double F[4], double P, double n, double en, double ux, double uy, double ut,
                      const CellCons& c) {
  const bool bad = !(isfinite_(P) && isfinite_(n) && isfinite_(en));
  double weff = (en + P) + c.Pi;
  double Ptot = P + c.Pi;
  PiC pc = shear_tensor(ux, uy, ut, c.pixx, c.pixy, c.piyy);
  const double f0 = NCH ? (((n * ut) + nu_tau(ux, uy, ut, c.nux, c.nuy)) - c.D) : 0.0;
  const double f1 = (((weff * ut) * ux) + pc.tx) - c.Sx;
  const double f2 = (((weff * ut) * uy) + pc.ty) - c.Sy;
  const double f3 = ((((weff * ut) * ut) - Ptot) + pc.tt) - c.E;
  F[0] = bad ? inf_() : f0;
  F[1] = bad ? inf_() : f1;
  F[2] = bad ? inf_() : f2;
  F[3] = bad ? inf_() : f3;
}

/* evalF_2d!, src2d/primrec2d.jl:360-390 */
template <int EOS, bool NCH>
FX_HD void evalF(double F[4], const double x[4], const CellCons& c, const DevParams& d, EosMemo& memo) {
  double yT = x[0], phi = x[1], ux = x[2], uy = x[3];
  if (!(isfinite_(yT) && isfinite_(phi) && isfinite_(ux) && isfinite_(uy))) {
    F[0] = F[1] = F[2] = F[3] = inf_(); return;
  }
  double T = fx_exp(yT);
  double mu = d.p.m_hq + (T * phi);
  double ut = utau(ux, uy);
  double P, n, en;
  eos_Pne_memo<EOS>(T, mu, d, memo, &P, &n, &en);
  evalF_rows<NCH>(F, P, n, en, ux, uy, ut, c);
}

FX_HD bool finite4(const double F[4]) {
  return isfinite_(F[0]) && isfinite_(F[1]) && isfinite_(F[2]) && isfinite_(F[3]);
}

/* solve_gauss_n!, src2d/primrec2d.jl:33-87, for n = N (3 or 4) */
template <int N>
FX_HD bool solve_gauss(double delta[4], const double J[4][4], const double F[4]) {
  double A[4][5];
#pragma unroll
  for (int r = 0; r < N; ++r) {
#pragma unroll
    for (int c = 0; c < N; ++c) A[r][c] = J[r][c];
    A[r][N] = -F[r];
  }
  double smax = 0.0;
#pragma unroll
  for (int r = 0; r < N; ++r)
#pragma unroll
    for (int c = 0; c < N; ++c) smax = jmax(smax, fabs_(A[r][c]));
  if (!isfinite_(smax) || smax == 0.0) return false;
  double pivtol = 1e-15 * smax;
#pragma unroll
  for (int k = 0; k < N; ++k) {
    int p = k;
    double amax = fabs_(A[k][k]);
#pragma unroll
    for (int r = k + 1; r < N; ++r)
      if (fabs_(A[r][k]) > amax) { amax = fabs_(A[r][k]); p = r; }
    if (amax < pivtol) return false;
    /* row swap with static indexing (keeps A in registers) */
#pragma unroll
    for (int r = k + 1; r < N; ++r) {
      if (p == r) {
#pragma unroll
        for (int c = k; c <= N; ++c) { double t = A[k][c]; A[k][c] = A[r][c]; A[r][c] = t; }
      }
    }
    double invp = 1.0 / A[k][k];
#pragma unroll
    for (int r = k + 1; r < N; ++r) {
      double f = A[r][k] * invp;
      if (f == 0.0) continue;
#pragma unroll
      for (int c = k; c <= N; ++c) A[r][c] -= f * A[k][c];
    }
  }
#pragma unroll
  for (int r = N - 1; r >= 0; --r) {
    double s = A[r][N];
#pragma unroll
    for (int c = r + 1; c < N; ++c) s -= A[r][c] * delta[c];
    delta[r] = s / A[r][r];
  }
#pragma unroll
  for (int r = 0; r < N; ++r) if (!isfinite_(delta[r])) return false;
  return true;
}

/* _invert_e_for_T, src2d/primrec2d.jl:300-314 */
template <int EOS>
FX_HD double invert_e_for_T(double e_target, double phi, const DevParams& d) {
  double lo = d.log_T_min, hi = d.log_T_solve_max;
  if (e_target <= 0.0) return lo;
  for (int it = 0; it < 60; ++it) {
    double mid = 0.5 * (lo + hi);
    double Tm = fx_exp(mid);
    double Pm, em;
    eos_Pe_2d<EOS>(Tm, d.p.m_hq + (Tm * phi), d, &Pm, &em);
    if (!isfinite_(em) || em > e_target) hi = mid; else lo = mid;
  }
  return 0.5 * (lo + hi);
}

/* seed_from_conserved_2d, src2d/primrec2d.jl:323-347 */
template <int EOS>
FX_HD void seed_from_conserved(double E, double Sx, double Sy, double phi, const DevParams& d,
                               double* yT, double* ux, double* uy) {
  double M = sqrt_((Sx * Sx) + (Sy * Sy));
  if (!isfinite_(E) || E <= 0.0) { *yT = d.log_seed_T; *ux = 0.0; *uy = 0.0; return; }
  double P = E / 3.0;
  double y = d.log_seed_T;
  double v = 0.0;
  for (int it = 0; it < 3; ++it) {
    double denom = E + P;
    v = denom > FV_TINY ? jmin(M / denom, 0.999999) : 0.0;
    double ee = (denom * (1.0 - (v * v))) - P;
    if (ee <= 0.0) ee = jmax(E, FV_TINY);
    y = invert_e_for_T<EOS>(ee, phi, d);
    double T = fx_exp(y);
    double Pn, en;
    eos_Pe_2d<EOS>(T, d.p.m_hq + (T * phi), d, &Pn, &en);
    if (!isfinite_(Pn)) break;
    P = Pn;
  }
  double gam = 1.0 / sqrt_(jmax(1.0 - (v * v), 1e-16));
  double us = gam * v;
  double sx = M > FV_TINY ? (us * Sx) / M : 0.0;
  double sy = M > FV_TINY ? (us * Sy) / M : 0.0;
  *yT = y;
  *ux = jclamp(sx, -FV_U_CAP, FV_U_CAP);
  *uy = jclamp(sy, -FV_U_CAP, FV_U_CAP);
}

/* _solve_phi_bisect, src2d/primrec2d.jl:416-434 */
template <int EOS>
FX_HD void solve_phi_bisect(double D, double T, double ux, double uy, double nux, double nuy,
                            const DevParams& d, EosMemo& c, double* phi, bool* ok) {
  double ut = utau(ux, uy);
  double target = D - nu_tau(ux, uy, ut, nux, nuy);
  double m = d.p.m_hq;
  if (!isfinite_(target) || target <= 0.0) { *phi = -FV_PHI_CAP; *ok = false; return; }
  double lo = -FV_PHI_CAP, hi = FV_PHI_CAP;
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    double P, nm, en;
    eos_Pne_memo<EOS>(T, m + (T * mid), d, c, &P, &nm, &en);
    if (isfinite_(nm) && (nm * ut) > target) hi = mid; else lo = mid;
  }
  double f = 0.5 * (lo + hi);
  double P, nf, en;
  eos_Pne_memo<EOS>(T, m + (T * f), d, c, &P, &nf, &en);
  *phi = f; *ok = isfinite_(nf);
}

/* the vacuum test and result of _cons_to_prim_attempt_2d! (src2d/primrec2d.jl:527-534) */
FX_HD bool is_vacuum(const CellCons& c) {
  return !isfinite_(c.E) || c.E <= FV_E_VAC || !isfinite_(c.D) || c.D < FV_D_VAC;
}

template <int EOS>
FX_HD Recovery vacuum_recovery(const CellCons& c, const DevParams& d) {
  Recovery out;
  out.reason = PRR_VACUUM; out.resnorm = 0.0;
  double P, n, en;
  eos_Pne<EOS>(FV_T_MIN, 0.0, d, &P, &n, &en);
  out.T = FV_T_MIN; out.mu = 0.0; out.ux = 0.0; out.uy = 0.0; out.n = 0.0; out.e = jmax(c.E, 0.0);
  out.P = P; out.ok = 0;
  return out;
}

/* _cons_to_prim_attempt_2d!, src2d/primrec2d.jl:511-742 */
template <int EOS, bool NCH>
FX_HD Recovery recover_attempt(const CellCons& c, const DevParams& d, double yT0, double phi0,
                               double ux0, double uy0, int maxit, double tol,
                               int budget = 0x7fffffff, bool* over_budget = nullptr) {
  Recovery out;
  const double yT_lo = d.log_T_min, yT_hi = d.log_T_solve_max;
  const double m = d.p.m_hq;
  out.reason = PRR_UNSET; out.resnorm = nan_();
  const double D = c.D, Sx = c.Sx, Sy = c.Sy, E = c.E;
  if (is_vacuum(c)) return vacuum_recovery<EOS>(c, d);
  const int NU = NCH ? 4 : 3;
  EosMemo memo; memo.reset();
  double x[4], F[4], Fp[4], Fm[4], J[4][4], delta[4];
  x[1] = (NCH && isfinite_(phi0)) ? jclamp(phi0, -FV_PHI_CAP, FV_PHI_CAP) : 0.0;
  if (isfinite_(yT0) && isfinite_(ux0) && isfinite_(uy0)) {
    x[0] = jclamp(yT0, yT_lo, yT_hi);
    x[2] = jclamp(ux0, -FV_U_CAP, FV_U_CAP);
    x[3] = jclamp(uy0, -FV_U_CAP, FV_U_CAP);
  } else {
    double sy, sx_, syy;
    seed_from_conserved<EOS>(E, Sx, Sy, x[1], d, &sy, &sx_, &syy);
    x[0] = jclamp(sy, yT_lo, yT_hi); x[2] = sx_; x[3] = syy;
  }
  evalF<EOS, NCH>(F, x, c, d, memo);
  if (!finite4(F)) {
    out.reason = PRR_NONFINITE_INITIAL;
    double T = jclamp(fx_exp(x[0]), FV_T_MIN, FV_T_SOLVE_MAX), P, n, en;
    eos_Pne<EOS>(T, m, d, &P, &n, &en);
    out.T = T; out.mu = m; out.ux = 0.0; out.uy = 0.0; out.n = 0.0; out.e = jmax(en, 0.0);
    out.P = P; out.ok = 0;
    return out;
  }
  const double sD = jmax(fabs_(D), 1e-12);
  const double sS = jmax(jmax(jmax(fabs_(Sx), fabs_(Sy)), 1e-10 * fabs_(E)), 1e-12);
  const double sE = jmax(fabs_(E), 1e-12);
  double rs[4];
  rs[0] = 1.0 / sD; rs[1] = 1.0 / sS; rs[2] = 1.0 / sS; rs[3] = 1.0 / sE;
  bool converged = false;
  double last_nrm = nan_();
  const int r_lo = NCH ? 0 : 1;

  for (int it = 1; it <= maxit; ++it) {
    double nrm = 0.0;
#pragma unroll
    for (int r = r_lo; r < 4; ++r) nrm = jmax(nrm, fabs_(F[r] * rs[r]));
    last_nrm = nrm;
    if (nrm < tol) { converged = true; out.reason = PRR_CONVERGED; break; }
    /* iteration budget of the fast pass: leave the cell to the full pass */
    if (it > budget) { *over_budget = true; return out; }
    bool ok_jac = true;
#pragma unroll
    for (int k = 0; k < NU; ++k) {
      const int s = NCH ? k : (k == 0 ? 0 : k + 1);
      double xs = x[s];
      double h = 1e-6 * jmax(1.0, fabs_(xs));
      x[s] = xs + h;
      evalF<EOS, NCH>(Fp, x, c, d, memo);
      x[s] = xs - h;
      evalF<EOS, NCH>(Fm, x, c, d, memo);
      x[s] = xs;
      if (!(finite4(Fp) && finite4(Fm))) { ok_jac = false; break; }
      double inv2h = 1.0 / (2.0 * h);
#pragma unroll
      for (int r = 0; r < NU; ++r) {
        const int rr = NCH ? r : r + 1;
        J[r][k] = ((Fp[rr] - Fm[rr]) * inv2h) * rs[rr];
      }
    }
    if (!ok_jac) { out.reason = PRR_NONFINITE_JACOBIAN; break; }
    double Fact[4];
#pragma unroll
    for (int r = 0; r < NU; ++r) {
      const int rr = NCH ? r : r + 1;
      delta[r] = 0.0;
      Fact[r] = F[rr] * rs[rr];
    }
    if (!solve_gauss<NU>(delta, J, Fact)) { out.reason = PRR_LINSOLVE_FAILED; break; }
    double alpha = 1.0;
#pragma unroll
    for (int k = 0; k < NU; ++k) {
      double ad = fabs_(delta[k]);
      if (ad > 1.0) alpha = jmin(alpha, 1.0 / ad);
    }
    const double xs1 = x[0], xs2 = x[1], xs3 = x[2], xs4 = x[3];
    bool accepted = false;
    for (int ls = 0; ls < 12; ++ls) {
      x[0] = xs1; x[1] = xs2; x[2] = xs3; x[3] = xs4;
      if (NCH) { x[0] += alpha * delta[0]; x[1] += alpha * delta[1]; x[2] += alpha * delta[2]; x[3] += alpha * delta[3]; }
      else { x[0] += alpha * delta[0]; x[2] += alpha * delta[1]; x[3] += alpha * delta[2]; }
      x[0] = jclamp(x[0], yT_lo, yT_hi);
      if (NCH) x[1] = jclamp(x[1], -FV_PHI_CAP, FV_PHI_CAP);
      x[2] = jclamp(x[2], -FV_U_CAP, FV_U_CAP);
      x[3] = jclamp(x[3], -FV_U_CAP, FV_U_CAP);
      evalF<EOS, NCH>(F, x, c, d, memo);
      if (finite4(F)) {
        double trial = 0.0;
#pragma unroll
        for (int r = r_lo; r < 4; ++r) trial = jmax(trial, fabs_(F[r] * rs[r]));
        if (trial < nrm * (1.0 - (1e-4 * alpha))) { accepted = true; break; }
      }
      alpha *= 0.5;
    }
    if (!accepted) { out.reason = PRR_LINESEARCH_FAILED; break; }
  }
  out.resnorm = last_nrm;
  double T = jclamp(fx_exp(x[0]), FV_T_MIN, FV_T_SOLVE_MAX);
  double mu = NCH ? (m + (T * x[1])) : m;
  double ux = x[2], uy = x[3];
  double P, n, en;
  eos_Pne_memo<EOS>(T, mu, d, memo, &P, &n, &en);
  if (!converged) out.reason = (out.reason == PRR_UNSET) ? PRR_MAXIT : out.reason;
  evalF<EOS, NCH>(F, x, c, d, memo);
  double rows[4] = {0.0, 0.0, 0.0, 0.0};
  double resnorm = 0.0;
#pragma unroll
  for (int r = r_lo; r < 4; ++r) { rows[r] = fabs_(F[r] * rs[r]); resnorm = jmax(resnorm, rows[r]); }
  out.resnorm = resnorm;
  out.T = T; out.mu = mu; out.ux = ux; out.uy = uy;
  if (!(isfinite_(resnorm) && resnorm < tol)) {
    double hyd = jmax(jmax(rows[1], rows[2]), rows[3]);
    if (NCH && isfinite_(hyd) && hyd < tol) {
      double phb; bool okb;
      solve_phi_bisect<EOS>(D, T, ux, uy, c.nux, c.nuy, d, memo, &phb, &okb);
      double xp = jclamp(phb, -FV_PHI_CAP, FV_PHI_CAP);
      mu = m + (T * xp);
      eos_Pne_memo<EOS>(T, mu, d, memo, &P, &n, &en);
      out.reason = okb ? PRR_CONVERGED : PRR_RESIDUAL_TOO_LARGE;
      out.mu = mu; out.n = jmax(n, 0.0); out.e = jmax(en, 0.0); out.P = P; out.ok = 1;
      return out;
    }
    out.reason = PRR_RESIDUAL_TOO_LARGE;
    out.n = n; out.e = jmax(en, 0.0); out.P = P; out.ok = 0;
    return out;
  }
  out.reason = PRR_CONVERGED;
  out.n = n; out.e = jmax(en, 0.0); out.P = P; out.ok = 1;
  return out;
}

/* cons_to_prim_2d!, src2d/primrec2d.jl:465-486 */
template <int EOS, bool NCH>
FX_HD Recovery recover(const CellCons& c, const DevParams& d, double yT0, double phi0, double ux0,
                       double uy0, int maxit, double tol) {
  Recovery r = recover_attempt<EOS, NCH>(c, d, yT0, phi0, ux0, uy0, maxit, tol);
  if (r.ok) return r;
  if (r.reason == PRR_VACUUM) return r;
  if (!(isfinite_(yT0) && isfinite_(ux0) && isfinite_(uy0))) return r;
  return recover_attempt<EOS, NCH>(c, d, nan_(), nan_(), nan_(), nan_(), maxit, tol);
}

/* ---------------------------------------------------------------------------
 * The warm-started attempt of the fast pass, with the EOS memo replaced by
 * explicit temperature parts. The memo of EOSCache2D only saves work: a hit
 * returns the bits of a fresh evaluation. Here the T-only part of the
 * LatticeHRG EOS (light P, e and e^x K2) is computed once per temperature and
 * handed to the evaluations that share it, so the 2 x NU Jacobian evaluations
 * of an iteration are straight-line independent code (two new temperatures,
 * T e^{+-h}, plus the current one for the other unknowns) that the compiler can
 * overlap, instead of a chain of calls that each branch on the memo.
 * ------------------------------------------------------------------------- */
struct TPart { double x, Pl, el, K2; };

/* the T-only part of eos_Pne_memo (src2d/primrec2d.jl:170-197) at T (before the floor) */
template <int EOS>
FX_HD void tpart(double T, const DevParams& d, TPart& tp) {
  if (EOS != FIVO_EOS_LATTICE_HRG) return;
  const double Tm = jmax(T, FV_T_MIN);
  tp.x = lhrg_x(Tm, d);
  double dP;
  light_eos<3>(Tm, d, &tp.Pl, &dP, nullptr);
  tp.el = (-tp.Pl) + (Tm * dP);
  tp.K2 = lhrg_K2(tp.x);
}

template <int EOS>
FX_HD void eos_tp(double T, double mu, const DevParams& d, const TPart& tp, double* P, double* n, double* en) {
  if (EOS != FIVO_EOS_LATTICE_HRG) { eos_Pne<EOS>(T, mu, d, P, n, en); return; }
  const double Tm = jmax(T, FV_T_MIN);
  lhrg_assemble(Tm, mu, d, tp.x, tp.Pl, tp.el, tp.K2, P, n, en);
}

/* evalF_2d! (src2d/primrec2d.jl:360-390) with tp the T-part of exp(x[0]);
 * *eo receives the EOS values at x when given */
struct EosAt { double P, n, en; };
template <int EOS, bool NCH>
FX_HD void evalF_tp(double F[4], const double x[4], double T, const CellCons& c, const DevParams& d,
                    const TPart& tp, EosAt* eo = nullptr) {
  double yT = x[0], phi = x[1], ux = x[2], uy = x[3];
  if (!(isfinite_(yT) && isfinite_(phi) && isfinite_(ux) && isfinite_(uy))) {
    F[0] = F[1] = F[2] = F[3] = inf_(); return;
  }
  double mu = d.p.m_hq + (T * phi);
  double ut = utau(ux, uy);
  double P, n, en;
  eos_tp<EOS>(T, mu, d, tp, &P, &n, &en);
  if (eo) { eo->P = P; eo->n = n; eo->en = en; }
  evalF_rows<NCH>(F, P, n, en, ux, uy, ut, c);
}

/* recover_attempt from a finite warm start (x0 already clamped), with the
 * iteration budget of the fast pass; the same arithmetic, rounded the same way */
template <int EOS, bool NCH>
FX_HD Recovery recover_fast(const CellCons& c, const DevParams& d, double yT0, double phi0, double ux0,
                            double uy0, int maxit, double tol, int budget, bool* over_budget,
                            int check_it = 0x7fffffff, double check_tol = 0.0, int* iters = nullptr) {
  Recovery out;
  const double yT_lo = d.log_T_min, yT_hi = d.log_T_solve_max;
  const double m = d.p.m_hq;
  out.reason = PRR_UNSET; out.resnorm = nan_();
  const double D = c.D, Sx = c.Sx, Sy = c.Sy, E = c.E;
  if (is_vacuum(c)) return vacuum_recovery<EOS>(c, d);
  const int NU = NCH ? 4 : 3;
  double x[4], F[4], J[4][4] = {}, delta[4];
  x[1] = (NCH && isfinite_(phi0)) ? jclamp(phi0, -FV_PHI_CAP, FV_PHI_CAP) : 0.0;
  x[0] = jclamp(yT0, yT_lo, yT_hi);
  x[2] = jclamp(ux0, -FV_U_CAP, FV_U_CAP);
  x[3] = jclamp(uy0, -FV_U_CAP, FV_U_CAP);
  double Tc = fx_exp(x[0]);
  TPart tpc;
  EosAt ec;    /* the EOS values of the last evaluation at x */
  tpart<EOS>(Tc, d, tpc);
  evalF_tp<EOS, NCH>(F, x, Tc, c, d, tpc, &ec);
  if (!finite4(F)) {
    out.reason = PRR_NONFINITE_INITIAL;
    double T = jclamp(fx_exp(x[0]), FV_T_MIN, FV_T_SOLVE_MAX), P, n, en;
    eos_Pne<EOS>(T, m, d, &P, &n, &en);
    out.T = T; out.mu = m; out.ux = 0.0; out.uy = 0.0; out.n = 0.0; out.e = jmax(en, 0.0);
    out.P = P; out.ok = 0;
    return out;
  }
  const double sD = jmax(fabs_(D), 1e-12);
  const double sS = jmax(jmax(jmax(fabs_(Sx), fabs_(Sy)), 1e-10 * fabs_(E)), 1e-12);
  const double sE = jmax(fabs_(E), 1e-12);
  double rs[4];
  rs[0] = 1.0 / sD; rs[1] = 1.0 / sS; rs[2] = 1.0 / sS; rs[3] = 1.0 / sE;
  bool converged = false;
  double last_nrm = nan_();
  const int r_lo = NCH ? 0 : 1;

  int nupd = 0;
  for (int it = 1; it <= maxit; ++it) {
    nupd = it - 1;
    double nrm = 0.0;
#pragma unroll
    for (int r = r_lo; r < 4; ++r) nrm = jmax(nrm, fabs_(F[r] * rs[r]));
    last_nrm = nrm;
    if (nrm < tol) { converged = true; out.reason = PRR_CONVERGED; break; }
    /* the budget of the fast pass, and the learned guess's test after check_it updates */
    if (it > budget || (it == check_it + 1 && !(nrm <= check_tol))) {
      *over_budget = true;
      if (iters) *iters = nupd;
      return out;
    }
    /* ---- Jacobian: all 2 NU evaluations, then the finiteness test of the columns */
    const double h0 = 1e-6 * jmax(1.0, fabs_(x[0]));
    double Tp = 0.0, Tn = 0.0;
    TPart tpp, tpn;
#pragma unroll 1
    for (int sg = 0; sg < 2; ++sg) {   /* T e^{+h}, then T e^{-h}: one inlined copy */
      const double Tq = fx_exp(sg ? x[0] - h0 : x[0] + h0);
      TPart t;
      tpart<EOS>(Tq, d, t);
      if (sg) { Tn = Tq; tpn = t; } else { Tp = Tq; tpp = t; }
    }
    /* one column per trip of a loop that is not unrolled: two evaluation sites
     * instead of 2 NU keep the kernel's code small (instruction fetch, not the
     * FP64 pipe, is what its warps wait on most). The column enters J from the
     * right and the earlier ones shift left, so J keeps static indices. */
    bool ok_jac = true;
#pragma unroll 1
    for (int k = 0; k < NU; ++k) {
      const int s = NCH ? k : (k == 0 ? 0 : k + 1);
      const double xs = s == 0 ? x[0] : (s == 1 ? x[1] : (s == 2 ? x[2] : x[3]));
      const double h = 1e-6 * jmax(1.0, fabs_(xs));
      const double xsp = xs + h, xsm = xs - h;
      double xp[4], xm[4];
      xp[0] = s == 0 ? xsp : x[0]; xm[0] = s == 0 ? xsm : x[0];
      xp[1] = s == 1 ? xsp : x[1]; xm[1] = s == 1 ? xsm : x[1];
      xp[2] = s == 2 ? xsp : x[2]; xm[2] = s == 2 ? xsm : x[2];
      xp[3] = s == 3 ? xsp : x[3]; xm[3] = s == 3 ? xsm : x[3];
      const bool ts = s == 0;
      TPart ap, am;
      ap.x = ts ? tpp.x : tpc.x; ap.Pl = ts ? tpp.Pl : tpc.Pl; ap.el = ts ? tpp.el : tpc.el; ap.K2 = ts ? tpp.K2 : tpc.K2;
      am.x = ts ? tpn.x : tpc.x; am.Pl = ts ? tpn.Pl : tpc.Pl; am.el = ts ? tpn.el : tpc.el; am.K2 = ts ? tpn.K2 : tpc.K2;
      double fp[4], fm[4];
      if (s <= 1) {
        evalF_tp<EOS, NCH>(fp, xp, ts ? Tp : Tc, c, d, ap);
        evalF_tp<EOS, NCH>(fm, xm, ts ? Tn : Tc, c, d, am);
      } else {
        /* a velocity column keeps x's T and phi, so mu and the EOS values are
         * those at x (the same pure function of the same arguments); the
         * shifted points are finite, x being finite and clamped */
        evalF_rows<NCH>(fp, ec.P, ec.n, ec.en, xp[2], xp[3], utau(xp[2], xp[3]), c);
        evalF_rows<NCH>(fm, ec.P, ec.n, ec.en, xm[2], xm[3], utau(xm[2], xm[3]), c);
      }
      ok_jac = ok_jac && finite4(fp) && finite4(fm);
      const double inv2h = 1.0 / (2.0 * h);
#pragma unroll
      for (int r = 0; r < NU; ++r) {
        const int rr = NCH ? r : r + 1;
#pragma unroll
        for (int q = 0; q + 1 < NU; ++q) J[r][q] = J[r][q + 1];
        J[r][NU - 1] = ((fp[rr] - fm[rr]) * inv2h) * rs[rr];
      }
    }
    if (!ok_jac) { out.reason = PRR_NONFINITE_JACOBIAN; break; }
    double Fact[4];
#pragma unroll
    for (int r = 0; r < NU; ++r) {
      const int rr = NCH ? r : r + 1;
      delta[r] = 0.0;
      Fact[r] = F[rr] * rs[rr];
    }
    if (!solve_gauss<NU>(delta, J, Fact)) { out.reason = PRR_LINSOLVE_FAILED; break; }
    double alpha = 1.0;
#pragma unroll
    for (int k = 0; k < NU; ++k) {
      double ad = fabs_(delta[k]);
      if (ad > 1.0) alpha = jmin(alpha, 1.0 / ad);
    }
    const double xs1 = x[0], xs2 = x[1], xs3 = x[2], xs4 = x[3];
    bool accepted = false;
    for (int ls = 0; ls < 12; ++ls) {
      x[0] = xs1; x[1] = xs2; x[2] = xs3; x[3] = xs4;
      if (NCH) { x[0] += alpha * delta[0]; x[1] += alpha * delta[1]; x[2] += alpha * delta[2]; x[3] += alpha * delta[3]; }
      else { x[0] += alpha * delta[0]; x[2] += alpha * delta[1]; x[3] += alpha * delta[2]; }
      x[0] = jclamp(x[0], yT_lo, yT_hi);
      if (NCH) x[1] = jclamp(x[1], -FV_PHI_CAP, FV_PHI_CAP);
      x[2] = jclamp(x[2], -FV_U_CAP, FV_U_CAP);
      x[3] = jclamp(x[3], -FV_U_CAP, FV_U_CAP);
      Tc = fx_exp(x[0]);
      tpart<EOS>(Tc, d, tpc);
      evalF_tp<EOS, NCH>(F, x, Tc, c, d, tpc, &ec);
      if (finite4(F)) {
        double trial = 0.0;
#pragma unroll
        for (int r = r_lo; r < 4; ++r) trial = jmax(trial, fabs_(F[r] * rs[r]));
        if (trial < nrm * (1.0 - (1e-4 * alpha))) { accepted = true; break; }
      }
      alpha *= 0.5;
    }
    if (!accepted) { out.reason = PRR_LINESEARCH_FAILED; break; }
  }
  if (iters) *iters = nupd;
  out.resnorm = last_nrm;
  /* Here Tc = exp(x[0]), tpc is its temperature part and F the residual at x:
   * every exit of the loop leaves the three from the last evaluation at x. The
   * closing EOS call reuses tpc unless the clamp moved T, and the closing
   * residual is F itself (the same pure function of the same arguments). */
  double T = jclamp(Tc, FV_T_MIN, FV_T_SOLVE_MAX);
  double mu = NCH ? (m + (T * x[1])) : m;
  double ux = x[2], uy = x[3];
  double P, n, en;
  {
    TPart tpf = tpc;
    if (!(T == Tc)) tpart<EOS>(T, d, tpf);
    eos_tp<EOS>(T, mu, d, tpf, &P, &n, &en);
  }
  if (!converged) out.reason = (out.reason == PRR_UNSET) ? PRR_MAXIT : out.reason;
  double rows[4] = {0.0, 0.0, 0.0, 0.0};
  double resnorm = 0.0;
#pragma unroll
  for (int r = r_lo; r < 4; ++r) { rows[r] = fabs_(F[r] * rs[r]); resnorm = jmax(resnorm, rows[r]); }
  out.resnorm = resnorm;
  out.T = T; out.mu = mu; out.ux = ux; out.uy = uy;
  if (!(isfinite_(resnorm) && resnorm < tol)) {
    double hyd = jmax(jmax(rows[1], rows[2]), rows[3]);
    if (NCH && isfinite_(hyd) && hyd < tol) {
      EosMemo memo; memo.reset();
      double phb; bool okb;
      solve_phi_bisect<EOS>(D, T, ux, uy, c.nux, c.nuy, d, memo, &phb, &okb);
      double xp = jclamp(phb, -FV_PHI_CAP, FV_PHI_CAP);
      mu = m + (T * xp);
      eos_Pne_memo<EOS>(T, mu, d, memo, &P, &n, &en);
      out.reason = okb ? PRR_CONVERGED : PRR_RESIDUAL_TOO_LARGE;
      out.mu = mu; out.n = jmax(n, 0.0); out.e = jmax(en, 0.0); out.P = P; out.ok = 1;
      return out;
    }
    out.reason = PRR_RESIDUAL_TOO_LARGE;
    out.n = n; out.e = jmax(en, 0.0); out.P = P; out.ok = 0;
    return out;
  }
  out.reason = PRR_CONVERGED;
  out.n = n; out.e = jmax(en, 0.0); out.P = P; out.ok = 1;
  return out;
}

/* ==================== prim -> cons and fluxes ==================== */

/* PrimIdealVisc2D without the ok flag; dissipatives in physical units */
struct Prim { double T, mu, ux, uy, n, e, P, cs2, nux, nuy, Pi, pixx, pixy, piyy, pieta; };

/* prim_to_cons_2d!, src2d/primrec2d.jl:753-796, writing the conserved four into
 * uc[0..3] (Dtau, Sx, Sy, E); also returns cs2 at the same T (for HLLE).
 * Returns false (and leaves uc untouched) when the EOS state is not valid. */
template <int EOS>
FX_HD bool prim_to_cons(double uc[4], Prim& pr, double T, double mu, double ux, double uy,
                        const double dis[7], double tau, const DevParams& d) {
  double Tc = jmax(T, FV_T_MIN);
  double ut = utau(ux, uy);
  double P, n, en, cs2;
  eos_Pne_cs2<EOS>(Tc, mu, d, &P, &n, &en, &cs2);
  pr.T = Tc; pr.mu = mu;
  pr.nux = dis[0]; pr.nuy = dis[1]; pr.Pi = dis[2]; pr.pixx = dis[3]; pr.pixy = dis[4];
  pr.piyy = dis[5]; pr.pieta = dis[6];
  if (!(isfinite_(P) && isfinite_(n) && isfinite_(en)) || en <= 0.0) {
    pr.ux = 0.0; pr.uy = 0.0; pr.n = 0.0; pr.e = 0.0; pr.P = 0.0; pr.cs2 = cs2;
    return false;
  }
  double weff = (en + P) + dis[2];
  double Ptot = P + dis[2];
  PiC pc = shear_tensor(ux, uy, ut, dis[3], dis[4], dis[5]);
  double Jt = (n * ut) + nu_tau(ux, uy, ut, dis[0], dis[1]);
  uc[0] = tau * Jt;
  uc[1] = ((weff * ut) * ux) + pc.tx;
  uc[2] = ((weff * ut) * uy) + pc.ty;
  uc[3] = (((weff * ut) * ut) - Ptot) + pc.tt;
  pr.ux = ux; pr.uy = uy; pr.n = n; pr.e = en; pr.P = P; pr.cs2 = cs2;
  return true;
}

/* wavespeeds_2d, src2d/fluxes2d.jl:87-113 (cs2 precomputed by prim_to_cons) */
template <bool XDIR>
FX_HD void wavespeeds(const Prim& p, double pinn, double* lm, double* lp) {
  double cs2 = jclamp(p.cs2, 0.0, 0.999);
  double w = p.e + p.P;
  if (w > FV_TINY) cs2 = jmin(cs2 + ((fabs_(p.Pi) + fabs_(pinn)) / w), 0.999);
  double ut = utau(p.ux, p.uy);
  double iu = safe_inv(ut);
  double vx = p.ux * iu, vy = p.uy * iu;
  double v2 = (vx * vx) + (vy * vy);
  double vn = XDIR ? vx : vy;
  double den = 1.0 - (v2 * cs2);
  if (den <= FV_TINY) { *lm = -1.0; *lp = 1.0; return; }
  double cs = safe_sqrt(cs2);
  double rad = (1.0 - v2) * (den - ((vn * vn) * (1.0 - cs2)));
  double disc = cs * safe_sqrt(jmax(rad, 0.0));
  double a = ((vn * (1.0 - cs2)) - disc) / den;
  double b = ((vn * (1.0 - cs2)) + disc) / den;
  *lm = jclamp(a, -1.0, 1.0);
  *lp = jclamp(b, -1.0, 1.0);
}

/* the conserved four rows of flux_cell_2d! (src2d/fluxes2d.jl:24-69) and the
 * normal velocity v that the advected rows multiply */
template <bool XDIR>
FX_HD void flux_cons4(double F[4], const Prim& p, double tau, double* vn) {
  double ux = p.ux, uy = p.uy;
  double ut = utau(ux, uy);
  double iu = safe_inv(ut);
  double vx = ux * iu, vy = uy * iu;
  double Ptot = p.P + p.Pi;
  double weff = (p.e + p.P) + p.Pi;
  PiC pc = shear_tensor(ux, uy, ut, p.pixx, p.pixy, p.piyy);
  double Jx = (p.n * ux) + p.nux, Jy = (p.n * uy) + p.nuy;
  if (XDIR) {
    F[0] = tau * Jx;
    F[1] = (((weff * ux) * ux) + Ptot) + pc.xx;
    F[2] = ((weff * ux) * uy) + pc.xy;
    F[3] = ((weff * ut) * ux) + pc.tx;
    *vn = vx;
  } else {
    F[0] = tau * Jy;
    F[1] = ((weff * ux) * uy) + pc.xy;
    F[2] = (((weff * uy) * uy) + Ptot) + pc.yy;
    F[3] = ((weff * ut) * uy) + pc.ty;
    *vn = vy;
  }
}

/* flux_cell_2d!, src2d/fluxes2d.jl:24-69: conserved four into F[0..3], the
 * advected dissipatives (only with advect_*) into F[4..10] by field order
 * nux, nuy, Pi, pixx, pixy, piyy, pieta. */
template <bool XDIR>
FX_HD void flux_cell(double F[11], const Prim& p, double tau, const DevParams& d) {
  double v;
  flux_cons4<XDIR>(F, p, tau, &v);
  bool an = d.hasNu && d.p.advect_nu, aP = d.hasPi && d.p.advect_Pi, ap = d.hasShear && d.p.advect_pi;
  F[4] = an ? p.nux * v : 0.0;
  F[5] = an ? p.nuy * v : 0.0;
  F[6] = aP ? p.Pi * v : 0.0;
  F[7] = ap ? p.pixx * v : 0.0;
  F[8] = ap ? p.pixy * v : 0.0;
  F[9] = ap ? p.piyy * v : 0.0;
  F[10] = ap ? p.pieta * v : 0.0;
}

/* mc_limiter, src/utils.jl:14-22 */
FX_HD double mc_limiter(double a, double b) {
  if (jsign(a) != jsign(b)) return 0.0;
  double s = jsign(a);
  double aa = fabs_(a), bb = fabs_(b);
  return s * jmin(2.0 * aa, jmin(2.0 * bb, 0.5 * (aa + bb)));
}

}  // namespace fv
#endif
