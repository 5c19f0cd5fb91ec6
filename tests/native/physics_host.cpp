/*
 * Host build of the library's per-cell physics (csrc/physics.cuh, compiled as
 * plain C++), exported for tests/test_physics_host.py, which compares it bit
 * for bit with the oracle on the CPU. Test code only.
 */
#include <cstring>
#include "../../fivohydro.jl_b200/csrc/physics.cuh"

using namespace fv;

static DevParams mk(const fivo_params* p) {
  DevParams d;
  std::memset(&d, 0, sizeof(d));
  d.p = *p;
  d.ncharge = (p->eos_kind == FIVO_EOS_CONFORMAL_HQ) ? (p->g_hq > 0.0) : 1;
  const double fmgev = 1.0 / 0.1973269804;
  d.fmgev3 = (fmgev * fmgev) * fmgev;
  d.pi2 = FX_PI * FX_PI;
  d.aSB = (d.pi2 / 90.0) * p->g_eff;
  double m = p->m_hq, g = p->g_hq;
  d.A_conf = (g * (m * m)) / (2.0 * d.pi2);
  d.A_lhrg = ((p->canon_factor * g) * (m * m)) / (2.0 * d.pi2);
  d.lA = 0.01 * (p->lhrg_d * p->lhrg_d);
  d.lB = 0.1 * (p->lhrg_c * p->lhrg_c);
  d.log_T_min = fx_log(FV_T_MIN);
  d.log_T_solve_max = fx_log(FV_T_SOLVE_MAX);
  d.log_seed_T = fx_log(jmax(0.15, FV_T_MIN));
  return d;
}

extern "C" {
void ph_exp(long n, const double* x, double* o) { for (long i = 0; i < n; ++i) o[i] = fx_exp(x[i]); }
void ph_log(long n, const double* x, double* o) { for (long i = 0; i < n; ++i) o[i] = fx_log(x[i]); }
void ph_pow4(long n, const double* x, double* o) { for (long i = 0; i < n; ++i) o[i] = fx_pow4(x[i]); }
void ph_hypot(long n, const double* x, const double* y, double* o) { for (long i = 0; i < n; ++i) o[i] = fx_hypot(x[i], y[i]); }
void ph_besselkx(int nu, long n, const double* x, double* o) { for (long i = 0; i < n; ++i) o[i] = fx_besselkx(nu, x[i]); }

void ph_eos(const fivo_params* p, long n, const double* T, const double* mu, double* P, double* nq, double* e,
            double* cs2) {
  DevParams d = mk(p);
  for (long i = 0; i < n; ++i) {
    if (p->eos_kind == FIVO_EOS_LATTICE_HRG) {
      eos_Pne<FIVO_EOS_LATTICE_HRG>(T[i], mu[i], d, P + i, nq + i, e + i);
      cs2[i] = eos_cs2<FIVO_EOS_LATTICE_HRG>(T[i], d);
    } else {
      eos_Pne<FIVO_EOS_CONFORMAL_HQ>(T[i], mu[i], d, P + i, nq + i, e + i);
      cs2[i] = eos_cs2<FIVO_EOS_CONFORMAL_HQ>(T[i], d);
    }
  }
}

void ph_cons_to_prim(const fivo_params* p, long n, double tau, const double* cons, const double* warm,
                     double* prim, unsigned char* ok, unsigned char* reason) {
  DevParams d = mk(p);
  for (long i = 0; i < n; ++i) {
    const double* c = cons + 11 * i;
    CellCons cc;
    cc.D = c[0]; cc.Sx = c[1]; cc.Sy = c[2]; cc.E = c[3]; cc.nux = c[4]; cc.nuy = c[5]; cc.Pi = c[6];
    cc.pixx = c[7]; cc.pixy = c[8]; cc.piyy = c[9]; cc.pieta = c[10];
    double y0 = nan_(), f0 = nan_(), x0 = nan_(), v0 = nan_();
    if (warm) { y0 = warm[4 * i]; f0 = warm[4 * i + 1]; x0 = warm[4 * i + 2]; v0 = warm[4 * i + 3]; }
    Recovery r;
    if (p->eos_kind == FIVO_EOS_LATTICE_HRG) r = recover<FIVO_EOS_LATTICE_HRG, true>(cc, d, y0, f0, x0, v0, p->primrec_maxit, p->primrec_tol);
    else if (d.ncharge) r = recover<FIVO_EOS_CONFORMAL_HQ, true>(cc, d, y0, f0, x0, v0, p->primrec_maxit, p->primrec_tol);
    else r = recover<FIVO_EOS_CONFORMAL_HQ, false>(cc, d, y0, f0, x0, v0, p->primrec_maxit, p->primrec_tol);
    double* o = prim + 7 * i;
    o[0] = r.T; o[1] = r.mu; o[2] = r.ux; o[3] = r.uy; o[4] = r.n; o[5] = r.e; o[6] = r.P;
    ok[i] = r.ok; reason[i] = r.reason;
  }
}

/* the fast pass's recovery (recover_fast, explicit EOS temperature parts) against the
 * memo-based first attempt from the same finite warm start, for every cell: returns
 * the number of cells whose results differ in any bit */
long ph_fast_vs_attempt(const fivo_params* p, long n, double tau, const double* cons, const double* warm, int budget) {
  DevParams d = mk(p);
  long bad = 0;
  for (long i = 0; i < n; ++i) {
    const double* c = cons + 11 * i;
    CellCons cc;
    cc.D = c[0]; cc.Sx = c[1]; cc.Sy = c[2]; cc.E = c[3]; cc.nux = c[4]; cc.nuy = c[5]; cc.Pi = c[6];
    cc.pixx = c[7]; cc.pixy = c[8]; cc.piyy = c[9]; cc.pieta = c[10];
    const double* w = warm + 4 * i;
    bool over = false;
    Recovery a, b;
    if (p->eos_kind == FIVO_EOS_LATTICE_HRG) {
      a = recover_attempt<FIVO_EOS_LATTICE_HRG, true>(cc, d, w[0], w[1], w[2], w[3], p->primrec_maxit, p->primrec_tol);
      b = recover_fast<FIVO_EOS_LATTICE_HRG, true>(cc, d, w[0], w[1], w[2], w[3], p->primrec_maxit, p->primrec_tol, budget, &over);
    } else {
      a = recover_attempt<FIVO_EOS_CONFORMAL_HQ, true>(cc, d, w[0], w[1], w[2], w[3], p->primrec_maxit, p->primrec_tol);
      b = recover_fast<FIVO_EOS_CONFORMAL_HQ, true>(cc, d, w[0], w[1], w[2], w[3], p->primrec_maxit, p->primrec_tol, budget, &over);
    }
    if (over) continue;   /* the fast pass would defer this cell */
    const double va[8] = {a.T, a.mu, a.ux, a.uy, a.n, a.e, a.P, a.resnorm};
    const double vb[8] = {b.T, b.mu, b.ux, b.uy, b.n, b.e, b.P, b.resnorm};
    if (std::memcmp(va, vb, sizeof(va)) != 0 || a.ok != b.ok || a.reason != b.reason) ++bad;
  }
  return bad;
}
}
