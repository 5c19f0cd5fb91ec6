/*
 * oracle/oracle_capi.cpp — extern "C" face of the CPU oracle, for the tests
 * (ctypes) and for bench.py's CPU-baseline leg. TEST INFRASTRUCTURE ONLY.
 * Signatures mirror include/fivo2d.h with an `oracle_` prefix; the state is
 * the reference's AoS U[a, i] (cell i, field a at U[i*nv + a]).
 */
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include "oracle_core.h"

using namespace orc;

namespace {
thread_local std::string g_err;
struct OCtx {
  Grid g;
  Model m;
  Work w;
  std::vector<double> U;
  int64_t nsteps_run = 0;
};
}  // namespace

extern "C" {

const char* oracle_last_error(void) { return g_err.c_str(); }

void* oracle_ctx_create(const fivo_params* p, int nx, int ny, int ng, double xmax, double ymax) {
  if (!p || nx <= 8 || ny <= 8 || ng != 3 || !(xmax > 0) || !(ymax > 0)) { g_err = "bad grid"; return nullptr; }
  OCtx* c = new OCtx();
  const char* err = nullptr;
  if (!make_model(*p, c->m, &err)) { g_err = err ? err : "bad model"; delete c; return nullptr; }
  make_grid(nx, ny, ng, xmax, ymax, c->g);
  make_work(c->g, c->m, c->w);
  c->U.assign((size_t)c->m.L.nv * c->g.Ntot, 0.0);
  return c;
}

void oracle_ctx_destroy(void* h) { delete (OCtx*)h; }

int oracle_ctx_info(void* h, int* nv, int64_t* ntot, double* evac) {
  OCtx* c = (OCtx*)h;
  if (nv) *nv = c->m.L.nv;
  if (ntot) *ntot = c->g.Ntot;
  if (evac) *evac = c->m.E_vac_cut;
  return 0;
}

void oracle_set_state(void* h, const double* U) { OCtx* c = (OCtx*)h; std::memcpy(c->U.data(), U, c->U.size() * 8); }
void oracle_get_state(void* h, double* U) { OCtx* c = (OCtx*)h; std::memcpy(U, c->U.data(), c->U.size() * 8); }

void oracle_set_history(void* h, const double* x0_yT, const double* x0_phi, const double* x0_ux,
                        const double* x0_uy, const double* ux_prev, const double* uy_prev,
                        const double* alpha_prev, const double* T_prev) {
  OCtx* c = (OCtx*)h;
  size_t n = (size_t)c->g.Ntot * 8;
  if (x0_yT) std::memcpy(c->w.x0_yT.data(), x0_yT, n);
  if (x0_phi) std::memcpy(c->w.x0_phi.data(), x0_phi, n);
  if (x0_ux) std::memcpy(c->w.x0_ux.data(), x0_ux, n);
  if (x0_uy) std::memcpy(c->w.x0_uy.data(), x0_uy, n);
  if (ux_prev) std::memcpy(c->w.ux_prev.data(), ux_prev, n);
  if (uy_prev) std::memcpy(c->w.uy_prev.data(), uy_prev, n);
  if (alpha_prev) std::memcpy(c->w.alpha_prev.data(), alpha_prev, n);
  if (T_prev) std::memcpy(c->w.T_prev.data(), T_prev, n);
}

void oracle_get_history(void* h, double* x0_yT, double* x0_phi, double* x0_ux, double* x0_uy,
                        double* ux_prev, double* uy_prev, double* alpha_prev, double* T_prev) {
  OCtx* c = (OCtx*)h;
  size_t n = (size_t)c->g.Ntot * 8;
  if (x0_yT) std::memcpy(x0_yT, c->w.x0_yT.data(), n);
  if (x0_phi) std::memcpy(x0_phi, c->w.x0_phi.data(), n);
  if (x0_ux) std::memcpy(x0_ux, c->w.x0_ux.data(), n);
  if (x0_uy) std::memcpy(x0_uy, c->w.x0_uy.data(), n);
  if (ux_prev) std::memcpy(ux_prev, c->w.ux_prev.data(), n);
  if (uy_prev) std::memcpy(uy_prev, c->w.uy_prev.data(), n);
  if (alpha_prev) std::memcpy(alpha_prev, c->w.alpha_prev.data(), n);
  if (T_prev) std::memcpy(T_prev, c->w.T_prev.data(), n);
}

void oracle_reset_history(void* h) {
  OCtx* c = (OCtx*)h;
  c->nsteps_run = 0;
  for (auto* v : {&c->w.x0_yT, &c->w.x0_phi, &c->w.x0_ux, &c->w.x0_uy, &c->w.ux_prev, &c->w.uy_prev,
                  &c->w.alpha_prev, &c->w.T_prev, &c->w.nux_prev, &c->w.nuy_prev})
    std::fill(v->begin(), v->end(), O_NAN);
}

void oracle_set_nu_history(void* h, const double* nux_prev, const double* nuy_prev) {
  OCtx* c = (OCtx*)h;
  size_t n = c->w.nux_prev.size() * 8;
  if (nux_prev) std::memcpy(c->w.nux_prev.data(), nux_prev, n);
  if (nuy_prev) std::memcpy(c->w.nuy_prev.data(), nuy_prev, n);
}

void oracle_get_nu_history(void* h, double* nux_prev, double* nuy_prev) {
  OCtx* c = (OCtx*)h;
  size_t n = c->w.nux_prev.size() * 8;
  if (nux_prev) std::memcpy(nux_prev, c->w.nux_prev.data(), n);
  if (nuy_prev) std::memcpy(nuy_prev, c->w.nuy_prev.data(), n);
}

void oracle_get_primitives(void* h, double* yT, double* phi, double* mu, double* alpha, double* ux,
                           double* uy, double* P, double* n, double* e, uint8_t* ok) {
  OCtx* c = (OCtx*)h;
  size_t N = (size_t)c->g.Ntot, nb = N * 8;
  if (yT) std::memcpy(yT, c->w.yT.data(), nb);
  if (phi) std::memcpy(phi, c->w.phi.data(), nb);
  if (mu) std::memcpy(mu, c->w.mu.data(), nb);
  if (alpha) std::memcpy(alpha, c->w.alpha.data(), nb);
  if (ux) std::memcpy(ux, c->w.ux.data(), nb);
  if (uy) std::memcpy(uy, c->w.uy.data(), nb);
  if (P) std::memcpy(P, c->w.P.data(), nb);
  if (n) std::memcpy(n, c->w.n.data(), nb);
  if (e) std::memcpy(e, c->w.e.data(), nb);
  if (ok) std::memcpy(ok, c->w.ok.data(), N);
}

void oracle_get_counters(void* h, fivo_counters* out) {
  OCtx* c = (OCtx*)h;
  std::memset(out, 0, sizeof(*out));
  out->nprimfail = c->w.nprimfail; out->nvacuum = c->w.nvacuum; out->primfail_index = c->w.primfail_i;
  out->primfail_reason = c->w.primfail_reason; out->primfail_resnorm = c->w.primfail_resnorm;
  out->amax = c->w.amax; out->nmood = c->w.nmood; out->nhalve = c->w.nhalve;
}

void oracle_rhs(void* h, double tau, int bc, const uint8_t* mask, double* dU) {
  OCtx* c = (OCtx*)h;
  rhs_2d(c->w.k.data(), c->U.data(), c->g, tau, c->m, c->w, bc, E_FLOOR, mask);
  if (dU) std::memcpy(dU, c->w.k.data(), c->w.k.size() * 8);
}

void oracle_step(void* h, int integrator, double tau, double dtau, int max_halve, int max_mood, int bc,
                 double* used, int* ok) {
  OCtx* c = (OCtx*)h;
  bool r = integrator == FIVO_SSPRK3
               ? step_ssprk3_2d(c->U.data(), c->g, tau, dtau, c->m, c->w, bc, max_halve, used)
               : step_ssprk2_2d(c->U.data(), c->g, tau, dtau, c->m, c->w, bc, max_halve, max_mood, used);
  *ok = r ? 1 : 0;
}

int64_t oracle_update_primitives(void* h, double tau, int bc) {
  OCtx* c = (OCtx*)h;
  return update_primitives_2d(c->U.data(), c->g, tau, c->m, c->w, bc);
}

void oracle_relax(void* h, double tau, double dtau) {
  OCtx* c = (OCtx*)h;
  relax_dissipative_2d(c->U.data(), c->g, tau, dtau, c->m, c->w);
}

void oracle_project_shear(void* h, double* maxr, double* meanr) {
  OCtx* c = (OCtx*)h;
  project_shear(c->U.data(), c->g, c->w, c->m, maxr, meanr);
}

double oracle_compute_dt(void* h, double tau, double cfl, double cfltau) {
  OCtx* c = (OCtx*)h;
  return compute_dt_2d(c->w, c->g, tau, cfl, cfltau);
}

void oracle_run(void* h, double tau0, double taufinal, double cfl, double cfltau, int integrator, int bc,
                int64_t max_steps, int reset_history, fivo_run_result* out) {
  OCtx* c = (OCtx*)h;
  run_sim_2d(c->U.data(), c->g, c->m, c->w, tau0, taufinal, cfl, cfltau, integrator, bc,
             reset_history != 0, max_steps, out);
  c->nsteps_run = out->nsteps;
}

void oracle_advance(void* h, double tau, double taufinal, double cfl, double cfltau, int integrator, int bc,
                    int64_t max_steps, fivo_run_result* out) {
  OCtx* c = (OCtx*)h;
  std::memset(out, 0, sizeof(*out));
  advance_sim_2d(c->U.data(), c->g, c->m, c->w, tau, taufinal, cfl, cfltau, integrator, bc, max_steps,
                 &c->nsteps_run, out);
}

void oracle_finalize_ic(void* h, double tau0, int bc) {
  OCtx* c = (OCtx*)h;
  finalize_ic(c->U.data(), c->g, c->m, bc, E_FLOOR, tau0);
}

/* set_cell!, main2D.jl:142-154, for ncell cells (U column left untouched on failure) */
int oracle_set_cells(const fivo_params* p, int64_t ncell, double tau, const double* T, const double* alpha,
                     const double* ux, const double* uy, const double* Pi, const double* pixx,
                     const double* pixy, const double* piyy, const double* nux, const double* nuy,
                     double* U, uint8_t* ok) {
  Model m;
  const char* err = nullptr;
  if (!make_model(*p, m, &err)) { g_err = err ? err : "bad model"; return 2; }
  const Layout& L = m.L;
#pragma omp parallel for
  for (int64_t i = 0; i < ncell; ++i) {
    double vx = ux[i], vy = uy[i];
    double ut = std::sqrt((1.0 + (vx * vx)) + (vy * vy));
    double pxx = pixx ? pixx[i] : 0.0, pxy = pixy ? pixy[i] : 0.0, pyy = piyy ? piyy[i] : 0.0;
    double iu = safe_inv(ut);
    double tx = ((vx * pxx) + (vy * pxy)) * iu;
    double ty = ((vx * pxy) + (vy * pyy)) * iu;
    double tt = ((vx * tx) + (vy * ty)) * iu;
    double pieta = (tt - pxx) - pyy;
    bool r = prim_to_cons_2d(U + i * L.nv, T[i], alpha[i] * T[i], vx, vy, nux ? nux[i] : 0.0,
                             nuy ? nuy[i] : 0.0, Pi ? Pi[i] : 0.0, pxx, pxy, pyy, pieta, tau, *p, L, nullptr);
    if (ok) ok[i] = r ? 1 : 0;
  }
  return 0;
}

void oracle_eos_Pne(const fivo_params* p, int64_t n, const double* T, const double* mu, double* P,
                    double* nq, double* e) {
  for (int64_t i = 0; i < n; ++i) eos_Pne(T[i], mu[i], *p, P + i, nq + i, e + i);
}

void oracle_eos_cs2(const fivo_params* p, int64_t n, const double* T, const double* mu, double* cs2) {
  for (int64_t i = 0; i < n; ++i) cs2[i] = eos_cs2(T[i], mu[i], *p);
}

void oracle_cons_to_prim(const fivo_params* p, int64_t n, double tau, const double* cons, const double* warm,
                         double* prim, uint8_t* ok, uint8_t* reason) {
  int maxit = p->primrec_maxit > 0 ? p->primrec_maxit : 80;
  double tol = p->primrec_tol > 0 ? p->primrec_tol : 1e-12;
#pragma omp parallel for
  for (int64_t i = 0; i < n; ++i) {
    const double* c = cons + 11 * i;
    double y0 = O_NAN, f0 = O_NAN, x0 = O_NAN, v0 = O_NAN;
    if (warm) { y0 = warm[4 * i]; f0 = warm[4 * i + 1]; x0 = warm[4 * i + 2]; v0 = warm[4 * i + 3]; }
    RecoveryOut r = cons_to_prim_2d(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[7], c[8], c[9], c[10],
                                    tau, *p, y0, f0, x0, v0, maxit, tol);
    double* o = prim + 7 * i;
    o[0] = r.T; o[1] = r.mu; o[2] = r.ux; o[3] = r.uy; o[4] = r.n; o[5] = r.e; o[6] = r.P;
    ok[i] = r.ok ? 1 : 0;
    if (reason) reason[i] = r.reason;
  }
}

void oracle_besselkx(int nu, int64_t n, const double* x, double* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = o_besselkx(nu, x[i]);
}
void oracle_exp(int64_t n, const double* x, double* out) { for (int64_t i = 0; i < n; ++i) out[i] = o_exp(x[i]); }
void oracle_log(int64_t n, const double* x, double* out) { for (int64_t i = 0; i < n; ++i) out[i] = o_log(x[i]); }
void oracle_pow4(int64_t n, const double* x, double* out) { for (int64_t i = 0; i < n; ++i) out[i] = o_pow4(x[i]); }
void oracle_hypot(int64_t n, const double* x, const double* y, double* out) {
  for (int64_t i = 0; i < n; ++i) out[i] = o_hypot(x[i], y[i]);
}

/* the consistent first moment's closed forms; in[] = ux, uy, ut, T, dxT, dyT, dtT, nux, nuy, n,
 * dn_dT, tau_n, Ds, hp, theta, ax, ay, dxux, dxuy, dyux, dyuy (21 values) */
void oracle_cfm_source(const double* in, uint32_t terms, double* sx, double* sy) {
  const double* v = in;
  cfm_source(v[0], v[1], v[2], v[3], v[4], v[5], v[6], v[7], v[8], v[9], v[10], v[11], v[12], v[13], v[14],
             v[15], v[16], v[17], v[18], v[19], v[20], terms, sx, sy);
}
void oracle_m2_source(const double* in44, uint32_t terms, double* out5) { m2_source(in44, terms, out5); }
void oracle_m2_coeffs(double T, double n, double tn, double Ds, double h, double m, double* out5) {
  m2_coeffs(T, n, tn, Ds, h, m, out5);
}
double oracle_m2_tauM(double T, double tn, double m) { return m2_tauM(T, tn, m); }
void oracle_m2_sigma_nu(const double* in18, double* out4) { m2_sigma_nu(in18, out4); }
void oracle_m2_rank1_traceless(const double* in7, double* out3) { m2_rank1_traceless(in7, out3); }

void oracle_cfm_h_hprime(const fivo_params* p, double T, double* h, double* hp) { cfm_h_hprime(T, *p, h, hp); }
double oracle_cfm_dn_dT(const fivo_params* p, double T, double n) { return cfm_dn_dT(T, n, *p); }
void oracle_diff_coeffs(const fivo_params* p, double T, double mu, double n, double* kappa, double* taun,
                        double* dN) {
  cfm_diff_coeffs(T, mu, n, *p, kappa, taun, dN);
}

/* record!(tau) of freeze_surface, freezeout2d.jl:94-115, on the context's last
 * primitives; arrays nx x ny (cell (a, b) at a*ny + b); *refroze accumulates */
void oracle_fo_record(void* h, double tau, double tau_prev, double T_fo, double* tau_fo, double* uxf,
                      double* uyf, double* Tprev, uint8_t* above, int64_t* refroze) {
  OCtx* c = (OCtx*)h;
  const Grid& g = c->g;
  for (int a = 0; a < g.Nx; ++a)
    for (int b = 0; b < g.Ny; ++b) {
      const int64_t k = (int64_t)a * g.Ny + b;
      const int64_t i = (int64_t)(g.ng + a) * g.Nytot + (g.ng + b);
      const double T = o_exp(c->w.yT[i]);
      if (T > T_fo) {
        if (!std::isnan(tau_fo[k])) *refroze += 1;
        above[k] = 1;
        tau_fo[k] = O_NAN;
      } else if (above[k] && std::isnan(tau_fo[k])) {
        const double Tp = Tprev[k];
        tau_fo[k] = (std::isnan(Tp) || Tp <= T_fo) ? tau : tau_prev + ((tau - tau_prev) * (Tp - T_fo)) / (Tp - T);
        uxf[k] = c->w.ux[i];
        uyf[k] = c->w.uy[i];
      }
      Tprev[k] = T;
    }
}

/* grad1, freezeout2d.jl:132-141 */
static double fo_grad1(const double* A, int ny, int a, int b, int dir, double dx) {
  const double lo = dir == 1 ? A[(a - 1) * ny + b] : A[a * ny + b - 1];
  const double hi = dir == 1 ? A[(a + 1) * ny + b] : A[a * ny + b + 1];
  const double cc = A[a * ny + b];
  if (!std::isnan(lo) && !std::isnan(hi)) return (hi - lo) / (2.0 * dx);
  if (!std::isnan(hi)) return (hi - cc) / dx;
  if (!std::isnan(lo)) return (cc - lo) / dx;
  return O_NAN;
}

/* pion_yield, freezeout2d.jl:144-190, in its loop order (a outer, summed in order);
 * prm = (T_fo, m, pt_lo, pt_hi, eta_max, f_yield), ngrid = (n_eta, n_pt, n_phi);
 * out = (N_boltzmann, N_bose, negative fraction) */
void oracle_pion_yield(int nx, int ny, double dx, const double* tau_fo, const double* uxf, const double* uyf,
                       const double* prm, const int* ngrid, double* out) {
  const double T_fo = prm[0], m = prm[1], pt_lo = prm[2], pt_hi = prm[3], eta_max = prm[4], fy = prm[5];
  const int n_eta = ngrid[0], n_pt = ngrid[1], n_phi = ngrid[2];
  const double dpt = (pt_hi - pt_lo) / (double)(n_pt - 1);
  const double dphi = (2.0 * M_PI) / (double)n_phi;
  const double deta = (2.0 * eta_max) / (double)(n_eta - 1);
  double tot = 0.0, totB = 0.0, negc = 0.0, posc = 0.0;
  for (int a = 1; a <= nx - 2; ++a) {
    double acc = 0.0, accB = 0.0, neg = 0.0, pos = 0.0;
    for (int b = 1; b <= ny - 2; ++b) {
      const int64_t k = (int64_t)a * ny + b;
      if (std::isnan(tau_fo[k])) continue;
      const double gx = fo_grad1(tau_fo, ny, a, b, 1, dx), gy = fo_grad1(tau_fo, ny, a, b, 2, dx);
      if (std::isnan(gx) || std::isnan(gy)) continue;
      const double tau = tau_fo[k], ux = uxf[k], uy = uyf[k];
      const double ut = std::sqrt((1.0 + (ux * ux)) + (uy * uy));
      for (int ipt = 0; ipt < n_pt; ++ipt) {
        const double pt = pt_lo + (double)ipt * dpt;
        const double mT = std::sqrt((pt * pt) + (m * m));
        for (int iphi = 0; iphi < n_phi; ++iphi) {
          const double phi = (double)iphi * dphi;
          const double px = pt * std::cos(phi), py = pt * std::sin(phi);
          for (int ie = 0; ie < n_eta; ++ie) {
            const double eta = -eta_max + (double)ie * deta;
            const double ch = std::cosh(eta);
            const double dSp = tau * (((mT * ch) - (gx * px)) - (gy * py));
            const double Es = (((ut * mT) * ch) - (ux * px)) - (uy * py);
            const double x = Es / T_fo;
            const double fB = std::exp(-x);
            const double fb = x > 1e-8 ? 1.0 / (std::exp(x) - 1.0) : 0.0;
            const double w = (((((dSp * pt) * dpt) * dphi) * deta) * dx) * dx;
            acc += w * fB;
            accB += w * fb;
            if (dSp < 0.0) neg += -(w * fB); else pos += w * fB;
          }
        }
      }
    }
    tot += acc; totB += accB; negc += neg; posc += pos;
  }
  const double pref = fy / std::pow((2.0 * M_PI) * 0.1973269804, 3);
  out[0] = pref * tot;
  out[1] = pref * totB;
  out[2] = negc / std::max(posc + negc, 1e-30);
}

}  /* extern "C" */
