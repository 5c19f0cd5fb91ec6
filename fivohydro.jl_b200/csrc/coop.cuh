/*
 * coop.cuh — cons_to_prim_2d! solved by one warp for one cell.
 *
 * The rare cells the warm-started recovery cannot finish quickly (a cold start
 * with its 3 x 60-step temperature bisection, a long or failing Newton, the
 * 200-step charge bisection) are sequential chains of EOS evaluations; run by
 * one thread, the longest chain sets the duration of the whole pass. Here all
 * 32 lanes of a warp work on one cell and evaluate, at once, the points the
 * sequential algorithm would evaluate one after another:
 *
 *   bisection     the 31 midpoints of the next five levels of the bisection
 *                 tree (each lane derives its node's interval with the same
 *                 halvings the sequential loop performs); the warp then walks
 *                 the tree with the ballot of the 31 predicates;
 *   Jacobian      the 2 x NU central-difference evaluations, one per lane;
 *   line search   the 12 step lengths alpha, alpha/2, ..., one per lane; the
 *                 first accepted one is taken, as the sequential loop would;
 *                 in the same round, 2 x NU more lanes evaluate the Jacobian
 *                 points of the next iteration around the full step, which is
 *                 the trial usually accepted, so an iteration costs one round.
 *
 * Every value a lane computes is computed with the same operations as in
 * recover_attempt (physics.cuh), and every decision is taken from the same
 * predicate values, so the result has the bits of the sequential algorithm.
 * The EOS memo is per lane; it only changes which evaluations are repeated.
 * All 32 lanes must call these functions together with the same arguments;
 * every lane returns the same result. A `stop` flag set by another warp ends an
 * attempt early with an unusable result: the warm and the cold attempt of a
 * cell run on two warps at once, and the cold one is abandoned when the warm
 * one succeeds (cons_to_prim_2d! would not have run it).
 */
#ifndef FIVO_COOP_CUH
#define FIVO_COOP_CUH

#include "physics.cuh"

namespace fv {

#define FV_FULL 0xffffffffu

__device__ __forceinline__ double shfl_d(double v, int src) { return __shfl_sync(FV_FULL, v, src); }

/* Warp-uniform read of a stop flag another warp may set (null: never stops). */
__device__ __forceinline__ bool stop_requested(const volatile int* stop) {
  if (!stop) return false;
  int v = 0;
  if ((threadIdx.x & 31) == 0) v = *stop;
  return __shfl_sync(FV_FULL, v, 0) != 0;
}

/* Interval of node (lane + 1) of a bisection tree rooted at (lo, hi), heap
 * order: the children of node k are 2k ("predicate true": hi = mid) and 2k + 1
 * ("false": lo = mid). */
__device__ __forceinline__ void bisect_node(int lane, double lo, double hi, double* a, double* b) {
  const int node = lane + 1;
  const int depth = 31 - __clz(node);
  for (int l = depth - 1; l >= 0; --l) {
    double mid = 0.5 * (lo + hi);
    if ((node >> l) & 1) lo = mid; else hi = mid;
  }
  *a = lo; *b = hi;
}

/* Follow `levels` levels of the tree with the predicates in `bal` (bit k =
 * predicate of node k + 1). Returns false if a level left (lo, hi) unchanged:
 * every later level would then repeat it, so the bisection has converged. */
__device__ __forceinline__ bool bisect_walk(unsigned bal, int levels, double* lo, double* hi) {
  int node = 1;
  for (int l = 0; l < levels; ++l) {
    double mid = 0.5 * (*lo + *hi);
    bool p = (bal >> (node - 1)) & 1u;
    double nlo = p ? *lo : mid, nhi = p ? mid : *hi;
    bool same = bits(nlo) == bits(*lo) && bits(nhi) == bits(*hi);
    *lo = nlo; *hi = nhi;
    if (same) return false;
    node = 2 * node + (p ? 0 : 1);
  }
  return true;
}

/* _invert_e_for_T (src2d/primrec2d.jl:300-314), 60 levels in 12 rounds of 5 */
template <int EOS>
__device__ double invert_e_warp(double e_target, double phi, const DevParams& d, int lane,
                                const volatile int* stop) {
  double lo = d.log_T_min, hi = d.log_T_solve_max;
  if (e_target <= 0.0) return lo;
  for (int it = 0; it < 60; it += 5) {
    if (stop_requested(stop)) break;
    double a, b;
    bisect_node(lane, lo, hi, &a, &b);
    bool pred = false;
    if (lane < 31) {
      double mid = 0.5 * (a + b);
      double Tm = fx_exp(mid);
      double Pm, em;
      eos_Pe_2d<EOS>(Tm, d.p.m_hq + (Tm * phi), d, &Pm, &em);
      pred = !isfinite_(em) || em > e_target;
    }
    unsigned bal = __ballot_sync(FV_FULL, pred);
    if (!bisect_walk(bal, 5, &lo, &hi)) break;
  }
  return 0.5 * (lo + hi);
}

/* seed_from_conserved_2d (src2d/primrec2d.jl:323-347) */
template <int EOS>
__device__ void seed_warp(double E, double Sx, double Sy, double phi, const DevParams& d, double* yT,
                          double* ux, double* uy, int lane, const volatile int* stop) {
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
    y = invert_e_warp<EOS>(ee, phi, d, lane, stop);
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

/* _solve_phi_bisect (src2d/primrec2d.jl:416-434), 200 levels in rounds of 5 */
template <int EOS>
__device__ void phi_bisect_warp(double D, double T, double ux, double uy, double nux, double nuy,
                                const DevParams& d, EosMemo& memo, double* phi, bool* ok, int lane) {
  double ut = utau(ux, uy);
  double target = D - nu_tau(ux, uy, ut, nux, nuy);
  double m = d.p.m_hq;
  if (!isfinite_(target) || target <= 0.0) { *phi = -FV_PHI_CAP; *ok = false; return; }
  double lo = -FV_PHI_CAP, hi = FV_PHI_CAP;
  for (int it = 0; it < 200; it += 5) {
    double a, b;
    bisect_node(lane, lo, hi, &a, &b);
    bool pred = false;
    if (lane < 31) {
      double mid = 0.5 * (a + b);
      double P, nm, en;
      eos_Pne_memo<EOS>(T, m + (T * mid), d, memo, &P, &nm, &en);
      pred = isfinite_(nm) && (nm * ut) > target;
    }
    unsigned bal = __ballot_sync(FV_FULL, pred);
    if (!bisect_walk(bal, 5, &lo, &hi)) break;
  }
  double f = 0.5 * (lo + hi);
  double P, nf, en;
  eos_Pne_memo<EOS>(T, m + (T * f), d, memo, &P, &nf, &en);
  *phi = f; *ok = isfinite_(nf);
}

__device__ __forceinline__ double pick4(const double x[4], int s) {
  return s == 0 ? x[0] : (s == 1 ? x[1] : (s == 2 ? x[2] : x[3]));
}

/* trial point of the line search: x + al * delta with the bounds of the unknowns
 * (src2d/primrec2d.jl:660-668) */
template <bool NCH>
__device__ __forceinline__ void trial_point(const double x[4], const double delta[4], double al, double yT_lo,
                                            double yT_hi, double xt[4]) {
  xt[0] = x[0]; xt[1] = x[1]; xt[2] = x[2]; xt[3] = x[3];
  if (NCH) {
    xt[0] = x[0] + al * delta[0]; xt[1] = x[1] + al * delta[1];
    xt[2] = x[2] + al * delta[2]; xt[3] = x[3] + al * delta[3];
  } else {
    xt[0] = x[0] + al * delta[0]; xt[2] = x[2] + al * delta[1]; xt[3] = x[3] + al * delta[2];
  }
  xt[0] = jclamp(xt[0], yT_lo, yT_hi);
  if (NCH) xt[1] = jclamp(xt[1], -FV_PHI_CAP, FV_PHI_CAP);
  xt[2] = jclamp(xt[2], -FV_U_CAP, FV_U_CAP);
  xt[3] = jclamp(xt[3], -FV_U_CAP, FV_U_CAP);
}

/* point j of the central differences at x: x +- h e_s for unknown k = j / 2
 * (+ for even j), h = 1e-6 max(1, |x_s|) (src2d/primrec2d.jl:605-618) */
template <bool NCH>
__device__ __forceinline__ void jac_point(const double x[4], int j, double xl[4]) {
  const int k = j >> 1;
  const int s = NCH ? k : (k == 0 ? 0 : k + 1);
  double xs = pick4(x, s);
  double h = 1e-6 * jmax(1.0, fabs_(xs));
  double xv = (j & 1) ? xs - h : xs + h;
  double a0 = x[0], a1 = x[1], a2 = x[2], a3 = x[3];
  xl[0] = s == 0 ? xv : a0; xl[1] = s == 1 ? xv : a1;
  xl[2] = s == 2 ? xv : a2; xl[3] = s == 3 ? xv : a3;
}

/* _cons_to_prim_attempt_2d! (src2d/primrec2d.jl:511-742), one warp */
template <int EOS, bool NCH>
__device__ __forceinline__ Recovery attempt_warp(const CellCons& c, const DevParams& d, double yT0, double phi0, double ux0,
                                 double uy0, int maxit, double tol, int lane, const volatile int* stop) {
  Recovery out;
  const double yT_lo = d.log_T_min, yT_hi = d.log_T_solve_max;
  const double m = d.p.m_hq;
  out.reason = PRR_UNSET; out.resnorm = nan_();
  const double D = c.D, Sx = c.Sx, Sy = c.Sy, E = c.E;
  if (is_vacuum(c)) return vacuum_recovery<EOS>(c, d);
  const int NU = NCH ? 4 : 3;
  EosMemo memo; memo.reset();
  double x[4], F[4], J[4][4], delta[4];
  x[1] = (NCH && isfinite_(phi0)) ? jclamp(phi0, -FV_PHI_CAP, FV_PHI_CAP) : 0.0;
  if (isfinite_(yT0) && isfinite_(ux0) && isfinite_(uy0)) {
    x[0] = jclamp(yT0, yT_lo, yT_hi);
    x[2] = jclamp(ux0, -FV_U_CAP, FV_U_CAP);
    x[3] = jclamp(uy0, -FV_U_CAP, FV_U_CAP);
  } else {
    double sy, sx_, syy;
    seed_warp<EOS>(E, Sx, Sy, x[1], d, &sy, &sx_, &syy, lane, stop);
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

  /* Fj: on lanes < 2 NU, the Jacobian evaluations at the current x (valid when
   * have_jac); jac_ok: all of them finite */
  double Fj[4] = {0.0, 0.0, 0.0, 0.0};
  bool have_jac = false, jac_ok = true;
  const unsigned spec_mask = ((1u << (2 * NU)) - 1u) << 12;
  for (int it = 1; it <= maxit; ++it) {
    double nrm = 0.0;
#pragma unroll
    for (int r = r_lo; r < 4; ++r) nrm = jmax(nrm, fabs_(F[r] * rs[r]));
    last_nrm = nrm;
    if (nrm < tol) { converged = true; out.reason = PRR_CONVERGED; break; }
    if (stop_requested(stop)) { out.ok = 0; out.reason = PRR_UNSET; return out; }
    /* ---- Jacobian: lane 2k evaluates x + h e_s, lane 2k+1 x - h e_s (s = unknown k) */
    if (!have_jac) {
      bool fin = true;
      double xl[4];
      jac_point<NCH>(x, lane & 7, xl);
      if (lane < 2 * NU) {
        evalF<EOS, NCH>(Fj, xl, c, d, memo);
        fin = finite4(Fj);
      }
      jac_ok = __all_sync(FV_FULL, fin);
    }
    if (!jac_ok) { out.reason = PRR_NONFINITE_JACOBIAN; break; }
    /* 1 / (2h) of column k on lane k: independent IEEE divisions do not overlap
     * within a lane, across lanes they cost one */
    double inv2h_l;
    {
      const int k = lane & 3;
      const int s = NCH ? k : (k == 0 ? 0 : k + 1);
      double h = 1e-6 * jmax(1.0, fabs_(pick4(x, s)));
      inv2h_l = 1.0 / (2.0 * h);
    }
    /* lane 2k holds F(x + h e_k), lane 2k + 1 F(x - h e_k): the even lane forms
     * the difference from its partner's rows, then each entry is broadcast once */
    double dF[4];
#pragma unroll
    for (int r = 0; r < NU; ++r) {
      const int rr = NCH ? r : r + 1;
      dF[r] = Fj[rr] - __shfl_xor_sync(FV_FULL, Fj[rr], 1);
    }
#pragma unroll
    for (int k = 0; k < NU; ++k) {
      const double inv2h = shfl_d(inv2h_l, k);
#pragma unroll
      for (int r = 0; r < NU; ++r) {
        const int rr = NCH ? r : r + 1;
        J[r][k] = (shfl_d(dF[r], 2 * k) * inv2h) * rs[rr];
      }
    }
    double Fact[4];
#pragma unroll
    for (int r = 0; r < NU; ++r) {
      const int rr = NCH ? r : r + 1;
      delta[r] = 0.0;
      Fact[r] = F[rr] * rs[rr];
    }
    if (!solve_gauss<NU>(delta, J, Fact)) { out.reason = PRR_LINSOLVE_FAILED; break; }
    /* alpha = min(1, min over |delta_k| > 1 of 1 / |delta_k|) as the reference
     * takes it; a correctly rounded reciprocal is monotone, so the minimum of the
     * reciprocals is the reciprocal of the maximum: one division, same bits
     * (a NaN |delta_k| fails `> 1` in both forms, an infinite one gives 0) */
    double amax = 0.0;
#pragma unroll
    for (int k = 0; k < NU; ++k) {
      double ad = fabs_(delta[k]);
      if (ad > 1.0 && !(ad <= amax)) amax = ad;
    }
    const double alpha = amax > 1.0 ? 1.0 / amax : 1.0;
    /* ---- one round: lane l < 12 tries alpha * 2^-l (the line search); lanes
     * 12 .. 12 + 2 NU - 1 evaluate the Jacobian at the first trial point, which
     * the next iteration uses when that trial is the one accepted. The l
     * halvings of the sequential loop are exact while the result is normal,
     * which alpha >= 2^-1011 guarantees for l <= 11; below that the halvings are
     * repeated as written (warp-uniform). */
    double al = alpha * (lane < 12 ? from_bits((uint64_t)(1023 - lane) << 52) : 1.0);
    if (!(alpha >= 0x1p-1011)) {
      al = alpha;
      if (lane < 12)
        for (int q = 0; q < lane; ++q) al *= 0.5;
    }
    double xt[4];
    trial_point<NCH>(x, delta, al, yT_lo, yT_hi, xt);
    if (lane >= 12) {
      double xj[4];
      jac_point<NCH>(xt, (lane - 12) & 7, xj);
      xt[0] = xj[0]; xt[1] = xj[1]; xt[2] = xj[2]; xt[3] = xj[3];
    }
    double Ft[4] = {0.0, 0.0, 0.0, 0.0};
    bool acc = false, fspec = true;
    if (lane < 12 + 2 * NU) {
      evalF<EOS, NCH>(Ft, xt, c, d, memo);   /* one call site for the whole round */
      const bool fin = finite4(Ft);
      if (lane >= 12) fspec = fin;
      else if (fin) {
        double trial = 0.0;
#pragma unroll
        for (int r = r_lo; r < 4; ++r) trial = jmax(trial, fabs_(Ft[r] * rs[r]));
        acc = trial < nrm * (1.0 - (1e-4 * al));
      }
    }
    unsigned ab = __ballot_sync(FV_FULL, acc);
    unsigned fb = __ballot_sync(FV_FULL, fspec);
    const int src = ab ? (__ffs(ab) - 1) : 11;
    double Fs[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      x[q] = shfl_d(xt[q], src);
      Fs[q] = shfl_d(Ft[q], (lane + 12) & 31);
      F[q] = shfl_d(Ft[q], src);
    }
    if (!ab) { out.reason = PRR_LINESEARCH_FAILED; break; }
    have_jac = (src == 0);
    if (have_jac) {
#pragma unroll
      for (int q = 0; q < 4; ++q) Fj[q] = Fs[q];
      jac_ok = (fb & spec_mask) == spec_mask;
    }
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
      phi_bisect_warp<EOS>(D, T, ux, uy, c.nux, c.nuy, d, memo, &phb, &okb, lane);
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

/* cons_to_prim_2d! (src2d/primrec2d.jl:465-486), one warp */
template <int EOS, bool NCH>
__device__ Recovery recover_warp(const CellCons& c, const DevParams& d, double yT0, double phi0, double ux0,
                                 double uy0, int maxit, double tol, int lane) {
  /* one call site for both attempts keeps a single inlined copy of the solver */
  const bool warm = isfinite_(yT0) && isfinite_(ux0) && isfinite_(uy0);
  Recovery r;
  for (int a = 0; a < 2; ++a) {
    const bool first = a == 0;
    r = attempt_warp<EOS, NCH>(c, d, first ? yT0 : nan_(), first ? phi0 : nan_(), first ? ux0 : nan_(),
                               first ? uy0 : nan_(), maxit, tol, lane, nullptr);
    if (r.ok || r.reason == PRR_VACUUM || !warm) break;
  }
  return r;
}

}  // namespace fv
#endif
