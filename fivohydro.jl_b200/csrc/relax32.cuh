/*
 * relax32.cuh — the relaxation (relax_dissipative_2d!, src2d/dissipation2d.jl:293-705)
 * with its sources in FP32: the kinematics (theta, a^mu and the velocity gradients),
 * the Navier-Stokes targets, the projected-derivative and upwind-advection terms,
 * the second-order couplings and the consistent first moment's sources are formed in
 * FP32. The stencil differences themselves are taken in FP64 and rounded once (the
 * temporal ones subtract values a step apart), the transport coefficients (EOS and
 * Bessel functions) and the backward-Euler update of each dissipative field stay
 * FP64, and so do the shear projection and its residual monitor.
 *
 * Used by FIVO_PRECISION_FP32 (fivo_ctx_set_precision) together with the FP32 face
 * pass; the operations are relax_cell's (kernels.cuh), in the same order.
 */
#pragma once
#include "kernels.cuh"

namespace fv {

__device__ __forceinline__ float posf(float x) { return x > 1e-30f ? x : 1e-30f; }
__device__ __forceinline__ float safe_inv32(float x) { return 1.0f / posf(x); }

struct Kin32 { float th, ax, ay, at, dxux, dxuy, dyux, dyuy; };

/* ns_shear_target_2d, src2d/dissipation2d.jl:181-192, in FP32 */
__device__ __forceinline__ void ns_shear32(float ux, float uy, float ut, float itau, const Kin32& k, float eta,
                                           float* xx, float* xy, float* yy) {
  const float third = k.th / 3.0f;
  const float sxx = (k.dxux + ux * k.ax) - third * (1.0f + ux * ux);
  const float syy = (k.dyuy + uy * k.ay) - third * (1.0f + uy * uy);
  const float sxy = (0.5f * (k.dxuy + k.dyux) + 0.5f * (ux * k.ay + uy * k.ax)) - third * (ux * uy);
  const float m2 = -2.0f * eta;
  *xx = m2 * sxx; *xy = m2 * sxy; *yy = m2 * syy;
  (void)ut; (void)itau;
}

/* pi_sigma_contractions_2d, src2d/hq_consistent_m2_2d.jl:201-210, in FP32 */
__device__ void pi_sigma32(float ux, float uy, float pxx, float pxy, float pyy, float peta, float sxx, float sxy,
                           float syy, float seta, float* ps, float* cxx, float* cxy, float* cyy) {
  const float ux2 = ux * ux, uy2 = uy * uy, ux3 = ux2 * ux, uy3 = uy2 * uy, ux4 = ux2 * ux2;
  const float opuy2 = 1.0f + uy2;
  const float u2 = (1.0f + ux2) + uy2;
  float num = 2.0f * pxy * sxy + pyy * syy + 2.0f * pxy * sxy * ux2 + 2.0f * pyy * syy * ux2 + pyy * syy * ux4 -
              2.0f * pxy * sxx * ux * uy - 2.0f * pyy * sxy * ux * uy - 2.0f * pxy * syy * ux * uy -
              2.0f * pyy * sxy * ux3 * uy - 2.0f * pxy * syy * ux3 * uy + 2.0f * pxy * sxy * uy2 +
              pyy * sxx * ux2 * uy2 + 4.0f * pxy * sxy * ux2 * uy2 - 2.0f * pxy * sxx * ux * uy3 +
              pxx * sxx * (opuy2 * opuy2) + peta * seta * (u2 * u2);
  num += pxx * ux * uy * (syy * ux * uy - 2.0f * sxy * opuy2);
  *ps = num / (u2 * u2);
  *cxx = (pxx * sxx + pxy * sxy) - ((pxx * ux + pxy * uy) * (sxx * ux + sxy * uy)) / u2;
  *cyy = (pxy * sxy + pyy * syy) - ((pxy * ux + pyy * uy) * (sxy * ux + syy * uy)) / u2;
  *cxy = (pyy * ((sxy + sxy * ux2) - sxx * ux * uy) + pxy * (((sxx + syy) + syy * ux2) - 2.0f * sxy * ux * uy + sxx * uy2) +
          pxx * ((sxy - syy * ux * uy) + sxy * uy2)) / (2.0f * u2);
}

/* vorticity_coupling_2d, src2d/hq_consistent_m2_2d.jl:442-468, in FP32 */
__device__ void vorticity32(float ux, float uy, float ut, float pxx, float pxy, float pyy, float ax, float ay,
                            float dtux, float dtuy, float dxux, float dxuy, float dyux, float dyuy, float* wxx,
                            float* wxy, float* wyy) {
  const float iu = safe_inv32(ut);
  const float at = (ux * ax + uy * ay) * iu;
  const float dxut = (ux * dxux + uy * dxuy) * iu, dyut = (ux * dyux + uy * dyuy) * iu;
  const float wtx = 0.5f * ((-dtux + ut * ax) - (dxut + ux * at));
  const float wty = 0.5f * ((-dtuy + ut * ay) - (dyut + uy * at));
  const float wxy_ = 0.5f * ((dxuy + ux * ay) - (dyux + uy * ax));
  const float tx = (ux * pxx + uy * pxy) * iu, ty = (ux * pxy + uy * pyy) * iu;
  const float Mxx = -tx * wtx - pxy * wxy_, Mxy = -tx * wty + pxx * wxy_;
  const float Myx = -ty * wtx - pyy * wxy_, Myy = -ty * wty + pxy * wxy_;
  *wxx = 2.0f * Mxx; *wxy = Mxy + Myx; *wyy = 2.0f * Myy;
}

template <int EOS>
__device__ __forceinline__ double relax_cell32(const DevParams& d, const DevState& Uq, const DevState& Uo,
                                               const DevPrims& w, const DevHist& h, double tau, double D,
                                               int do_relax, int do_project, long long i) {
  double rel_out = -1.0;
  const int ix = (int)(i / d.Nytot), iy = (int)(i % d.Nytot);
  const int ng = d.ng;
  const bool interior = ix >= ng && ix < ng + d.Nx && iy >= ng && iy < ng + d.Ny;
  const double* QNux = d.hasNu ? Uq.f[d.iNux] : nullptr;
  const double* QNuy = d.hasNu ? Uq.f[d.iNuy] : nullptr;
  const double* QPi = d.hasPi ? Uq.f[d.iPi] : nullptr;
  const double* QPixx = d.hasShear ? Uq.f[d.iPixx] : nullptr;
  const double* QPixy = d.hasShear ? Uq.f[d.iPixy] : nullptr;
  const double* QPiyy = d.hasShear ? Uq.f[d.iPiyy] : nullptr;
  const double* QPieta = d.hasShear ? Uq.f[d.iPieta] : nullptr;
  double v_nux = d.hasNu ? QNux[i] : 0.0, v_nuy = d.hasNu ? QNuy[i] : 0.0;
  double v_Pi = d.hasPi ? QPi[i] : 0.0;
  double v_pixx = d.hasShear ? QPixx[i] : 0.0, v_pixy = d.hasShear ? QPixy[i] : 0.0;
  double v_piyy = d.hasShear ? QPiyy[i] : 0.0, v_pieta = d.hasShear ? QPieta[i] : 0.0;
  const fivo_params& p = d.p;
  const double ux = w.ux[i], uy = w.uy[i];
  const double ut = utau(ux, uy);
  if (do_relax && interior && w.ok[i]) {
    const double invdx = 1.0 / d.dx, invdy = 1.0 / d.dy;
    const long long st = d.Nytot;
    const float uxf = (float)ux, uyf = (float)uy, utf = (float)ut;
    const long long jx = ux >= 0 ? i - st : i + st;
    const long long jy = uy >= 0 ? i - 1 : i + 1;
    /* the upwind difference in FP64, rounded once, the advection term in FP32 */
    auto upw = [&](const double* Q, double q0) {
      const double qx = Q[jx], qy = Q[jy];
      const float dqx = (float)(ux >= 0 ? (q0 - qx) * invdx : (qx - q0) * invdx);
      const float dqy = (float)(uy >= 0 ? (q0 - qy) * invdy : (qy - q0) * invdy);
      return uxf * dqx + uyf * dqy;
    };
    Kin32 k;
    {
      const double ix2 = 1.0 / (2.0 * d.dx), iy2 = 1.0 / (2.0 * d.dy);
      k.dxux = (float)((w.ux[i + st] - w.ux[i - st]) * ix2);
      k.dxuy = (float)((w.uy[i + st] - w.uy[i - st]) * ix2);
      k.dyux = (float)((w.ux[i + 1] - w.ux[i - 1]) * iy2);
      k.dyuy = (float)((w.uy[i + 1] - w.uy[i - 1]) * iy2);
      const double uxp = h.ux_prev[i], uyp = h.uy_prev[i];
      const bool have_prev = isfinite_(uxp) && isfinite_(uyp);
      const float dtux = have_prev ? (float)((ux - uxp) / D) : 0.0f;
      const float dtuy = have_prev ? (float)((uy - uyp) / D) : 0.0f;
      const float iut = safe_inv32(utf);
      k.th = ((uxf * dtux + uyf * dtuy) * iut + k.dxux + k.dyuy) + utf * (float)safe_inv(tau);
      k.ax = (utf * dtux + uxf * k.dxux) + uyf * k.dyux;
      k.ay = (utf * dtuy + uxf * k.dxuy) + uyf * k.dyuy;
      k.at = (uxf * k.ax + uyf * k.ay) * iut;
    }
    const double T = fx_exp(w.yT[i]), mu = w.mu[i], n = w.n[i], en = w.e[i], P = w.P[i];
    const double s_ent = eos_entropy(T, mu, n, en, P);
    /* ---- bulk ---- */
    if (p.enable_bulk && d.hasPi) {
      double Pin = v_Pi;
      double zeta = 0.0, tPi = 0.0;
      if (p.bulk_kind != FIVO_BULK_ZERO) {
        double cs2 = eos_cs2<EOS>(T, d);
        double peak;
        if (p.bulk_kind == FIVO_BULK_LORENTZ) { double q = (T - 0.175) / 0.024; peak = p.zeta_over_s / (1.0 + (q * q)); }
        else { double q = (T - p.bulk_T0) / p.bulk_width; peak = p.zeta_over_s * fx_exp(-0.5 * (q * q)); }
        zeta = (peak * FV_INVFMGEV) * jmax(s_ent, 0.0);
        double sp = posden(s_ent);
        double Dl = jmax(fabs_((1.0 / 3.0) - cs2), 1e-8);
        tPi = (safe_div(zeta, ((posden(T) * sp) * posden(p.tauPi_coeff))) * (1.0 / (Dl * Dl))) + 0.1;
      }
      const float PiNS = -(float)zeta * k.th;
      double A = safe_div(tPi * ut, D);
      float adv = p.relax_advect_Pi ? -(float)tPi * upw(QPi, v_Pi) : 0.0f;
      double dPi = p.deltaPi_factor * tPi;
      if (p.lambda_Pi_pi_factor != 0.0 && p.enable_shear && d.hasShear) {
        float sxx, sxy, syy, ps, c1, c2, c3;
        ns_shear32(uxf, uyf, utf, 0.0f, k, -0.5f, &sxx, &sxy, &syy);
        const float seta = utf * (float)safe_inv(tau) - k.th / 3.0f;
        pi_sigma32(uxf, uyf, (float)v_pixx, (float)v_pixy, (float)v_piyy, (float)v_pieta, sxx, sxy, syy, seta, &ps,
                   &c1, &c2, &c3);
        adv = adv - (float)(p.lambda_Pi_pi_factor * tPi) * ps;
      }
      double num = ((A * Pin) + (double)PiNS) + (double)adv;
      Pin = dPi == 0.0 ? num / (A + 1.0) : num / jmax((A + 1.0) + (dPi * (double)k.th), 0.5 * (A + 1.0));
      Pin = jmax(Pin, -0.99 * jmax(P, 0.0));
      if (p.Pi_clip_factor > 0) { double cap = p.Pi_clip_factor * fabs_(P); Pin = jclamp(Pin, -cap, cap); }
      v_Pi = Pin;
    }
    /* ---- shear ---- */
    if (p.enable_shear && d.hasShear) {
      double eta = 0.0, tpi = 0.0, dpi = 0.0;
      if (p.shear_kind == FIVO_SHEAR_QGP) {
        eta = (jmax(p.eta_over_s, 0.0) * jmax(s_ent, 0.0)) * FV_INVFMGEV;
        double Ts = posden(T) * posden(s_ent);
        tpi = safe_div(eta, (Ts * posden(p.tauShear_coeff)));
        dpi = p.deltaShear_factor * tpi;
      } else {
        dpi = p.deltaShear_factor * 0.0;
      }
      double pixx = v_pixx, pixy = v_pixy, piyy = v_piyy;
      float nsxx, nsxy, nsyy;
      ns_shear32(uxf, uyf, utf, 0.0f, k, (float)eta, &nsxx, &nsxy, &nsyy);
      const float iut = safe_inv32(utf);
      const float pxxf = (float)pixx, pxyf = (float)pixy, pyyf = (float)piyy;
      const float tx = (uxf * pxxf + uyf * pxyf) * iut, ty = (uxf * pxyf + uyf * pyyf) * iut;
      const float cx = (-tx * k.at + pxxf * k.ax) + pxyf * k.ay;
      const float cy = (-ty * k.at + pxyf * k.ax) + pyyf * k.ay;
      double A = safe_div(tpi * ut, D);
      double den = jmax((A + 1.0) + (dpi * (double)k.th), 0.5 * (A + 1.0));
      const float pd = p.shear_projected_deriv ? (float)tpi : 0.0f;
      const bool ra = p.relax_advect_pi != 0;
      const float tpif = (float)tpi;
      float axx = ra ? -tpif * upw(QPixx, v_pixx) : 0.0f;
      float axy = ra ? -tpif * upw(QPixy, v_pixy) : 0.0f;
      float ayy = ra ? -tpif * upw(QPiyy, v_piyy) : 0.0f;
      if (p.terms & FIVO_TERM_SHEAR_VORTICITY) {
        const float dtux = ((k.ax - uxf * k.dxux) - uyf * k.dyux) * iut;
        const float dtuy = ((k.ay - uxf * k.dxuy) - uyf * k.dyuy) * iut;
        float wxx, wxy, wyy;
        vorticity32(uxf, uyf, utf, pxxf, pxyf, pyyf, k.ax, k.ay, dtux, dtuy, k.dxux, k.dxuy, k.dyux, k.dyuy, &wxx,
                    &wxy, &wyy);
        axx -= tpif * wxx; axy -= tpif * wxy; ayy -= tpif * wyy;
      }
      if (p.taupi_pi_factor != 0.0 || p.lambda_pi_Pi_factor != 0.0) {
        float sxx, sxy, syy;
        ns_shear32(uxf, uyf, utf, 0.0f, k, -0.5f, &sxx, &sxy, &syy);
        const float seta = utf * (float)safe_inv(tau) - k.th / 3.0f;
        if (p.taupi_pi_factor != 0.0) {
          const float tpp = (float)(p.taupi_pi_factor * tpi);
          float ps, cxx, cxy, cyy;
          pi_sigma32(uxf, uyf, pxxf, pxyf, pyyf, (float)v_pieta, sxx, sxy, syy, seta, &ps, &cxx, &cxy, &cyy);
          axx -= tpp * (cxx - ((1.0f + uxf * uxf) * ps) / 3.0f);
          axy -= tpp * (cxy - ((uxf * uyf) * ps) / 3.0f);
          ayy -= tpp * (cyy - ((1.0f + uyf * uyf) * ps) / 3.0f);
        }
        if (p.lambda_pi_Pi_factor != 0.0 && p.enable_bulk && d.hasPi) {
          const float lP = (float)((p.lambda_pi_Pi_factor * tpi) * v_Pi);
          axx -= lP * sxx; axy -= lP * sxy; ayy -= lP * syy;
        }
      }
      pixx = ((((A * pixx) + (double)nsxx) + (double)(pd * (2.0f * uxf * cx))) + (double)axx) / den;
      pixy = ((((A * pixy) + (double)nsxy) + (double)(pd * (uxf * cy + uyf * cx))) + (double)axy) / den;
      piyy = ((((A * piyy) + (double)nsyy) + (double)(pd * (2.0f * uyf * cy))) + (double)ayy) / den;
      if (p.pi_clip_factor > 0) {
        double cap = p.pi_clip_factor * fabs_(P);
        pixx = jclamp(pixx, -cap, cap); pixy = jclamp(pixy, -cap, cap); piyy = jclamp(piyy, -cap, cap);
      }
      double pe = project_traceless(ux, uy, ut, pixx, pixy, piyy);
      v_pixx = pixx; v_pixy = pixy; v_piyy = piyy; v_pieta = pe;
    }
    /* ---- charge ---- */
    if (p.enable_diff && d.hasNu) {
      double wv;
      {
        double lo = p.vacuum_n_lo, hi = p.vacuum_n_hi;
        wv = hi <= lo ? 1.0 : (n <= lo ? 0.0 : (n >= hi ? 1.0 : (n - lo) / (hi - lo)));
      }
      if (wv <= 0.0) { v_nux = 0.0; v_nuy = 0.0; }
      else {
        double Tm = posden(T);
        double alpha = mu / Tm;
        double kappa = (safe_div(p.kappa_coeff, Tm) * jmax(n, 0.0)) / FV_FMGEV;
        double tn;
        diff_tauN<EOS>(d, Tm, alpha, &tn);
        double dN = p.deltaN_factor * tn;
        double nux = v_nux, nuy = v_nuy;
        const float dxa = (float)alpha_grad(w.alpha, i, st, ix, d.Nxtot, ng, invdx);
        const float dya = (float)alpha_grad(w.alpha, i, 1, iy, d.Nytot, ng, invdy);
        double ap = h.alpha_prev[i];
        const float dta = isfinite_(ap) ? (float)((w.alpha[i] - ap) / D) : 0.0f;
        float nsx = 0.0f, nsy = 0.0f;
        if (p.terms & FIVO_TERM_NU_GRADALPHA) {
          const float Da = (utf * dta + uxf * dxa) + uyf * dya;
          nsx = -(float)kappa * (dxa + uxf * Da);
          nsy = -(float)kappa * (dya + uyf * Da);
        }
        if (p.consistent_fm) {
          const double Tp = h.T_prev[i];
          const float dtT = isfinite_(Tp) ? (float)((T - Tp) / D) : 0.0f;
          const float dxT = (float)((fx_exp(w.yT[i + st]) - fx_exp(w.yT[i - st])) / (2.0 * d.dx));
          const float dyT = (float)((fx_exp(w.yT[i + 1]) - fx_exp(w.yT[i - 1])) / (2.0 * d.dy));
          const float hp = (float)hq_hprime(T, d);
          const float dn_dT = (float)hq_dn_dT(T, n, d);
          const float Ds = (float)(safe_div(p.kappa_coeff, T) / FV_FMGEV);
          const float Tmf = (float)jmax(T, FV_T_MIN), nf = (float)n, tnf = (float)tn;
          const float nuxf = (float)nux, nuyf = (float)nuy;
          /* consistent_fm_source_2d, src2d/hq_consistent_firstmoment2d.jl:218-282, in FP32 */
          const float DT = (utf * dtT + uxf * dxT) + uyf * dyT;
          const float gTx = dxT + uxf * DT, gTy = dyT + uyf * DT;
          const float iut = safe_inv32(utf);
          const float nut = (uxf * nuxf + uyf * nuyf) * iut;
          const float dtux = ((k.ax - uxf * k.dxux) - uyf * k.dyux) * iut;
          const float dtuy = ((k.ay - uxf * k.dxuy) - uyf * k.dyuy) * iut;
          const float ngux = (nut * dtux + nuxf * k.dxux) + nuyf * k.dyux;
          const float nguy = (nut * dtuy + nuxf * k.dxuy) + nuyf * k.dyuy;
          const uint32_t t = p.terms;
          const float br = ((t & FIVO_TERM_FM_EXPANSION) ? tnf * k.th : 0.0f) +
                           ((t & FIVO_TERM_FM_DLNH) ? ((Ds / Tmf) * hp) * DT : 0.0f);
          const float pref = (Ds / Tmf) * (nf + Tmf * dn_dT);
          const float csx = (((t & FIVO_TERM_FM_GRADT) ? pref * gTx : 0.0f) +
                             ((t & FIVO_TERM_FM_INERTIAL) ? (tnf * nf) * k.ax : 0.0f)) +
                            ((t & FIVO_TERM_FM_NU_GRADU) ? tnf * ngux : 0.0f) + nuxf * br;
          const float csy = (((t & FIVO_TERM_FM_GRADT) ? pref * gTy : 0.0f) +
                             ((t & FIVO_TERM_FM_INERTIAL) ? (tnf * nf) * k.ay : 0.0f)) +
                            ((t & FIVO_TERM_FM_NU_GRADU) ? tnf * nguy : 0.0f) + nuyf * br;
          nsx -= csx; nsy -= csy;
        }
        nsx *= (float)wv; nsy *= (float)wv;
        if (p.vacuum_ramp_relax) { tn = wv * tn; dN = wv * dN; }
        const float nut = (uxf * (float)nux + uyf * (float)nuy) * safe_inv32(utf);
        const float nua = (-nut * k.at + (float)nux * k.ax) + (float)nuy * k.ay;
        double A = safe_div(tn * ut, D);
        double den = jmax((A + 1.0) + (dN * (double)k.th), 0.5 * (A + 1.0));
        const float pdn = p.diff_projected_deriv ? (float)tn : 0.0f;
        const float anx = p.relax_advect_nu ? -(float)tn * upw(QNux, v_nux) : 0.0f;
        const float any_ = p.relax_advect_nu ? -(float)tn * upw(QNuy, v_nuy) : 0.0f;
        nux = ((((A * nux) + (double)nsx) + (double)((pdn * uxf) * nua)) + (double)anx) / den;
        nuy = ((((A * nuy) + (double)nsy) + (double)((pdn * uyf) * nua)) + (double)any_) / den;
        if (p.nu_clip_factor > 0) {
          double cap = (p.nu_clip_factor * jmax(n, 0.0)) * ut;
          double mag = fx_hypot(nux, nuy);
          if (mag > cap && mag > FV_TINY) { double sc = cap / mag; nux *= sc; nuy *= sc; }
        }
        v_nux = nux; v_nuy = nuy;
      }
    }
  }
  if (do_project && d.hasShear && interior) {
    double rel = shear_residual_rel(ux, uy, ut, v_pixx, v_pixy, v_piyy, v_pieta);
    rel_out = rel;
    if (p.shear_constraint_project) v_pieta = project_traceless(ux, uy, ut, v_pixx, v_pixy, v_piyy);
  }
  if (d.hasNu) { Uo.f[d.iNux][i] = v_nux; Uo.f[d.iNuy][i] = v_nuy; }
  if (d.hasPi) Uo.f[d.iPi][i] = v_Pi;
  if (d.hasShear) {
    Uo.f[d.iPixx][i] = v_pixx; Uo.f[d.iPixy][i] = v_pixy; Uo.f[d.iPiyy][i] = v_piyy; Uo.f[d.iPieta][i] = v_pieta;
  }
  return rel_out;
}

template <int EOS>
__device__ __forceinline__ void relax32_body(const DevParams& d, const DevState& Uq, const DevState& Uo,
                                             const DevPrims& w, const DevHist& h, double tau, double D, int do_relax,
                                             int do_project, DevFlags* fl, long long i) {
  double rel = -1.0;
  if (i < d.Ntot) rel = relax_cell32<EOS>(d, Uq, Uo, w, h, tau, D, do_relax, do_project, i);
  if (do_project && d.hasShear) {
    double mx = rel > 0.0 ? rel : 0.0, sm = rel >= 0.0 ? rel : 0.0;
    for (int o = 16; o > 0; o >>= 1) {
      mx = jmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      sm += __shfl_xor_sync(0xffffffffu, sm, o);
    }
    if ((threadIdx.x & 31) == 0) {
      atomic_max_pos(&fl->shear_max_bits, mx);
      if (sm != 0.0) atomicAdd(&fl->shear_sum, sm);
    }
  }
}

template <int EOS>
__global__ void __launch_bounds__(128) k_relax32(DevParams d, DevState Uq, DevState Uo, DevPrims w, DevHist h,
                                                 double tau, double D, int do_relax, int do_project, DevFlags* fl) {
  relax32_body<EOS>(d, Uq, Uo, w, h, tau, D, do_relax, do_project, fl,
                    (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

}  // namespace fv
