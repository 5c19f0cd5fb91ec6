/*
 * kernels.cuh — CUDA kernels of the 2+1D stage (sm_100a, FP64).
 *
 * Data layout in HBM (structure of arrays): every state row a is a plane of
 * Ntot doubles, cell i = ix*Nytot + iy (y contiguous, so a warp covers 32
 * consecutive y cells and every plane access is a coalesced 256-byte stream).
 * Primitives, warm starts and history are planes of the same shape.
 *
 * Per RK stage (rhs_2d! + the stage combination + sanitize_stage_2d! +
 * state_ok_2d, src2d/timestepper2d.jl:113-140):
 *   k_bc          ghost frame of U_base               (apply_bc_2d!)
 *   k_primitive   Newton recovery, every cell          (_primitive_pass!)
 *   k_stage       per tile: MUSCL + prim->cons + HLLE on all faces touching
 *                 the tile (amax over every face, ghosts included), then for
 *                 each interior cell: divergence + Bjorken source, RK
 *                 combination, floors, S-E and nu bounds, admissibility
 *   k_bc          ghost frame of U_out
 * Relaxation (relax_dissipative_2d! + project_shear!): k_relax, one thread per
 * cell, reading the pre-relaxation dissipative planes and writing a second set.
 */
#ifndef FIVO_KERNELS_CUH
#define FIVO_KERNELS_CUH

#include "physics.cuh"
#include "coop.cuh"
#include "guess.cuh"

/* resident blocks of 128 threads per SM the recovery and face kernels are
 * compiled for (their register budget): measured optima, overridable */
#ifndef FV_FAST_MINB
#define FV_FAST_MINB 4
#endif
#ifndef FV_FACE_MINB
#define FV_FACE_MINB 8
#endif

namespace fv {

#define FV_MAXV 11   /* rows of the flow: conserved four + the medium's dissipative seven */
#define FV_MAXP 16   /* every row of a state: + the charm second moment's five */

struct DevState { double* f[FV_MAXP]; };

struct DevPrims {
  double *yT, *phi, *mu, *alpha, *ux, *uy, *P, *n, *e;
  uint8_t* ok;
};

struct DevHist {
  double *x0_yT, *x0_phi, *x0_ux, *x0_uy, *ux_prev, *uy_prev, *alpha_prev, *T_prev;
  double *nux_prev, *nuy_prev;   /* the charge current after the last relaxation (second moment) */
};

/* device-side flags and reductions, mirrored into pinned host memory */
struct DevFlags {
  unsigned long long amax_bits;   /* max over faces of max(|sL|,|sR|), as ordered bits */
  unsigned long long rep;         /* (first failing cell << 8) | reason                */
  long long nprimfail, nvacuum;
  long long nbad;                 /* inadmissible interior cells of the last stage     */
  unsigned long long shear_max_bits;
  double shear_sum;
  double sumD, maxu, minPtot;     /* end-of-run diagnostics                             */
  int status;                     /* nonzero: a device loop hit its cap                 */
  int pad;
  unsigned int qcount_p, qnext_p; /* deferred recoveries of the current pass           */
  unsigned int qcount_q, qnext_q; /* the learned retry's leftovers for the full recovery */
  unsigned int qcount_a, qnext_a; /* deferred admissibility inversions of the stage     */
  unsigned long long tot_p, tot_a;/* deferred cells summed over passes (kernel timing)   */
  /* Newton statistics, cumulative until reset (what & 32): updates and attempts of
   * the warm-started fast pass; of the learned guess (attempts, accepted); of the
   * warm attempts that follow a rejected learned guess */
  unsigned long long it_fast, n_fast, it_learn, n_learn, ok_learn, it_fb, n_fb;
};

__device__ __forceinline__ void atomic_max_pos(unsigned long long* a, double v) {
  /* v >= 0 and not NaN: the IEEE bit pattern orders like the value */
  if (v > 0.0) atomicMax(a, (unsigned long long)__double_as_longlong(v));
}

/* slot of layout row a in the flux vector (0..3 conserved, 4..10 dissipatives) */
__device__ __forceinline__ int slot_of(const DevParams& d, int a) {
  if (a < 4) return a;
  if (d.hasNu && a == d.iNux) return 4;
  if (d.hasNu && a == d.iNuy) return 5;
  if (d.hasPi && a == d.iPi) return 6;
  if (a == d.iPixx) return 7;
  if (a == d.iPixy) return 8;
  if (a == d.iPiyy) return 9;
  return 10;
}

/* the plane of flux slot s (slot_of inverted; -1 when the model has no such plane) */
__device__ __forceinline__ int plane_of(const DevParams& d, int s) {
  return s < 4 ? s : (s == 4 ? d.iNux : (s == 5 ? d.iNuy : (s == 6 ? d.iPi : (s == 7 ? d.iPixx :
         (s == 8 ? d.iPixy : (s == 9 ? d.iPiyy : d.iPieta))))));
}

__device__ __forceinline__ void load_dis(const DevParams& d, const DevState& U, long long i, double dis[7]) {
  dis[0] = d.hasNu ? U.f[d.iNux][i] : 0.0;
  dis[1] = d.hasNu ? U.f[d.iNuy][i] : 0.0;
  dis[2] = d.hasPi ? U.f[d.iPi][i] : 0.0;
  dis[3] = d.hasShear ? U.f[d.iPixx][i] : 0.0;
  dis[4] = d.hasShear ? U.f[d.iPixy][i] : 0.0;
  dis[5] = d.hasShear ? U.f[d.iPiyy][i] : 0.0;
  dis[6] = d.hasShear ? U.f[d.iPieta][i] : 0.0;
}

/* ---------------------------------------------------------------- boundary */

/* apply_bc_2d!, src2d/bc2d.jl:14-65. Both passes together leave every ghost
 * cell equal to U[clamp(ix), clamp(iy)] (outflow) or U[wrap(ix), wrap(iy)]
 * (periodic), which is what one thread per ghost cell writes. */
__device__ __forceinline__ void bc_body(const DevParams& d, const DevState& U, int bc, long long t) {
  const int ng = d.ng, Nx = d.Nx, Ny = d.Ny;
  const long long nframe = (long long)d.Nxtot * d.Nytot - (long long)Nx * Ny;
  if (t >= nframe) return;
  /* enumerate the ghost frame: rows ix < ng or ix >= ng+Nx fully, else the y edges */
  int ix, iy;
  long long full = (long long)ng * d.Nytot;
  if (t < full) { ix = (int)(t / d.Nytot); iy = (int)(t % d.Nytot); }
  else if (t < 2 * full) { t -= full; ix = ng + Nx + (int)(t / d.Nytot); iy = (int)(t % d.Nytot); }
  else {
    t -= 2 * full;
    int per = 2 * ng;
    ix = ng + (int)(t / per);
    int r = (int)(t % per);
    iy = r < ng ? r : ng + Ny + (r - ng);
  }
  int sx, sy;
  if (bc == FIVO_BC_PERIODIC) {
    sx = ix < ng ? ix + Nx : (ix >= ng + Nx ? ix - Nx : ix);
    sy = iy < ng ? iy + Ny : (iy >= ng + Ny ? iy - Ny : iy);
  } else {
    sx = ix < ng ? ng : (ix >= ng + Nx ? ng + Nx - 1 : ix);
    sy = iy < ng ? ng : (iy >= ng + Ny ? ng + Ny - 1 : iy);
  }
  long long dst = (long long)ix * d.Nytot + iy, src = (long long)sx * d.Nytot + sy;
  for (int a = 0; a < d.nv; ++a) U.f[a][dst] = U.f[a][src];
}

__global__ void k_bc(DevParams d, DevState U, int bc) {
  bc_body(d, U, bc, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

/* ------------------------------------------------------- primitive recovery */

/* _primitive_pass!, src2d/rhs2d.jl:67-160, one thread per cell (ghosts too) */
template <int EOS, bool NCH>
__global__ void __launch_bounds__(128) k_primitive(DevParams d, DevState U, DevPrims w, DevHist h,
                                                   double tau, DevFlags* fl) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  CellCons c;
  c.D = safe_div(U.f[d.iDtau][i], tau);
  c.Sx = U.f[d.iSx][i]; c.Sy = U.f[d.iSy][i]; c.E = U.f[d.iE][i];
  double dis[7];
  load_dis(d, U, i, dis);
  c.nux = dis[0]; c.nuy = dis[1]; c.Pi = dis[2]; c.pixx = dis[3]; c.pixy = dis[4]; c.piyy = dis[5];
  c.pieta = dis[6];
  Recovery r = recover<EOS, NCH>(c, d, h.x0_yT[i], h.x0_phi[i], h.x0_ux[i], h.x0_uy[i],
                                 d.p.primrec_maxit, d.p.primrec_tol);
  double T = r.T, mu = r.mu, ux = r.ux, uy = r.uy, n = r.n, en = r.e, P = r.P;
  if (!r.ok) {
    if (r.reason == PRR_VACUUM) atomicAdd((unsigned long long*)&fl->nvacuum, 1ULL);
    else {
      atomicAdd((unsigned long long*)&fl->nprimfail, 1ULL);
      atomicMin(&fl->rep, ((unsigned long long)i << 8) | r.reason);
    }
    T = FV_T_MIN; mu = 0.0; ux = 0.0; uy = 0.0;
    eos_Pne<EOS>(T, mu, d, &P, &n, &en);
    en = jmax(en, 0.0); n = 0.0;
  }
  double Tm = jmax(T, FV_T_MIN);
  double yT = fx_log(Tm);
  double phi = jclamp((mu - d.p.m_hq) / Tm, -FV_PHI_CAP, FV_PHI_CAP);
  w.yT[i] = yT; w.phi[i] = phi; w.mu[i] = mu; w.alpha[i] = mu / Tm;
  w.ux[i] = ux; w.uy[i] = uy; w.P[i] = P; w.n[i] = n; w.e[i] = en; w.ok[i] = r.ok;
  if (r.ok) { h.x0_yT[i] = yT; h.x0_phi[i] = phi; h.x0_ux[i] = ux; h.x0_uy[i] = uy; }
  else { double q = nan_(); h.x0_yT[i] = q; h.x0_phi[i] = q; h.x0_ux[i] = q; h.x0_uy[i] = q; }
}

/* ------------------------------------------------------------------ faces */

/* One face between cell i (left) and ip = i + st: reconstructed face states
 * (reconstruct_muscl_2d!), prim_to_cons with the first-order and vacuum-floor
 * fallbacks (_faces_2d!), HLLE (hlle_flux_2d!). Writes nv fluxes (layout order)
 * to Fh and returns max(|sL|, |sR|). k = 0-based index of the left cell along
 * the face normal, kmax = cells along it. */
template <int EOS, bool XDIR>
__device__ double face_flux(const DevParams& d, const DevState& U, const DevPrims& w, long long i,
                            long long st, int k, int kmax, double tau, const uint8_t* ffo, double* Fh) {
  const long long ip = i + st;
  const int ng = d.ng;
  double disL[7], disR[7];
  load_dis(d, U, i, disL);
  load_dis(d, U, ip, disR);
  bool forced = ffo != nullptr && (ffo[i] || ffo[ip]);
  bool good = false;
  Prim pL, pR;
  double ucL[4], ucR[4];
  bool floorL = false, floorR = false;
  if (!forced) {
    double l[4], r[4];
    const double* fld[4] = {w.yT, w.phi, w.ux, w.uy};
    bool first = (k + 1 <= ng) || (k + 1 >= kmax - ng);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double* v = fld[q];
      double vi = v[i], vp = v[ip];
      if (first) { l[q] = vi; r[q] = vp; continue; }
      double vm = v[i - st], vpp = v[ip + st];
      double si = mc_limiter(vi - vm, vp - vi);
      double sp = mc_limiter(vp - vi, vpp - vp);
      double a = vi + 0.5 * si;
      double b = vp - 0.5 * sp;
      l[q] = jclamp(a, jmin(jmin(vm, vi), vp), jmax(jmax(vm, vi), vp));
      r[q] = jclamp(b, jmin(jmin(vi, vp), vpp), jmax(jmax(vi, vp), vpp));
    }
    double TL = fx_exp(l[0]); double muL = d.p.m_hq + (TL * l[1]);
    double TR = fx_exp(r[0]); double muR = d.p.m_hq + (TR * r[1]);
    bool okL = prim_to_cons<EOS>(ucL, pL, TL, muL, l[2], l[3], disL, tau, d);
    bool okR = prim_to_cons<EOS>(ucR, pR, TR, muR, r[2], r[3], disR, tau, d);
    good = okL && okR && ucL[0] >= 0.0 && ucR[0] >= 0.0 && ucL[3] >= FV_E_FLOOR && ucR[3] >= FV_E_FLOOR;
  }
  if (!good) {
    double TLc = fx_exp(w.yT[i]), muLc = w.mu[i];
    double TRc = fx_exp(w.yT[ip]), muRc = w.mu[ip];
    bool okL = prim_to_cons<EOS>(ucL, pL, TLc, muLc, w.ux[i], w.uy[i], disL, tau, d);
    bool okR = prim_to_cons<EOS>(ucR, pR, TRc, muRc, w.ux[ip], w.uy[ip], disR, tau, d);
    if (!(okL && okR)) {
      /* _floor_prim_2d!, src2d/rhs2d.jl:259-268 */
      if (!okL) {
        floorL = true;
        ucL[0] = 0.0; ucL[1] = 0.0; ucL[2] = 0.0; ucL[3] = FV_E_FLOOR;
        pL.T = FV_T_MIN; pL.mu = 0.0; pL.ux = 0.0; pL.uy = 0.0; pL.n = 0.0; pL.e = FV_E_FLOOR; pL.P = 0.0;
        pL.nux = pL.nuy = pL.Pi = pL.pixx = pL.pixy = pL.piyy = pL.pieta = 0.0;
      }
      if (!okR) {
        floorR = true;
        ucR[0] = 0.0; ucR[1] = 0.0; ucR[2] = 0.0; ucR[3] = FV_E_FLOOR;
        pR.T = FV_T_MIN; pR.mu = 0.0; pR.ux = 0.0; pR.uy = 0.0; pR.n = 0.0; pR.e = FV_E_FLOOR; pR.P = 0.0;
        pR.nux = pR.nuy = pR.Pi = pR.pixx = pR.pixy = pR.piyy = pR.pieta = 0.0;
      }
    }
  }
  if (floorL) pL.cs2 = eos_cs2<EOS>(FV_T_MIN, d);
  if (floorR) pR.cs2 = eos_cs2<EOS>(FV_T_MIN, d);
  double FL[11], FR[11];
  flux_cell<XDIR>(FL, pL, tau, d);
  flux_cell<XDIR>(FR, pR, tau, d);
  double lmL, lpL, lmR, lpR;
  wavespeeds<XDIR>(pL, XDIR ? pL.pixx : pL.piyy, &lmL, &lpL);
  wavespeeds<XDIR>(pR, XDIR ? pR.pixx : pR.piyy, &lmR, &lpR);
  double sL = jmin(lmL, lmR), sR = jmax(lpL, lpR);
  /* conserved columns of the two states incl. the stored dissipatives (zero when floored) */
  double cl[11], cr[11];
  cl[0] = ucL[0]; cl[1] = ucL[1]; cl[2] = ucL[2]; cl[3] = ucL[3];
  cr[0] = ucR[0]; cr[1] = ucR[1]; cr[2] = ucR[2]; cr[3] = ucR[3];
#pragma unroll
  for (int q = 0; q < 7; ++q) { cl[4 + q] = floorL ? 0.0 : disL[q]; cr[4 + q] = floorR ? 0.0 : disR[q]; }
  if (sL >= 0) {
    for (int a = 0; a < d.nvf; ++a) Fh[a] = FL[slot_of(d, a)];
  } else if (sR <= 0) {
    for (int a = 0; a < d.nvf; ++a) Fh[a] = FR[slot_of(d, a)];
  } else {
    double inv = 1.0 / ((sR - sL) + FV_TINY);
    for (int a = 0; a < d.nvf; ++a) {
      int s = slot_of(d, a);
      Fh[a] = (((sR * FL[s]) - (sL * FR[s])) + ((sR * sL) * (cr[s] - cl[s]))) * inv;
    }
  }
  return jmax(fabs_(sL), fabs_(sR));
}

/* --------------------------------------------------------------- the stage */

/* combination modes (src2d/timestepper2d.jl:122-130, 158-178) */
enum { COMB_EULER = 0, COMB_BLEND = 1, COMB_THIRD = 2, COMB_RHS_ONLY = 3 };

struct StageArgs {
  DevState Ub;      /* state the RHS is evaluated on (= U_in of the combination) */
  DevState Uold;    /* the step's entry state (blended stages)                    */
  DevState Uout;
  DevPrims w;
  const uint8_t* ffo;   /* force_first_order mask or null */
  uint8_t* bad;         /* per-cell inadmissible flag (interior)                   */
  double* dU;           /* optional: RHS planes (nv x Ntot), for fivo_rhs          */
  double tau, tau_state, dt, wold, wnew;
  int mode;
  DevFlags* fl;
};

#define ST_CX 8
#define ST_CY 32
#define ST_NFX ((ST_CX + 1) * ST_CY)
#define ST_NFY (ST_CX * (ST_CY + 1))

__device__ __forceinline__ double peff_of(const DevParams& d, const double u[FV_MAXV], double Pw) {
  double Peff = 0.0;
  if (isfinite_(Pw)) Peff = jmax(Pw, 0.0);
  if (d.hasPi) { double v = u[d.iPi]; if (isfinite_(v)) Peff += fabs_(v); }
  if (d.hasShear) {
    double v;
    v = u[d.iPixx]; if (isfinite_(v)) Peff += fabs_(v);
    v = u[d.iPixy]; if (isfinite_(v)) Peff += fabs_(v);
    v = u[d.iPiyy]; if (isfinite_(v)) Peff += fabs_(v);
    v = u[d.iPieta]; if (isfinite_(v)) Peff += fabs_(v);
  }
  return Peff;
}

/* enforce_floors_2d! + enforce_S_energy_constraint_2d! + enforce_nu_charge_constraint_2d!
 * for one interior cell (src2d/floors2d.jl:24-210). Pw = work.P (NaN if absent). */
__device__ __forceinline__ void sanitize_cell(const DevParams& d, double u[FV_MAXV], int ix, int iy, double tau_state,
                              double Pw, bool haveP, double Emin) {
  double Evac = jmax(Emin, d.E_vac_cut);
  double rdom = d.p.r_domain;
  bool blank = false, done = false;
  if (isfinite_(rdom)) {
    double x = d.xmin + (((double)(ix + 1 - d.ng)) - 0.5) * d.dx;
    double y = d.ymin + (((double)(iy + 1 - d.ng)) - 0.5) * d.dy;
    if ((x * x) + (y * y) > rdom * rdom) { u[d.iE] = Emin; blank = true; done = true; }
  }
  if (!done) {
    double Ei = u[d.iE];
    if (!isfinite_(Ei)) { u[d.iE] = Emin; blank = true; done = true; }
    else if (Ei < Evac) { u[d.iE] = Emin; blank = true; done = true; }
    else if (Ei <= 1e6 * Emin) blank = true;
  }
  if (blank) {
    u[d.iSx] = 0.0; u[d.iSy] = 0.0; u[d.iDtau] = 0.0;
    if (d.hasNu) { u[d.iNux] = 0.0; u[d.iNuy] = 0.0; }
    if (d.hasPi) u[d.iPi] = 0.0;
    if (d.hasShear) { u[d.iPixx] = 0.0; u[d.iPixy] = 0.0; u[d.iPiyy] = 0.0; u[d.iPieta] = 0.0; }
  }
  if (!done) {
    double Di = u[d.iDtau];
    if (!isfinite_(Di) || Di < 0.0) u[d.iDtau] = 0.0;
    if (!isfinite_(u[d.iSx])) u[d.iSx] = 0.0;
    if (!isfinite_(u[d.iSy])) u[d.iSy] = 0.0;
    for (int a = 4; a < d.nvf; ++a) if (!isfinite_(u[a])) u[a] = 0.0;
  }
  /* S-E bound */
  {
    double Ei = u[d.iE], Sx = u[d.iSx], Sy = u[d.iSy];
    if (isfinite_(Ei) && isfinite_(Sx) && isfinite_(Sy) && !(Ei <= 0)) {
      double Peff = peff_of(d, u, haveP ? Pw : nan_());
      double Smax = FV_CHI_SRE * (Ei + Peff);
      double aS = fx_hypot(Sx, Sy);
      if (aS > Smax) {
        double sc = Smax / (aS + FV_TINY);
        u[d.iSx] = Sx * sc; u[d.iSy] = Sy * sc;
      }
    }
  }
  /* nu bound */
  if (d.hasNu) {
    double Dt = u[d.iDtau] / tau_state;
    double nux = u[d.iNux], nuy = u[d.iNuy];
    if (isfinite_(Dt) && isfinite_(nux) && isfinite_(nuy)) {
      if (Dt <= 0.0) { u[d.iNux] = 0.0; u[d.iNuy] = 0.0; }
      else {
        double cap = 0.999 * Dt;
        double an = fx_hypot(nux, nuy);
        if (an > cap) {
          double sc = cap / (an + FV_TINY);
          u[d.iNux] = nux * sc; u[d.iNuy] = nuy * sc;
        }
      }
    }
  }
}

/* cell_admissible_2d, src2d/floors2d.jl:281-337 */
template <int EOS, bool NCH>
__device__ bool cell_admissible(const DevParams& d, const double u[FV_MAXV], double tau, bool okw,
                                double ux, double uy, double Pw) {
  const double Emin = FV_E_FLOOR;
  double E = u[d.iE], Sx = u[d.iSx], Sy = u[d.iSy], Dt = u[d.iDtau];
  if (!(isfinite_(E) && isfinite_(Sx) && isfinite_(Sy) && isfinite_(Dt))) return false;
  if (!(E >= Emin)) return false;
  if (!(Dt >= 0.0)) return false;
  for (int a = 4; a < d.nvf; ++a) if (!isfinite_(u[a])) return false;
  if (E <= 1e6 * Emin) return true;
  if (okw) {
    double ut = utau(ux, uy);
    double iu = safe_inv(ut);
    double vx = ux * iu, vy = uy * iu;
    if (!(isfinite_(vx) && isfinite_(vy))) return false;
    double lim = (1.0 - 1e-12) * (1.0 - 1e-12);
    if (!((vx * vx) + (vy * vy) < lim)) return false;
  }
  double Peff = peff_of(d, u, Pw);
  if (fx_hypot(Sx, Sy) <= ((FV_SR_MARGIN * FV_CHI_SRE) * (E + Peff))) return true;
  CellCons c;
  c.D = safe_div(Dt, tau); c.Sx = Sx; c.Sy = Sy; c.E = E;
  c.nux = d.hasNu ? u[d.iNux] : 0.0; c.nuy = d.hasNu ? u[d.iNuy] : 0.0;
  c.Pi = d.hasPi ? u[d.iPi] : 0.0;
  c.pixx = d.hasShear ? u[d.iPixx] : 0.0; c.pixy = d.hasShear ? u[d.iPixy] : 0.0;
  c.piyy = d.hasShear ? u[d.iPiyy] : 0.0; c.pieta = d.hasShear ? u[d.iPieta] : 0.0;
  Recovery r = recover<EOS, NCH>(c, d, nan_(), nan_(), nan_(), nan_(), 80, 1e-12);
  return r.ok || r.reason == PRR_VACUUM;
}

/* The charm second moment's rows in a stage (rows nvf..nv-1). flux_cell_2d! gives
 * them no entries and prim_to_cons_2d! never writes their face columns (zero), so
 * every branch of hlle_flux_2d! returns +0 for them, the assembly gives dU = +0
 * (src2d/rhs2d.jl:240-243) and the rows only pass through the stage combination,
 * with the same arithmetic as every other row. The floors and the admissibility
 * test do not read them (src2d/floors2d.jl). */
__device__ __forceinline__ void stage_m2_rows(const DevParams& d, const StageArgs& s, long long i) {
  const size_t N = (size_t)d.Ntot;
  for (int a = d.nvf; a < d.nv; ++a) {
    const double k = 0.0;
    if (s.dU) s.dU[(size_t)a * N + i] = k;
    const double ub = s.Ub.f[a][i];
    double u = ub;
    if (s.mode == COMB_EULER) u = ub + (s.dt * k);
    else if (s.mode == COMB_BLEND) u = (s.wold * s.Uold.f[a][i]) + (s.wnew * (ub + (s.dt * k)));
    else if (s.mode == COMB_THIRD) u = (s.Uold.f[a][i] + (2.0 * (ub + (s.dt * k)))) / 3.0;
    if (s.mode != COMB_RHS_ONLY) s.Uout.f[a][i] = u;
  }
}

/* rhs_2d! (faces, sources, assembly) fused with the stage combination, the
 * sanitiser and the admissibility test. One CTA per ST_CX x ST_CY tile of the
 * full (ghost-inclusive) grid. */
template <int EOS, bool NCH>
__global__ void __launch_bounds__(256) k_stage(DevParams d, StageArgs s) {
  extern __shared__ double sm[];
  double* Fx = sm;                              /* ST_NFX x nvf */
  double* Fy = sm + (size_t)ST_NFX * d.nvf;     /* ST_NFY x nvf */
  const int cx0 = blockIdx.x * ST_CX, cy0 = blockIdx.y * ST_CY;
  const int tid = threadIdx.x;
  double amax = 0.0;
  /* ---- faces ---- */
  for (int f = tid; f < ST_NFX + ST_NFY; f += blockDim.x) {
    if (f < ST_NFX) {
      int lx = f / ST_CY, ly = f % ST_CY;
      int ix = cx0 - 1 + lx, iy = cy0 + ly;
      if (ix < 0 || ix > d.Nxtot - 2 || iy >= d.Nytot) continue;
      long long i = (long long)ix * d.Nytot + iy;
      double a = face_flux<EOS, true>(d, s.Ub, s.w, i, d.Nytot, ix, d.Nxtot, s.tau, s.ffo,
                                      Fx + (size_t)f * d.nvf);
      if (a > amax) amax = a;
    } else {
      int g = f - ST_NFX;
      int lx = g / (ST_CY + 1), ly = g % (ST_CY + 1);
      int ix = cx0 + lx, iy = cy0 - 1 + ly;
      if (iy < 0 || iy > d.Nytot - 2 || ix >= d.Nxtot) continue;
      long long i = (long long)ix * d.Nytot + iy;
      double a = face_flux<EOS, false>(d, s.Ub, s.w, i, 1, iy, d.Nytot, s.tau, s.ffo,
                                       Fy + (size_t)g * d.nvf);
      if (a > amax) amax = a;
    }
  }
  /* block max of amax -> one atomic */
  for (int o = 16; o > 0; o >>= 1) amax = jmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  __shared__ double red[8];
  if ((tid & 31) == 0) red[tid >> 5] = amax;
  __syncthreads();
  if (tid == 0) {
    double m = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) m = jmax(m, red[k]);
    atomic_max_pos(&s.fl->amax_bits, m);
  }
  /* ---- cells ---- */
  const int lx = tid / ST_CY, ly = tid % ST_CY;
  const int ix = cx0 + lx, iy = cy0 + ly;
  const int ng = d.ng;
  if (ix < ng || ix >= ng + d.Nx || iy < ng || iy >= ng + d.Ny) return;
  const long long i = (long long)ix * d.Nytot + iy;
  const int nv = d.nvf;
  const double invdx = 1.0 / d.dx, invdy = 1.0 / d.dy;
  const double* fxR = Fx + (size_t)((lx + 1) * ST_CY + ly) * nv;
  const double* fxL = Fx + (size_t)(lx * ST_CY + ly) * nv;
  const double* fyT = Fy + (size_t)(lx * (ST_CY + 1) + ly + 1) * nv;
  const double* fyB = Fy + (size_t)(lx * (ST_CY + 1) + ly) * nv;
  double ub[FV_MAXV];
  for (int a = 0; a < nv; ++a) ub[a] = s.Ub.f[a][i];
  const double Pw = s.w.P[i];
  /* source_cell_2d!, src2d/fluxes2d.jl:166-177 (+ the advected-scalar divv terms) */
  double Sr[FV_MAXV];
  for (int a = 0; a < nv; ++a) Sr[a] = 0.0;
  {
    double itau = safe_inv(s.tau);
    double Pi = d.hasPi ? ub[d.iPi] : 0.0, pieta = d.hasShear ? ub[d.iPieta] : 0.0;
    Sr[d.iSx] = (-ub[d.iSx]) * itau;
    Sr[d.iSy] = (-ub[d.iSy]) * itau;
    Sr[d.iE] = (-((ub[d.iE] + (Pw + Pi)) + pieta)) * itau;
    bool an = d.hasNu && d.p.advect_nu, aP = d.hasPi && d.p.advect_Pi, ap = d.hasShear && d.p.advect_pi;
    if (an || aP || ap) {
      /* compute_divv_2d!, src2d/rhs2d.jl:29-41 */
      const long long ixm = i - d.Nytot, ixp = i + d.Nytot;
      double vxp = s.w.ux[ixp] * safe_inv(utau(s.w.ux[ixp], s.w.uy[ixp]));
      double vxm = s.w.ux[ixm] * safe_inv(utau(s.w.ux[ixm], s.w.uy[ixm]));
      double vyp = s.w.uy[i + 1] * safe_inv(utau(s.w.ux[i + 1], s.w.uy[i + 1]));
      double vym = s.w.uy[i - 1] * safe_inv(utau(s.w.ux[i - 1], s.w.uy[i - 1]));
      double divv = ((0.5 * (vxp - vxm)) * invdx) + ((0.5 * (vyp - vym)) * invdy);
      if (an) { Sr[d.iNux] += ub[d.iNux] * divv; Sr[d.iNuy] += ub[d.iNuy] * divv; }
      if (aP) Sr[d.iPi] += ub[d.iPi] * divv;
      if (ap) {
        Sr[d.iPixx] += ub[d.iPixx] * divv; Sr[d.iPixy] += ub[d.iPixy] * divv;
        Sr[d.iPiyy] += ub[d.iPiyy] * divv; Sr[d.iPieta] += ub[d.iPieta] * divv;
      }
    }
  }
  double u[FV_MAXV];
  for (int a = 0; a < nv; ++a) {
    double k = (((-(fxR[a] - fxL[a])) * invdx) - ((fyT[a] - fyB[a]) * invdy)) + Sr[a];
    if (s.dU) s.dU[(size_t)a * d.Ntot + i] = k;
    if (s.mode == COMB_EULER) u[a] = ub[a] + (s.dt * k);
    else if (s.mode == COMB_BLEND) u[a] = (s.wold * s.Uold.f[a][i]) + (s.wnew * (ub[a] + (s.dt * k)));
    else if (s.mode == COMB_THIRD) u[a] = (s.Uold.f[a][i] + (2.0 * (ub[a] + (s.dt * k)))) / 3.0;
  }
  if (d.hasM2) stage_m2_rows(d, s, i);
  if (s.mode == COMB_RHS_ONLY) return;
  sanitize_cell(d, u, ix, iy, s.tau_state, Pw, true, FV_E_FLOOR);
  bool adm = cell_admissible<EOS, NCH>(d, u, s.tau_state, s.w.ok[i] != 0, s.w.ux[i], s.w.uy[i], Pw);
  s.bad[i] = adm ? 0 : 1;
  if (!adm) atomicAdd((unsigned long long*)&s.fl->nbad, 1ULL);
  for (int a = 0; a < nv; ++a) s.Uout.f[a][i] = u[a];
}

/* expand_bad_2d! one radius step, src2d/floors2d.jl:369-383 */
__global__ void k_expand_bad(DevParams d, const uint8_t* bad, uint8_t* out) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  int ix = (int)(i / d.Nytot), iy = (int)(i % d.Nytot);
  uint8_t b = bad[i];
  if (ix >= d.ng && ix < d.ng + d.Nx && iy >= d.ng && iy < d.ng + d.Ny && !b)
    b = (bad[i - 1] || bad[i + 1] || bad[i - d.Nytot] || bad[i + d.Nytot]) ? 1 : 0;
  out[i] = b;
}

/* finalize_ic! floors/bounds without a pressure (main2D.jl:164-171), interior */
__global__ void k_finalize_ic(DevParams d, DevState U, double tau0) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)d.Nx * d.Ny) return;
  int ix = d.ng + (int)(t / d.Ny), iy = d.ng + (int)(t % d.Ny);
  long long i = (long long)ix * d.Nytot + iy;
  double u[FV_MAXV];
  for (int a = 0; a < d.nvf; ++a) u[a] = U.f[a][i];
  sanitize_cell(d, u, ix, iy, tau0, 0.0, false, FV_E_FLOOR);
  for (int a = 0; a < d.nvf; ++a) U.f[a][i] = u[a];
}

/* ------------------------------------------------------------- relaxation */

/* MC-limited face-reconstructed gradient of alpha at interior cell i
 * (compute_alpha_grad_fv_2d!, src2d/dissipation2d.jl:225-260) */
__device__ __forceinline__ double alpha_grad(const double* a, long long i, long long st, int k, int kmax,
                                             int ng, double invd) {
  double am2 = a[i - 2 * st], am1 = a[i - st], a0 = a[i], ap1 = a[i + st], ap2 = a[i + 2 * st];
  double slm = mc_limiter(am1 - am2, a0 - am1);
  double sl0 = mc_limiter(a0 - am1, ap1 - a0);
  double slp = mc_limiter(ap1 - a0, ap2 - ap1);
  /* face[i] (left cell k) and face[i-st] (left cell k-1) */
  double fi = (k + 1 <= ng || k + 1 >= kmax - ng) ? 0.5 * (a0 + ap1)
                                                   : 0.5 * ((a0 + (0.5 * sl0)) + (ap1 - (0.5 * slp)));
  double fm = (k <= ng || k >= kmax - ng) ? 0.5 * (am1 + a0)
                                          : 0.5 * ((am1 + (0.5 * slm)) + (a0 - (0.5 * sl0)));
  return (fi - fm) * invd;
}

/* transport coefficients at one cell (src/primitives.jl:56-108,
 * src2d/transport2d.jl:19-155) */
template <int EOS>
__device__ void diff_tauN(const DevParams& d, double Tm, double alpha, double* taun) {
  const double m = d.p.m_hq;
  const double DsT = d.p.kappa_coeff, tauD = d.p.tauN_coeff;
  double z = m / Tm;
  if (EOS == FIVO_EOS_LATTICE_HRG) {
    if (z <= 0.0) { *taun = 0.0; return; }
    double b1, b2;
    if (z >= 1.0e4) { b1 = fx_besselkx_asym(1, z); b2 = fx_besselkx_asym(2, z); }
    else { double k0, k1; fx_k01x(z, &k0, &k1); b1 = k1; b2 = k0 + (2.0 / z) * k1; }
    double b3 = b1 + ((4.0 / z) * b2);
    double b4 = b2 + ((6.0 / z) * b3);
    double b5 = b3 + ((8.0 / z) * b4);
    double ex = fx_exp(jclamp(alpha - z, -700.0, 700.0));
    double tauq = (((d.p.g_hq * (DsT / ((96.0 * d.pi2) * ((Tm * Tm) * Tm)))) * fx_pow5(m)) * ex) *
                  (((2.0 * b1) - (3.0 * b3)) + b5);
    /* _fluidum_single_hadron_normalization_2d at max(Tm, T_MIN) */
    double Tn = jmax(Tm, FV_T_MIN);
    double zn = m / Tn;
    double b2n = b2, exn = ex;
    if (Tn != Tm) { b2n = fx_besselkx(2, zn); exn = fx_exp(jclamp(alpha - zn, -700.0, 700.0)); }
    double norm = ((((d.p.g_hq * (Tn / (2.0 * d.pi2))) * (m * m)) * exn) * b2n) * d.fmgev3;
    if (fabs_(norm) <= FV_TINY) { *taun = 0.0; return; }
    double tn = (tauq / norm) * (FV_FMGEV * FV_FMGEV);
    if (!isfinite_(tn)) { *taun = 0.0; return; }
    *taun = jmax(tn, 0.0) * tauD;
    return;
  }
  if (z <= 0) { *taun = 0.0; return; }
  if (z > 50.0) {
    double K2a = fx_besselkx(2, z), K3a = fx_besselkx(3, z);
    double tg = fabs_(K2a) > FV_TINY ? (((DsT * z) * (K3a / K2a)) / Tm) : ((DsT * z) / Tm);
    *taun = jmin((tg / FV_FMGEV) * tauD, 1e20);
    return;
  }
  double K1x = fx_besselkx(1, z), K2x = fx_besselkx(2, z), K3x = fx_besselkx(3, z), K5x = fx_besselkx(5, z);
  double numerator = ((2.0 * K1x) - (3.0 * K3x)) + K5x;
  double denominator = jmax(fabs_(K2x), FV_TINY);
  double ratio = (numerator / denominator) * jsign(K2x == 0 ? 1.0 : K2x);
  double z3 = ((z * z) * z) / Tm;
  if (!isfinite_(z3) || z3 > 1e50) z3 = 1e50;
  double tg = ((DsT / 48.0) * z3) * ratio;
  if (!isfinite_(tg) || fabs_(tg) > 1e50) { *taun = 1e50 * jsign(tg); return; }
  *taun = (tg / FV_FMGEV) * tauD;
}

/* pi_sigma_contractions_2d, src2d/hq_consistent_m2_2d.jl:201-210 */
__device__ void pi_sigma(double ux, double uy, double pxx, double pxy, double pyy, double peta,
                         double sxx, double sxy, double syy, double seta,
                         double* ps, double* cxx, double* cxy, double* cyy) {
  double ux2 = ux * ux, uy2 = uy * uy, ux3 = (ux * ux) * ux, uy3 = (uy * uy) * uy, ux4 = fx_pow4(ux);
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

struct Kin { double th, ax, ay, at, dxux, dxuy, dyux, dyuy; };

/* ---- the consistent charm first moment (src2d/hq_consistent_firstmoment2d.jl) ---- */

/* hq_h_hprime_2d, :145-160: dh/dT of the enthalpy per particle h = m K3/K2 */
__device__ __forceinline__ double hq_hprime(double T, const DevParams& d) {
  const double Tm = jmax(T, FV_T_MIN);
  const double m = d.p.m_hq;
  const double z = m / Tm;
  if (z <= 0.0) return 0.0;
  const double K1 = fx_besselkx(1, z), K2 = fx_besselkx(2, z), K3 = fx_besselkx(3, z), K4 = fx_besselkx(4, z);
  if (fabs_(K2) <= FV_TINY) return 0.0;
  const double hpv = ((m * z) / Tm) * ((((K2 + K4) * K2) - ((K1 + K3) * K3))) / ((2.0 * K2) * K2);
  return isfinite_(hpv) ? hpv : 0.0;
}

/* hq_dn_dT_2d, :172-182: dn/dT at fixed alpha = (n/T)(3 + z K1/K2) */
__device__ __forceinline__ double hq_dn_dT(double T, double n, const DevParams& d) {
  const double Tm = jmax(T, FV_T_MIN);
  const double z = d.p.m_hq / Tm;
  if (z <= 0.0) return 0.0;
  const double K1 = fx_besselkx(1, z), K2 = fx_besselkx(2, z);
  if (fabs_(K2) <= FV_TINY) return 0.0;
  const double v = (n / Tm) * (3.0 + ((z * K1) / K2));
  return isfinite_(v) ? v : 0.0;
}

/* consistent_fm_source_2d, :218-282: the sources s^i (written on the left-hand side
 * of the charge row, so the relaxation subtracts them), each behind its Terms switch */
__device__ __forceinline__ void consistent_fm_source(double ux, double uy, double ut, double T, double dxT,
                                                     double dyT, double dtT, double nux, double nuy, double n,
                                                     double dn_dT, double tn, double Ds, double hp, const Kin& k,
                                                     uint32_t terms, double* sx, double* sy) {
  const double Tm = jmax(T, FV_T_MIN);
  const double DT = ((ut * dtT) + (ux * dxT)) + (uy * dyT);
  const double gTx = dxT + (ux * DT);
  const double gTy = dyT + (uy * DT);
  const double nut = nu_tau(ux, uy, ut, nux, nuy);
  const double dtux = ((k.ax - (ux * k.dxux)) - (uy * k.dyux)) * safe_inv(ut);
  const double dtuy = ((k.ay - (ux * k.dxuy)) - (uy * k.dyuy)) * safe_inv(ut);
  const double ngux = ((nut * dtux) + (nux * k.dxux)) + (nuy * k.dyux);
  const double nguy = ((nut * dtuy) + (nux * k.dxuy)) + (nuy * k.dyuy);
  const double expansion = (terms & FIVO_TERM_FM_EXPANSION) ? tn * k.th : 0.0;
  const double dlnh = (terms & FIVO_TERM_FM_DLNH) ? ((Ds / Tm) * hp) * DT : 0.0;
  const double br = expansion + dlnh;
  const double pref = (Ds / Tm) * (n + (Tm * dn_dT));
  *sx = ((((terms & FIVO_TERM_FM_GRADT) ? pref * gTx : 0.0) + ((terms & FIVO_TERM_FM_INERTIAL) ? (tn * n) * k.ax : 0.0)) +
         ((terms & FIVO_TERM_FM_NU_GRADU) ? tn * ngux : 0.0)) + (nux * br);
  *sy = ((((terms & FIVO_TERM_FM_GRADT) ? pref * gTy : 0.0) + ((terms & FIVO_TERM_FM_INERTIAL) ? (tn * n) * k.ay : 0.0)) +
         ((terms & FIVO_TERM_FM_NU_GRADU) ? tn * nguy : 0.0)) + (nuy * br);
}

/* ns_shear_target_2d, src2d/dissipation2d.jl:181-192 */
__device__ __forceinline__ void ns_shear(double ux, double uy, double ut, double tau, const Kin& k,
                                         double eta, double* xx, double* xy, double* yy, double* et) {
  double third = k.th / 3.0;
  double sxx = (k.dxux + (ux * k.ax)) - (third * (1.0 + (ux * ux)));
  double syy = (k.dyuy + (uy * k.ay)) - (third * (1.0 + (uy * uy)));
  double sxy = ((0.5 * (k.dxuy + k.dyux)) + (0.5 * ((ux * k.ay) + (uy * k.ax)))) - (third * (ux * uy));
  double seta = (ut * safe_inv(tau)) - third;
  double m2 = -2.0 * eta;
  *xx = m2 * sxx; *xy = m2 * sxy; *yy = m2 * syy; *et = m2 * seta;
}

/* vorticity_coupling_2d, src2d/hq_consistent_m2_2d.jl:442-468 */
__device__ void vorticity_coupling(double ux, double uy, double ut, double pxx, double pxy, double pyy,
                                   double ax, double ay, double dtux, double dtuy, double dxux, double dxuy,
                                   double dyux, double dyuy, double* wxx, double* wxy, double* wyy) {
  double iu = safe_inv(ut);
  double at = ((ux * ax) + (uy * ay)) * iu;
  double dxut = ((ux * dxux) + (uy * dxuy)) * iu;
  double dyut = ((ux * dyux) + (uy * dyuy)) * iu;
  double Atx = (-dtux) + (ut * ax), Axt = dxut + (ux * at);
  double Aty = (-dtuy) + (ut * ay), Ayt = dyut + (uy * at);
  double Axy = dxuy + (ux * ay), Ayx = dyux + (uy * ax);
  double wtx = 0.5 * (Atx - Axt), wty = 0.5 * (Aty - Ayt), wxy_ = 0.5 * (Axy - Ayx);
  PiC pc = shear_tensor(ux, uy, ut, pxx, pxy, pyy);
  double Mxx = ((-pc.tx) * wtx) - (pc.xy * wxy_);
  double Mxy = ((-pc.tx) * wty) + (pc.xx * wxy_);
  double Myx = ((-pc.ty) * wtx) - (pc.yy * wxy_);
  double Myy = ((-pc.ty) * wty) + (pc.xy * wxy_);
  *wxx = 2.0 * Mxx; *wxy = Mxy + Myx; *wyy = 2.0 * Myy;
}

/* ---- the consistent charm second moment (src2d/hq_consistent_m2_2d.jl) ---- */

/* hq_h_hprime_2d, src2d/hq_consistent_firstmoment2d.jl:145-160: h = m K3/K2 and dh/dT */
__device__ __forceinline__ void hq_h_hp(double T, const DevParams& d, double* h, double* hp) {
  const double Tm = jmax(T, FV_T_MIN);
  const double m = d.p.m_hq;
  const double z = m / Tm;
  *h = 0.0; *hp = 0.0;
  if (z <= 0.0) return;
  const double K1 = fx_besselkx(1, z), K2 = fx_besselkx(2, z), K3 = fx_besselkx(3, z), K4 = fx_besselkx(4, z);
  if (fabs_(K2) <= FV_TINY) return;
  const double hv = (m * K3) / K2;
  const double hpv = ((m * z) / Tm) * ((((K2 + K4) * K2) - ((K1 + K3) * K3))) / ((2.0 * K2) * K2);
  *h = isfinite_(hv) ? hv : 0.0;
  *hp = isfinite_(hpv) ? hpv : 0.0;
}

/* tauM_charm_2d, src2d/transport2d.jl:177-184: tau_M = tau_n K4 K2 / (2 K3^2) */
__device__ __forceinline__ double tauM_charm(double T, double tn, double m) {
  const double Tm = jmax(T, FV_T_MIN), z = m / Tm;
  const double K2 = fx_besselkx(2, z), K3 = fx_besselkx(3, z), K4 = fx_besselkx(4, z);
  if (fabs_(K3) <= FV_TINY) return 0.0;
  const double v = ((tn * K4) * K2) / ((2.0 * K3) * K3);
  return (isfinite_(v) && v > 0) ? v : 0.0;
}

/* sigma_nu_2d, src2d/hq_consistent_m2_2d.jl:171-182 (the generated closed forms, in
 * their order; the eta-eta entry is not read by the source and is not formed) */
__device__ __noinline__ void sigma_nu(double uxv, double uyv, double uT, double tau, double nux, double nuy,
                                      double dtnx, double dxnx, double dynx, double dtny, double dxny, double dyny,
                                      double dtux, double dxux, double dyux, double dtuy, double dxuy, double dyuy,
                                      double* oxx, double* oxy, double* oyy) {
  const double sxx = (((((tau * ((1.0 + (uxv * uxv)) + (uyv * uyv))) * (((((((2.0 * dtnx) * ((uxv * uxv) * uxv)) - (dtny * uyv)) + ((2.0 * dxnx) * uT)) - (dyny * uT)) - ((uxv * uxv) * (((dtny * uyv) - ((2.0 * dxnx) * uT)) + (dyny * uT)))) + (uxv * (((2.0 * dtnx) + ((3.0 * dtnx) * (uyv * uyv))) + (((3.0 * dynx) * uyv) * uT))))) + (nuy * ((((((((-1.0) - ((dtux * tau) * uxv)) - (uxv * uxv)) + (((2.0 * dtux) * tau) * ((uxv * uxv) * uxv))) * ((uyv * uyv) * uyv)) - ((((2.0 * tau) * uxv) * ((1.0 + (uxv * uxv)) * (1.0 + (uxv * uxv)))) * ((dtuy * uxv) + (dxuy * uT)))) - (((tau * ((-1.0) + (2.0 * (uxv * uxv)))) * (uyv * uyv)) * ((dtuy + (dtuy * (uxv * uxv))) - ((dyux * uxv) * uT)))) + (((1.0 + (uxv * uxv)) * uyv) * ((((-1.0) + (((2.0 * dtux) * tau) * ((uxv * uxv) * uxv))) + ((dyuy * tau) * uT)) + ((uxv * uxv) * (((-1.0) + (((2.0 * dxux) * tau) * uT)) - (((2.0 * dyuy) * tau) * uT)))))))) + (nux * ((((((fx_pow5(uxv) * ((-1.0) + (((2.0 * dtuy) * tau) * uyv))) + (((tau * uyv) * (1.0 + (uyv * uyv))) * ((dtux * uyv) + (dyux * uT)))) + (((2.0 * tau) * fx_pow4(uxv)) * (((-dtux) - (dtux * (uyv * uyv))) + ((dxuy * uyv) * uT)))) - (((2.0 * tau) * (uxv * uxv)) * ((((dtux + ((2.0 * dtux) * (uyv * uyv))) + (dtux * fx_pow4(uyv))) + ((((-dxuy) + dyux) * uyv) * uT)) + ((dyux * ((uyv * uyv) * uyv)) * uT)))) - (uxv * (((1.0 + ((dtuy * tau) * ((uyv * uyv) * uyv))) + (((2.0 * dxux) * tau) * uT)) + ((uyv * uyv) * ((1.0 + (((2.0 * dxux) * tau) * uT)) + ((dyuy * tau) * uT)))))) + (((uxv * uxv) * uxv) * ((((((2.0 * dtuy) * tau) * uyv) + (((2.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) - (2.0 * (1.0 + ((dxux * tau) * uT)))) + ((uyv * uyv) * (((-1.0) - (((2.0 * dxux) * tau) * uT)) + (((2.0 * dyuy) * tau) * uT)))))))) / ((3.0 * tau) * fx_pow15(((1.0 + (uxv * uxv)) + (uyv * uyv)))));
  const double sxy = (((((tau * ((1.0 + (uxv * uxv)) + (uyv * uyv))) * ((((((3.0 * dtny) * ((uxv * uxv) * uxv)) + (((3.0 * dynx) * (1.0 + (uyv * uyv))) * uT)) + (3.0 * (((dtnx * uyv) * (1.0 + (uyv * uyv))) + (dxny * uT)))) + ((uxv * uxv) * ((dtnx * uyv) + ((3.0 * dxny) * uT)))) + (uxv * (((3.0 * dtny) + (dtny * (uyv * uyv))) + (((dxnx + dyny) * uyv) * uT))))) - (nuy * (((((((((4.0 * dtuy) * tau) * fx_pow5(uxv)) * uyv) + ((((3.0 * dxuy) * tau) * uyv) * uT)) + ((((4.0 * tau) * fx_pow4(uxv)) * uyv) * ((-(dtux * uyv)) + (dxuy * uT)))) - (((tau * (uxv * uxv)) * uyv) * (((((-7.0) * dxuy) * uT) + (((2.0 * dtux) * uyv) * (3.0 + (2.0 * (uyv * uyv))))) + ((dyux * uT) * (3.0 + (4.0 * (uyv * uyv))))))) + (((uxv * uxv) * uxv) * ((((((10.0 * dtuy) * tau) * uyv) + (((4.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) + (((3.0 * dyuy) * tau) * uT)) + ((uyv * uyv) * ((2.0 - (((4.0 * dxux) * tau) * uT)) + (((4.0 * dyuy) * tau) * uT)))))) + (uxv * (((((((6.0 * dtuy) * tau) * uyv) + (((4.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) + (2.0 * fx_pow4(uyv))) + (((3.0 * dyuy) * tau) * uT)) + ((uyv * uyv) * ((2.0 - (((3.0 * dxux) * tau) * uT)) + (((4.0 * dyuy) * tau) * uT)))))))) + (nux * (((((((2.0 * fx_pow4(uxv)) * uyv) * ((-1.0) + (((2.0 * dtuy) * tau) * uyv))) - (((((3.0 * dxux) * tau) * uyv) * (1.0 + (uyv * uyv))) * uT)) - ((((4.0 * tau) * ((uxv * uxv) * uxv)) * uyv) * ((dtux + (dtux * (uyv * uyv))) - ((dxuy * uyv) * uT)))) + (((uxv * uxv) * uyv) * ((((((-2.0) + (((6.0 * dtuy) * tau) * uyv)) + (((4.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) - (((4.0 * dxux) * tau) * uT)) + (((3.0 * dyuy) * tau) * uT)) + ((uyv * uyv) * (((-2.0) - (((4.0 * dxux) * tau) * uT)) + (((4.0 * dyuy) * tau) * uT)))))) - ((tau * uxv) * (((dyux * uT) * ((3.0 + (7.0 * (uyv * uyv))) + (4.0 * fx_pow4(uyv)))) + (uyv * ((((6.0 * dtux) + ((10.0 * dtux) * (uyv * uyv))) + ((4.0 * dtux) * fx_pow4(uyv))) - (((3.0 * dxuy) * uyv) * uT)))))))) / ((6.0 * tau) * fx_pow15(((1.0 + (uxv * uxv)) + (uyv * uyv)))));
  const double syy = (((((tau * ((1.0 + (uxv * uxv)) + (uyv * uyv))) * ((((((((-(dtnx * uxv)) + ((2.0 * dtny) * uyv)) + (((3.0 * dtny) * (uxv * uxv)) * uyv)) - ((dtnx * uxv) * (uyv * uyv))) + ((2.0 * dtny) * ((uyv * uyv) * uyv))) + ((((3.0 * dxny) * uxv) * uyv) * uT)) - ((dxnx * (1.0 + (uyv * uyv))) * uT)) + (((2.0 * dyny) * (1.0 + (uyv * uyv))) * uT))) + (nux * ((((((uxv * uxv) * uxv) * ((((-1.0) - ((dtuy * tau) * uyv)) - (uyv * uyv)) + (((2.0 * dtuy) * tau) * ((uyv * uyv) * uyv)))) - ((((2.0 * tau) * uyv) * ((1.0 + (uyv * uyv)) * (1.0 + (uyv * uyv)))) * ((dtux * uyv) + (dyux * uT)))) - (((tau * (uxv * uxv)) * ((-1.0) + (2.0 * (uyv * uyv)))) * ((dtux + (dtux * (uyv * uyv))) - ((dxuy * uyv) * uT)))) + ((uxv * (1.0 + (uyv * uyv))) * ((((-1.0) + (((2.0 * dtuy) * tau) * ((uyv * uyv) * uyv))) + ((dxux * tau) * uT)) + ((uyv * uyv) * (((-1.0) - (((2.0 * dxux) * tau) * uT)) + (((2.0 * dyuy) * tau) * uT)))))))) + (nuy * ((((((((-1.0) + (((2.0 * dtux) * tau) * uxv)) * fx_pow5(uyv)) + (((tau * uxv) * (1.0 + (uxv * uxv))) * ((dtuy * uxv) + (dxuy * uT)))) + (((2.0 * tau) * fx_pow4(uyv)) * (((-dtuy) - (dtuy * (uxv * uxv))) + ((dyux * uxv) * uT)))) - (((2.0 * tau) * (uyv * uyv)) * ((((dtuy + ((2.0 * dtuy) * (uxv * uxv))) + (dtuy * fx_pow4(uxv))) + (((dxuy - dyux) * uxv) * uT)) + ((dxuy * ((uxv * uxv) * uxv)) * uT)))) + (((uyv * uyv) * uyv) * ((((((2.0 * dtux) * tau) * uxv) + (((2.0 * dtux) * tau) * ((uxv * uxv) * uxv))) + ((uxv * uxv) * (((-1.0) + (((2.0 * dxux) * tau) * uT)) - (((2.0 * dyuy) * tau) * uT)))) - (2.0 * (1.0 + ((dyuy * tau) * uT)))))) - (uyv * (((1.0 + ((dtux * tau) * ((uxv * uxv) * uxv))) + (((2.0 * dyuy) * tau) * uT)) + ((uxv * uxv) * ((1.0 + ((dxux * tau) * uT)) + (((2.0 * dyuy) * tau) * uT)))))))) / ((3.0 * tau) * fx_pow15(((1.0 + (uxv * uxv)) + (uyv * uyv)))));
  *oxx = sxx; *oxy = sxy; *oyy = syy;
}

/* rank1_traceless_2d, src2d/hq_consistent_m2_2d.jl:225-234 */
__device__ __forceinline__ void rank1_traceless(double Ax, double Ay, double Bx, double By, double ux, double uy,
                                                double ut, double* qxx, double* qxy, double* qyy) {
  const double u2 = ut * ut;
  const double tr = ((Ay * ((By + (By * (ux * ux))) - ((Bx * ux) * uy))) + (Ax * ((Bx - ((By * ux) * uy)) + (Bx * (uy * uy))))) / u2;
  *qxx = (Ax * Bx) - (((1.0 + (ux * ux)) * tr) / 3.0);
  *qyy = (Ay * By) - (((1.0 + (uy * uy)) * tr) / 3.0);
  *qxy = (((Ay * Bx) + (Ax * By)) / 2.0) - (((ux * uy) * tr) / 3.0);
}

/* consistent_m2_source_2d (src2d/hq_consistent_m2_2d.jl:247-404), split in two: the
 * parts that do not depend on the moment's own fields (the coefficients, the medium's
 * and the current's shear, the rank-1 drives), computed once per cell, and the rows
 * as functions of (pxx, pxy, pyy, peta, PiQ), evaluated five times (once, and once
 * per perturbed channel for the implicit coefficients). Every expression is the
 * single-function form's, in its order, so the bits are the same. */
struct M2Cell {
  double ux, uy, ut, tau, tM, Tm;
  double sxx, sxy, syy, seta;      /* the medium's shear (unit viscosity) */
  double snxx, snxy, snyy;         /* the current's shear */
  double geo, DlnT, etabar, ABr, etaQ, zetaQ;
  double qxx, qxy, qyy;            /* class (iv) */
  double tB1, tB4, tB5, tB6, tB7;  /* the trace row's field-independent terms, in order */
  double th, ax, ay, dtux, dtuy, dxux, dxuy, dyux, dyuy;
  uint32_t t;
};

__device__ __noinline__ void m2_cell_prepare(M2Cell& c, double ux, double uy, double ut, double tau, double T,
                                             double dxT, double dyT, double dtT, double nux, double nuy, double dta,
                                             double dxa, double dya, double thnu, double dtnux, double dtnuy,
                                             double dxnux, double dxnuy, double dynux, double dynuy, const Kin& k,
                                             double dtux, double dtuy, double n, double tn, double Ds, double h,
                                             double hp, double tM, double etaM, double m, uint32_t t) {
  c.ux = ux; c.uy = uy; c.ut = ut; c.tau = tau; c.tM = tM; c.t = t;
  c.th = k.th; c.ax = k.ax; c.ay = k.ay; c.dtux = dtux; c.dtuy = dtuy;
  c.dxux = k.dxux; c.dxuy = k.dxuy; c.dyux = k.dyux; c.dyuy = k.dyuy;
  const double Tm = jmax(T, FV_T_MIN);
  c.Tm = Tm;
  c.etaQ = etaM;
  c.zetaQ = (5.0 / 3.0) * c.etaQ;
  /* hq_m2_coeffs_2d, :125-142 */
  const double T2 = jmax(Tm, FV_T_MIN), z = m / T2;
  const double K2 = fx_besselkx(2, z), K3 = fx_besselkx(3, z), K4 = fx_besselkx(4, z);
  const double K5 = K3 + ((8.0 * K4) / z);
  const double dl = (fabs_(K4) > FV_TINY && fabs_(K3) > FV_TINY)
                        ? z * (((K3 + K5) / (2.0 * K4)) - ((K2 + K4) / (2.0 * K3))) : 0.0;
  c.etabar = ((tn * n) * T2) / 2.0;
  const double lama = (Ds * ((m * m) + ((6.0 * T2) * h))) / (2.0 * T2);
  const double Aco = (m * m) + ((5.0 * T2) * h);
  const double abr = fabs_(K3) > FV_TINY ? 5.0 + ((z * K2) / K3) : 5.0;
  const double dlnC = isfinite_(dl) ? dl : 0.0;
  c.ABr = isfinite_(abr) ? abr : 5.0;
  ns_shear(ux, uy, ut, tau, k, -0.5, &c.sxx, &c.sxy, &c.syy, &c.seta);
  const double anudot = ((k.ax * nux) + (k.ay * nuy)) - ((((k.ax * ux) + (k.ay * uy)) * ((nux * ux) + (nuy * uy))) / (ut * ut));
  sigma_nu(ux, uy, ut, tau, nux, nuy, dtnux, dxnux, dynux, dtnuy, dxnuy, dynuy, dtux, k.dxux, k.dyux, dtuy, k.dxuy,
           k.dyuy, &c.snxx, &c.snxy, &c.snyy);
  const double DT = ((ut * dtT) + (ux * dxT)) + (uy * dyT);
  c.DlnT = DT / Tm;
  const double DlnC = dlnC * c.DlnT;
  const double Da = ((ut * dta) + (ux * dxa)) + (uy * dya);
  c.geo = (t & FIVO_TERM_M2_EXPANSION) ? tM * (((5.0 / 3.0) * k.th) + DlnC) : 0.0;
  const double gTx = (h + (Tm * hp)) * (dxT + (ux * DT));
  const double gTy = (h + (Tm * hp)) * (dyT + (uy * DT));
  double qaxx, qaxy, qayy, qgxx, qgxy, qgyy;
  rank1_traceless(k.ax, k.ay, nux, nuy, ux, uy, ut, &qaxx, &qaxy, &qayy);
  rank1_traceless(nux, nuy, gTx, gTy, ux, uy, ut, &qgxx, &qgxy, &qgyy);
  const bool ia = t & FIVO_TERM_M2_ACCEL_NU, ig = t & FIVO_TERM_M2_NU_GRADTH;
  c.qxx = (ia ? (2.0 * lama) * qaxx : 0.0) + (ig ? (Ds / Tm) * qgxx : 0.0);
  c.qyy = (ia ? (2.0 * lama) * qayy : 0.0) + (ig ? (Ds / Tm) * qgyy : 0.0);
  c.qxy = (ia ? (2.0 * lama) * qaxy : 0.0) + (ig ? (Ds / Tm) * qgxy : 0.0);
  const bool i1 = t & FIVO_TERM_M2_NU_GRADIENT, i2 = t & FIVO_TERM_M2_BG_GRADU;
  c.tB1 = i1 ? c.zetaQ * thnu : 0.0;
  c.tB4 = c.etabar * (((t & FIVO_TERM_M2_BG_DLNT) ? c.ABr * c.DlnT : 0.0) + (i2 ? (5.0 / 3.0) * k.th : 0.0));
  c.tB5 = ia ? ((Ds * Aco) / (3.0 * Tm)) * anudot : 0.0;
  c.tB6 = ig ? ((5.0 / 6.0) * (Ds / Tm)) *
                   (((nux * gTx) + (nuy * gTy)) - ((((nux * ux) + (nuy * uy)) * ((gTx * ux) + (gTy * uy))) / (ut * ut)))
             : 0.0;
  c.tB7 = (t & FIVO_TERM_M2_BG_DALPHA) ? c.etabar * Da : 0.0;
}

/* the rows d_tau (pQxx, pQxy, pQyy, PiQ) at the given fields */
__device__ __noinline__ void m2_cell_rows(const M2Cell& c, double pxx, double pxy, double pyy, double peta,
                                          double PiQ, double out[4]) {
  const double ux = c.ux, uy = c.uy, tM = c.tM;
  const uint32_t t = c.t;
  double ps, cxx, cxy, cyy;
  pi_sigma(ux, uy, pxx, pxy, pyy, peta, c.sxx, c.sxy, c.syy, c.seta, &ps, &cxx, &cxy, &cyy);
  const bool i1 = t & FIVO_TERM_M2_NU_GRADIENT, i2 = t & FIVO_TERM_M2_BG_GRADU;
  const bool i3 = t & FIVO_TERM_M2_PI_SIGMA, i4 = t & FIVO_TERM_M2_PIQ_SIGMA;
  double sxx = ((((((pxx + (i1 ? (2.0 * c.etaQ) * c.snxx : 0.0)) + (c.geo * pxx)) +
                  (i3 ? (2.0 * tM) * (cxx - (((1.0 + (ux * ux)) * ps) / 3.0)) : 0.0)) +
                 (i4 ? ((2.0 * tM) * PiQ) * c.sxx : 0.0)) + (i2 ? (2.0 * c.etabar) * c.sxx : 0.0)) + c.qxx);
  double syy = ((((((pyy + (i1 ? (2.0 * c.etaQ) * c.snyy : 0.0)) + (c.geo * pyy)) +
                  (i3 ? (2.0 * tM) * (cyy - (((1.0 + (uy * uy)) * ps) / 3.0)) : 0.0)) +
                 (i4 ? ((2.0 * tM) * PiQ) * c.syy : 0.0)) + (i2 ? (2.0 * c.etabar) * c.syy : 0.0)) + c.qyy);
  double sxy = ((((((pxy + (i1 ? (2.0 * c.etaQ) * c.snxy : 0.0)) + (c.geo * pxy)) +
                  (i3 ? (2.0 * tM) * (cxy - (((ux * uy) * ps) / 3.0)) : 0.0)) +
                 (i4 ? ((2.0 * tM) * PiQ) * c.sxy : 0.0)) + (i2 ? (2.0 * c.etabar) * c.sxy : 0.0)) + c.qxy);
  if (t & FIVO_TERM_M2_VORTICITY) {
    double wxx, wxy, wyy;
    vorticity_coupling(ux, uy, c.ut, pxx, pxy, pyy, c.ax, c.ay, c.dtux, c.dtuy, c.dxux, c.dxuy, c.dyux, c.dyuy,
                       &wxx, &wxy, &wyy);
    sxx += tM * wxx; sxy += tM * wxy; syy += tM * wyy;
  }
  if (t & FIVO_TERM_M2_PROJECTOR) {
    const double at = ((ux * c.ax) + (uy * c.ay)) / c.ut;
    const PiC Q = shear_tensor(ux, uy, c.ut, pxx, pxy, pyy);
    const double cx = (((-Q.tx) * at) + (Q.xx * c.ax)) + (Q.xy * c.ay);
    const double cy = (((-Q.ty) * at) + (Q.xy * c.ax)) + (Q.yy * c.ay);
    sxx -= tM * ((2.0 * ux) * cx);
    sxy -= tM * ((ux * cy) + (uy * cx));
    syy -= tM * ((2.0 * uy) * cy);
  }
  const double sB = (((((((PiQ + c.tB1) + (c.geo * PiQ)) + (i3 ? ((2.0 / 3.0) * tM) * ps : 0.0)) + c.tB4) + c.tB5) +
                      c.tB6) + c.tB7);
  const double den = tM * c.ut;
  out[0] = (-sxx) / den; out[1] = (-sxy) / den; out[2] = (-syy) / den; out[3] = (-sB) / den;
}

/* relax_dissipative_2d! (src2d/dissipation2d.jl:293-705) fused with
 * project_shear! (main2D.jl:332-358). Reads the dissipative planes of Uq (the
 * pre-relaxation snapshot), writes them to Uo; the conserved planes are shared.
 * Every cell writes its dissipative rows: interior ok cells relaxed, the rest
 * copied. Then the shear projection of every interior cell. */
template <int EOS, bool M2>
__device__ __forceinline__ double relax_cell(const DevParams& d, const DevState& Uq, const DevState& Uo,
                                             const DevPrims& w, const DevHist& h, double tau, double D,
                                             int do_relax, int do_project, long long i) {
  double rel_out = -1.0;
  const int ix = (int)(i / d.Nytot), iy = (int)(i % d.Nytot);
  const int ng = d.ng;
  const bool interior = ix >= ng && ix < ng + d.Nx && iy >= ng && iy < ng + d.Ny;
  /* the dissipative rows as named values (a layout-indexed array would live in
   * local memory); rows a sector does not have stay 0 and are not stored */
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
  /* the charm second moment's rows pQxx, pQxy, pQyy, pQeta, PiQ (consecutive) */
  double v_pQ[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  if (M2) {
#pragma unroll
    for (int j = 0; j < 5; ++j) v_pQ[j] = Uq.f[d.iPQxx + j][i];
  }
  const fivo_params& p = d.p;
  const double ux = w.ux[i], uy = w.uy[i];
  const double ut = utau(ux, uy);
  if (do_relax && interior && w.ok[i]) {
    const double invdx = 1.0 / d.dx, invdy = 1.0 / d.dy;
    const long long st = d.Nytot;
    /* upwind neighbours: chosen by the sign of u, loaded before any use */
    const long long jx = ux >= 0 ? i - st : i + st;
    const long long jy = uy >= 0 ? i - 1 : i + 1;
    auto upw = [&](const double* Q, double q0) {
      double qx = Q[jx], qy = Q[jy];
      double dqx = ux >= 0 ? (q0 - qx) * invdx : (qx - q0) * invdx;
      double dqy = uy >= 0 ? (q0 - qy) * invdy : (qy - q0) * invdy;
      return (ux * dqx) + (uy * dqy);
    };
    /* kinematics_2d, src2d/dissipation2d.jl:141-167 */
    Kin k;
    {
      double ix2 = 1.0 / (2.0 * d.dx), iy2 = 1.0 / (2.0 * d.dy);
      k.dxux = (w.ux[i + st] - w.ux[i - st]) * ix2;
      k.dxuy = (w.uy[i + st] - w.uy[i - st]) * ix2;
      k.dyux = (w.ux[i + 1] - w.ux[i - 1]) * iy2;
      k.dyuy = (w.uy[i + 1] - w.uy[i - 1]) * iy2;
      double uxp = h.ux_prev[i], uyp = h.uy_prev[i];
      bool have_prev = isfinite_(uxp) && isfinite_(uyp);
      double dtux = have_prev ? (ux - uxp) / D : 0.0;
      double dtuy = have_prev ? (uy - uyp) / D : 0.0;
      double dtut = ((ux * dtux) + (uy * dtuy)) * safe_inv(ut);
      k.th = ((dtut + k.dxux) + k.dyuy) + (ut * safe_inv(tau));
      k.ax = ((ut * dtux) + (ux * k.dxux)) + (uy * k.dyux);
      k.ay = ((ut * dtuy) + (ux * k.dxuy)) + (uy * k.dyuy);
      k.at = ((ux * k.ax) + (uy * k.ay)) * safe_inv(ut);
    }
    const double T = fx_exp(w.yT[i]), mu = w.mu[i], n = w.n[i], en = w.e[i], P = w.P[i];
    /* local_thermo: entropy and (bulk only) cs2 */
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
      double PiNS = (-zeta) * k.th;
      double A = safe_div(tPi * ut, D);
      double adv = p.relax_advect_Pi ? (-tPi) * upw(QPi, v_Pi) : 0.0;
      double dPi = p.deltaPi_factor * tPi;
      if (p.lambda_Pi_pi_factor != 0.0 && p.enable_shear && d.hasShear) {
        double sxx, sxy, syy, se, ps, c1, c2, c3;
        ns_shear(ux, uy, ut, tau, k, -0.5, &sxx, &sxy, &syy, &se);
        pi_sigma(ux, uy, v_pixx, v_pixy, v_piyy, v_pieta, sxx, sxy, syy, se, &ps, &c1, &c2, &c3);
        adv = adv - ((p.lambda_Pi_pi_factor * tPi) * ps);
      }
      double num = ((A * Pin) + PiNS) + adv;
      Pin = dPi == 0.0 ? num / (A + 1.0) : num / jmax((A + 1.0) + (dPi * k.th), 0.5 * (A + 1.0));
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
      double pixx = v_pixx, pixy = v_pixy, piyy = v_piyy, pieta = v_pieta;
      double nsxx, nsxy, nsyy, nse;
      ns_shear(ux, uy, ut, tau, k, eta, &nsxx, &nsxy, &nsyy, &nse);
      PiC pc = shear_tensor(ux, uy, ut, pixx, pixy, piyy);
      double cx = (((-pc.tx) * k.at) + (pc.xx * k.ax)) + (pc.xy * k.ay);
      double cy = (((-pc.ty) * k.at) + (pc.xy * k.ax)) + (pc.yy * k.ay);
      double A = safe_div(tpi * ut, D);
      double den = jmax((A + 1.0) + (dpi * k.th), 0.5 * (A + 1.0));
      double pd = p.shear_projected_deriv ? tpi : 0.0;
      bool ra = p.relax_advect_pi != 0;
      double axx = ra ? (-tpi) * upw(QPixx, v_pixx) : 0.0;
      double axy = ra ? (-tpi) * upw(QPixy, v_pixy) : 0.0;
      double ayy = ra ? (-tpi) * upw(QPiyy, v_piyy) : 0.0;
      if (p.terms & FIVO_TERM_SHEAR_VORTICITY) {
        double iu = safe_inv(ut);
        double dtux = ((k.ax - (ux * k.dxux)) - (uy * k.dyux)) * iu;
        double dtuy = ((k.ay - (ux * k.dxuy)) - (uy * k.dyuy)) * iu;
        double wxx, wxy, wyy;
        vorticity_coupling(ux, uy, ut, pixx, pixy, piyy, k.ax, k.ay, dtux, dtuy, k.dxux, k.dxuy,
                           k.dyux, k.dyuy, &wxx, &wxy, &wyy);
        axx -= tpi * wxx; axy -= tpi * wxy; ayy -= tpi * wyy;
      }
      if (p.taupi_pi_factor != 0.0 || p.lambda_pi_Pi_factor != 0.0) {
        double sxx, sxy, syy, se;
        ns_shear(ux, uy, ut, tau, k, -0.5, &sxx, &sxy, &syy, &se);
        if (p.taupi_pi_factor != 0.0) {
          double tpp = p.taupi_pi_factor * tpi;
          double ps, cxx, cxy, cyy;
          pi_sigma(ux, uy, pixx, pixy, piyy, pieta, sxx, sxy, syy, se, &ps, &cxx, &cxy, &cyy);
          axx -= tpp * (cxx - (((1.0 + (ux * ux)) * ps) / 3.0));
          axy -= tpp * (cxy - (((ux * uy) * ps) / 3.0));
          ayy -= tpp * (cyy - (((1.0 + (uy * uy)) * ps) / 3.0));
        }
        if (p.lambda_pi_Pi_factor != 0.0 && p.enable_bulk && d.hasPi) {
          /* bulk already updated above, as in the reference (bulk runs first) */
          double lP = (p.lambda_pi_Pi_factor * tpi) * v_Pi;
          axx -= lP * sxx; axy -= lP * sxy; ayy -= lP * syy;
        }
      }
      pixx = ((((A * pixx) + nsxx) + (pd * ((2.0 * ux) * cx))) + axx) / den;
      pixy = ((((A * pixy) + nsxy) + (pd * ((ux * cy) + (uy * cx)))) + axy) / den;
      piyy = ((((A * piyy) + nsyy) + (pd * ((2.0 * uy) * cy))) + ayy) / den;
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
        double dxa = alpha_grad(w.alpha, i, st, ix, d.Nxtot, ng, invdx);
        double dya = alpha_grad(w.alpha, i, 1, iy, d.Nytot, ng, invdy);
        double ap = h.alpha_prev[i];
        double dta = isfinite_(ap) ? (w.alpha[i] - ap) / D : 0.0;
        double nsx = 0.0, nsy = 0.0;
        if (p.terms & FIVO_TERM_NU_GRADALPHA) {
          double Da = ((ut * dta) + (ux * dxa)) + (uy * dya);
          nsx = (-kappa) * (dxa + (ux * Da));
          nsy = (-kappa) * (dya + (uy * Da));
        }
        /* the consistent first moment (src2d/dissipation2d.jl:589-623), subtracted */
        if (p.consistent_fm) {
          const double Tp = h.T_prev[i];
          const double dtT = isfinite_(Tp) ? (T - Tp) / D : 0.0;
          const double dxT = (fx_exp(w.yT[i + st]) - fx_exp(w.yT[i - st])) / (2.0 * d.dx);
          const double dyT = (fx_exp(w.yT[i + 1]) - fx_exp(w.yT[i - 1])) / (2.0 * d.dy);
          const double hp = hq_hprime(T, d);
          const double dn_dT = hq_dn_dT(T, n, d);
          const double Ds = safe_div(p.kappa_coeff, T) / FV_FMGEV;
          double csx, csy;
          consistent_fm_source(ux, uy, ut, T, dxT, dyT, dtT, nux, nuy, n, dn_dT, tn, Ds, hp, k, p.terms, &csx, &csy);
          nsx -= csx; nsy -= csy;
        }
        nsx *= wv; nsy *= wv;
        if (p.vacuum_ramp_relax) { tn = wv * tn; dN = wv * dN; }
        double nut = nu_tau(ux, uy, ut, nux, nuy);
        double nua = (((-nut) * k.at) + (nux * k.ax)) + (nuy * k.ay);
        double A = safe_div(tn * ut, D);
        double den = jmax((A + 1.0) + (dN * k.th), 0.5 * (A + 1.0));
        double pdn = p.diff_projected_deriv ? tn : 0.0;
        double anx = p.relax_advect_nu ? (-tn) * upw(QNux, v_nux) : 0.0;
        double any_ = p.relax_advect_nu ? (-tn) * upw(QNuy, v_nuy) : 0.0;
        nux = ((((A * nux) + nsx) + ((pdn * ux) * nua)) + anx) / den;
        nuy = ((((A * nuy) + nsy) + ((pdn * uy) * nua)) + any_) / den;
        if (p.nu_clip_factor > 0) {
          double cap = (p.nu_clip_factor * jmax(n, 0.0)) * ut;
          double mag = fx_hypot(nux, nuy);
          if (mag > cap && mag > FV_TINY) { double sc = cap / mag; nux *= sc; nuy *= sc; }
        }
        v_nux = nux; v_nuy = nuy;
        /* the charm second moment: relax_charm_m2_cell_2d!, src2d/dissipation2d.jl:722-888,
         * handed the ramped tau_n and this cell's relaxed current */
        if (M2) {
          const double mq = p.transport_mass > 0.0 ? p.transport_mass : p.m_hq;
          const double tMq = tauM_charm(T, tn, mq);
          const bool have_hist = isfinite_(h.alpha_prev[i]) && isfinite_(h.T_prev[i]);
          if (tMq > 0.0 && have_hist) {
            const double nxp = h.nux_prev[i], nyp = h.nuy_prev[i];
            const double dtnx = isfinite_(nxp) ? (nux - nxp) / D : 0.0;
            const double dtny = isfinite_(nyp) ? (nuy - nyp) / D : 0.0;
            const double dxnx = ((QNux[i + st] - QNux[i - st]) * 0.5) * invdx;
            const double dxny = ((QNuy[i + st] - QNuy[i - st]) * 0.5) * invdx;
            const double dynx = ((QNux[i + 1] - QNux[i - 1]) * 0.5) * invdy;
            const double dyny = ((QNuy[i + 1] - QNuy[i - 1]) * 0.5) * invdy;
            const double uxp = h.ux_prev[i], uyp = h.uy_prev[i];
            const double dtux2 = isfinite_(uxp) ? (ux - uxp) / D : 0.0;
            const double dtuy2 = isfinite_(uyp) ? (uy - uyp) / D : 0.0;
            const double nut2 = nu_tau(ux, uy, ut, nux, nuy);
            const double thnu = ((((((((ux * dtnx) + (uy * dtny)) + (nux * dtux2)) + (nuy * dtuy2)) * safe_inv(ut)) -
                                   ((nut2 * ((ux * dtux2) + (uy * dtuy2))) * safe_inv(ut * ut))) + dxnx) + dyny) +
                                (nut2 * safe_inv(tau));
            const double Tp2 = h.T_prev[i];
            const double dtT2 = isfinite_(Tp2) ? (T - Tp2) / D : 0.0;
            const double dxT2 = ((fx_exp(w.yT[i + st]) - fx_exp(w.yT[i - st])) * 0.5) * invdx;
            const double dyT2 = ((fx_exp(w.yT[i + 1]) - fx_exp(w.yT[i - 1])) * 0.5) * invdy;
            double h2, hp2;
            hq_h_hp(T, d, &h2, &hp2);
            const double Ds2 = safe_div(p.kappa_coeff, T) / FV_FMGEV;
            M2Cell mc;
            m2_cell_prepare(mc, ux, uy, ut, tau, T, dxT2, dyT2, dtT2, nux, nuy, dta, dxa, dya, thnu, dtnx, dtny,
                            dxnx, dxny, dynx, dyny, k, dtux2, dtuy2, n, tn, Ds2, h2, hp2, tMq,
                            (jmax(T, FV_T_MIN) * tn) / 2.0, mq, p.terms);
            double pQxx = v_pQ[0], pQxy = v_pQ[1], pQyy = v_pQ[2], pQeta = v_pQ[3], PiQv = v_pQ[4];
            double s0[4], s1[4];
            m2_cell_rows(mc, pQxx, pQxy, pQyy, pQeta, PiQv, s0);
            const double A2 = safe_div(tMq * ut, D);
            const double dp = 1e-7 * jmax(jmax(jmax(jmax(1.0, fabs_(pQxx)), fabs_(pQxy)), fabs_(pQyy)), fabs_(PiQv));
            /* one perturbed evaluation per channel: each row's slope in its own field */
            double c[4];
            m2_cell_rows(mc, pQxx + dp, pQxy, pQyy, pQeta, PiQv, s1);
            c[0] = (((-(s1[0] - s0[0])) / dp) * tMq) * ut;
            m2_cell_rows(mc, pQxx, pQxy + dp, pQyy, pQeta, PiQv, s1);
            c[1] = (((-(s1[1] - s0[1])) / dp) * tMq) * ut;
            m2_cell_rows(mc, pQxx, pQxy, pQyy + dp, pQeta, PiQv, s1);
            c[2] = (((-(s1[2] - s0[2])) / dp) * tMq) * ut;
            m2_cell_rows(mc, pQxx, pQxy, pQyy, pQeta, PiQv + dp, s1);
            c[3] = (((-(s1[3] - s0[3])) / dp) * tMq) * ut;
            const bool ram = p.relax_advect_m2 != 0;
            const double amxx = ram ? (-tMq) * upw(Uq.f[d.iPQxx], pQxx) : 0.0;
            const double amxy = ram ? (-tMq) * upw(Uq.f[d.iPQxy], pQxy) : 0.0;
            const double amyy = ram ? (-tMq) * upw(Uq.f[d.iPQyy], pQyy) : 0.0;
            const double amB = ram ? (-tMq) * upw(Uq.f[d.iPiQ], PiQv) : 0.0;
            const double Rxx = ((((-tMq) * ut) * s0[0]) - (c[0] * pQxx)) - amxx;
            const double Rxy = ((((-tMq) * ut) * s0[1]) - (c[1] * pQxy)) - amxy;
            const double Ryy = ((((-tMq) * ut) * s0[2]) - (c[2] * pQyy)) - amyy;
            const double RB = ((((-tMq) * ut) * s0[3]) - (c[3] * PiQv)) - amB;
            const double half = 0.5 * (A2 + 1.0);
            pQxx = ((A2 * pQxx) - Rxx) / jmax(A2 + c[0], half);
            pQxy = ((A2 * pQxy) - Rxy) / jmax(A2 + c[1], half);
            pQyy = ((A2 * pQyy) - Ryy) / jmax(A2 + c[2], half);
            PiQv = ((A2 * PiQv) - RB) / jmax(A2 + c[3], half);
            pQeta = project_traceless(ux, uy, ut, pQxx, pQxy, pQyy);
            v_pQ[0] = pQxx; v_pQ[1] = pQxy; v_pQ[2] = pQyy; v_pQ[3] = pQeta; v_pQ[4] = PiQv;
          }
        }
      }
    }
  }
  /* project_shear!: residual monitor and pieta from tracelessness, interior cells */
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
  if (M2) {
#pragma unroll
    for (int j = 0; j < 5; ++j) Uo.f[d.iPQxx + j][i] = v_pQ[j];
    /* the current's history for the next relaxation's d_tau nu (dissipation2d.jl:354-359):
     * every cell's nu after this relaxation */
    if (do_relax && d.hasNu) { h.nux_prev[i] = v_nux; h.nuy_prev[i] = v_nuy; }
  }
  return rel_out;
}

/* relax_dissipative_2d! + project_shear! on every cell. The shear-residual
 * monitor (max and sum over interior cells) is reduced over the warp before
 * its atomics: one per warp instead of one per cell on a single address. */
template <int EOS, bool M2>
__device__ __forceinline__ void relax_body(const DevParams& d, const DevState& Uq, const DevState& Uo,
                                           const DevPrims& w, const DevHist& h, double tau, double D, int do_relax,
                                           int do_project, DevFlags* fl, long long i) {
  double rel = -1.0;
  if (i < d.Ntot) rel = relax_cell<EOS, M2>(d, Uq, Uo, w, h, tau, D, do_relax, do_project, i);
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

template <int EOS, bool M2>
__global__ void __launch_bounds__(128) k_relax(DevParams d, DevState Uq, DevState Uo, DevPrims w,
                                               DevHist h, double tau, double D, int do_relax,
                                               int do_project, DevFlags* fl) {
  relax_body<EOS, M2>(d, Uq, Uo, w, h, tau, D, do_relax, do_project, fl,
                      (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

/* --------------------------------------------------------------- utilities */

/* flag resets on the device (no host staging, so nothing races a queued copy).
 * what: 1 = per-pass counters, 2 = amax (set to amax_bits), 4 = shear monitor,
 * 8 = end-of-run diagnostics */
__device__ __forceinline__ void reset_flags_dev(DevFlags* fl, int what, unsigned long long amax_bits) {
  if (what & 1) {
    fl->nprimfail = 0; fl->nvacuum = 0; fl->rep = 0x7fffffffffffffffULL;
    fl->qcount_p = 0; fl->qnext_p = 0; fl->qcount_a = 0; fl->qnext_a = 0;
    fl->qcount_q = 0; fl->qnext_q = 0;
  }
  if (what & 64) fl->nbad = 0;      /* inadmissible cells: accumulate over a step's stages otherwise */
  if (what & 2) fl->amax_bits = amax_bits;
  if (what & 4) { fl->shear_max_bits = 0; fl->shear_sum = 0.0; }
  if (what & 8) { fl->sumD = 0.0; fl->maxu = 0.0; fl->minPtot = inf_(); }
  if (what & 16) { fl->tot_p = 0; fl->tot_a = 0; }
  if (what & 32) { fl->it_fast = fl->n_fast = fl->it_learn = fl->n_learn = fl->ok_learn = fl->it_fb = fl->n_fb = 0; }
  fl->status = 0;
}

__global__ void k_reset_flags(DevFlags* fl, int what, unsigned long long amax_bits) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  reset_flags_dev(fl, what, amax_bits);
}

__global__ void k_fill_nan(double* p, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = nan_();
}

/* run_sim_2d! history snapshot (main2D.jl:458-463): alpha_prev = alpha, T_prev = exp(yT) */
__device__ __forceinline__ void snapshot_cell(const DevPrims& w, const DevHist& h, long long i) {
  h.alpha_prev[i] = w.alpha[i];
  h.T_prev[i] = fx_exp(w.yT[i]);
}

__global__ void k_snapshot(DevParams d, DevPrims w, DevHist h) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  snapshot_cell(w, h, i);
}

__global__ void k_copy_planes(DevState dst, DevState src, int a0, int a1, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int a = a0; a < a1; ++a) dst.f[a][i] = src.f[a][i];
}

/* AoS (Julia U[a, i]) <-> SoA planes */
__global__ void k_aos_to_soa(DevState U, const double* aos, int nv, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nv) return;
  long long i = t / nv; int a = (int)(t % nv);
  U.f[a][i] = aos[t];
}
__global__ void k_soa_to_aos(DevState U, double* aos, int nv, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * nv) return;
  long long i = t / nv; int a = (int)(t % nv);
  aos[t] = U.f[a][i];
}

/* run_sim_2d! diagnostics over the interior (main2D.jl:421-426, 542-556) */
__global__ void k_diag(DevParams d, DevState U, DevPrims w, DevFlags* fl, int want_u, double* part) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double sD = 0.0, mu = 0.0, mp = inf_();
  if (t < (long long)d.Nx * d.Ny) {
    int ix = d.ng + (int)(t / d.Ny), iy = d.ng + (int)(t % d.Ny);
    long long i = (long long)ix * d.Nytot + iy;
    sD = U.f[d.iDtau][i];
    if (want_u) {
      mu = fx_hypot(w.ux[i], w.uy[i]);
      if (w.P[i] > 0) mp = w.P[i] + (d.hasPi ? U.f[d.iPi][i] : 0.0);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    sD += __shfl_xor_sync(0xffffffffu, sD, o);
    mu = jmax(mu, __shfl_xor_sync(0xffffffffu, mu, o));
    mp = jmin(mp, __shfl_xor_sync(0xffffffffu, mp, o));
  }
  if ((threadIdx.x & 31) == 0) {
    /* the sum is finished by k_sum_parts in a fixed order, so it repeats exactly */
    part[t >> 5] = sD;
    if (want_u) {
      atomic_max_pos((unsigned long long*)&fl->maxu, mu);
      /* minPtot: min over positive and negative values via a CAS loop */
      double old = fl->minPtot;
      while (mp < old) {
        unsigned long long o = __double_as_longlong(old);
        unsigned long long r = atomicCAS((unsigned long long*)&fl->minPtot, o, (unsigned long long)__double_as_longlong(mp));
        if (r == o) break;
        old = __longlong_as_double((long long)r);
      }
    }
  }
}

/* ---------------------------------------------------- MC-Glauber initial condition */

/* sum over point sources of w_k exp(-|x - x_k|^2 / 2 width^2) / (2 pi width^2) at every
 * cell centre (ghosts too), in the order of the point list */
__global__ void k_glauber_deposit(DevParams d, const double* pts, const double* wts, long long np,
                                  double width, double* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  const int ix = (int)(i / d.Nytot), iy = (int)(i % d.Nytot);
  const double x = d.xmin + (((double)(ix + 1 - d.ng)) - 0.5) * d.dx;
  const double y = d.ymin + (((double)(iy + 1 - d.ng)) - 0.5) * d.dy;
  const double inv = 1.0 / ((2.0 * width) * width);
  const double norm = 1.0 / (((2.0 * FX_PI) * width) * width);
  double acc = 0.0;
  for (long long k = 0; k < np; ++k) {
    const double dxp = x - pts[2 * k], dyp = y - pts[2 * k + 1];
    const double wk = wts ? wts[k] : 1.0;
    acc = acc + ((wk * norm) * fx_exp((-((dxp * dxp) + (dyp * dyp))) * inv));
  }
  out[i] = acc;
}

/* max over every cell (into *mx, as ordered bits of a non-negative double) and the
 * per-warp partial sums over the interior (for k_sum_parts) */
__global__ void k_glauber_reduce(DevParams d, const double* s, const double* nb, unsigned long long* mx,
                                 double* part) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double m = 0.0, sum = 0.0;
  if (t < d.Ntot) {
    m = s[t];
    const int ix = (int)(t / d.Nytot), iy = (int)(t % d.Nytot);
    if (ix >= d.ng && ix < d.ng + d.Nx && iy >= d.ng && iy < d.ng + d.Ny) sum = nb[t];
  }
  for (int o = 16; o > 0; o >>= 1) {
    m = jmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomic_max_pos(mx, m);
    part[t >> 5] = sum;
  }
}

/* T from e = s * ((e_peak - e_edge) / max s) + e_edge by 90-step bisection of the
 * light-sector e(T) in log T, and alpha = log(n_target / n(T, alpha = 0)) with
 * n_target = the binary part + n_edge, floored at alpha_min where not finite */
__global__ void k_glauber_fields(DevParams d, const double* s, const double* nb, const unsigned long long* mx,
                                 const double* interior, double e_peak, double e_edge, double n_edge,
                                 double tau0, double ncharm, double alpha_min, double* Tout, double* aout) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot) return;
  const double smax = __longlong_as_double((long long)*mx);
  const double e = (s[i] * ((e_peak - e_edge) / smax)) + e_edge;
  double lo = d.log_T_min, hi = d.log_T_solve_max;
  for (int it = 0; it < 90; ++it) {
    const double mid = 0.5 * (lo + hi);
    const double Tm = jmax(fx_exp(mid), FV_T_MIN);
    double Pl, dP;
    light_eos<3>(Tm, d, &Pl, &dP, nullptr);
    const double em = (-Pl) + (Tm * dP);
    if (em > e) hi = mid; else lo = mid;
  }
  const double T = jmax(fx_exp(0.5 * (lo + hi)), FV_T_MIN);
  const double I = ((*interior) * d.dx) * d.dy;   /* the interior sum of nb times dx dy */
  const double ntgt = (I > 0.0 ? nb[i] * (ncharm / (tau0 * I)) : 0.0) + n_edge;
  const double x = lhrg_x(T, d);
  double Pl, dP;
  light_eos<3>(T, d, &Pl, &dP, nullptr);
  double P0, n0, e0;
  lhrg_assemble(T, 0.0, d, x, Pl, (-Pl) + (T * dP), lhrg_K2(x), &P0, &n0, &e0);
  double a = fx_log(ntgt / n0);
  a = isfinite_(a) ? jmax(a, alpha_min) : alpha_min;
  Tout[i] = T;
  aout[i] = a;
}

/* sum of the per-warp partial sums of k_diag in a fixed order (one block) */
__global__ void k_sum_parts(const double* part, long long n, double* out) {
  __shared__ double red[256];
  double acc = 0.0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) acc += part[k];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = red[0];
}

/* one-shot helpers for the C ABI's batched entry points */
template <int EOS>
__global__ void k_set_cells(DevParams d, long long n, double tau, const double* T, const double* alpha,
                            const double* ux, const double* uy, const double* Pi, const double* pixx,
                            const double* pixy, const double* piyy, const double* nux, const double* nuy,
                            double* U, uint8_t* ok) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double vx = ux[i], vy = uy[i];
  double ut = utau(vx, vy);
  double pxx = pixx ? pixx[i] : 0.0, pxy = pixy ? pixy[i] : 0.0, pyy = piyy ? piyy[i] : 0.0;
  double pieta = project_traceless(vx, vy, ut, pxx, pxy, pyy);
  double dis[7] = {nux ? nux[i] : 0.0, nuy ? nuy[i] : 0.0, Pi ? Pi[i] : 0.0, pxx, pxy, pyy, pieta};
  double uc[4];
  Prim pr;
  bool r = prim_to_cons<EOS>(uc, pr, T[i], alpha[i] * T[i], vx, vy, dis, tau, d);
  if (r) {
    double* col = U + i * d.nv;
    col[d.iDtau] = uc[0]; col[d.iSx] = uc[1]; col[d.iSy] = uc[2]; col[d.iE] = uc[3];
    if (d.hasNu) { col[d.iNux] = dis[0]; col[d.iNuy] = dis[1]; }
    if (d.hasPi) col[d.iPi] = dis[2];
    if (d.hasShear) { col[d.iPixx] = dis[3]; col[d.iPixy] = dis[4]; col[d.iPiyy] = dis[5]; col[d.iPieta] = dis[6]; }
  }
  ok[i] = r ? 1 : 0;
}

template <int EOS>
__global__ void k_eos(DevParams d, long long n, const double* T, const double* mu, double* P, double* nq,
                      double* e) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  eos_Pne<EOS>(T[i], mu[i], d, P + i, nq + i, e + i);
}

template <int EOS, bool NCH>
__global__ void k_cons_to_prim(DevParams d, long long n, double tau, const double* cons, const double* warm,
                               double* prim, uint8_t* ok, uint8_t* reason) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double* c = cons + 11 * i;
  CellCons cc;
  cc.D = c[0]; cc.Sx = c[1]; cc.Sy = c[2]; cc.E = c[3]; cc.nux = c[4]; cc.nuy = c[5]; cc.Pi = c[6];
  cc.pixx = c[7]; cc.pixy = c[8]; cc.piyy = c[9]; cc.pieta = c[10];
  double y0 = nan_(), f0 = nan_(), x0 = nan_(), v0 = nan_();
  if (warm) { y0 = warm[4 * i]; f0 = warm[4 * i + 1]; x0 = warm[4 * i + 2]; v0 = warm[4 * i + 3]; }
  Recovery r = recover<EOS, NCH>(cc, d, y0, f0, x0, v0, d.p.primrec_maxit, d.p.primrec_tol);
  double* o = prim + 7 * i;
  o[0] = r.T; o[1] = r.mu; o[2] = r.ux; o[3] = r.uy; o[4] = r.n; o[5] = r.e; o[6] = r.P;
  ok[i] = r.ok;
  if (reason) reason[i] = r.reason;
}

/* ======================================================================
 * Two-phase recovery and the split stage (the context path).
 *
 * A warp runs as long as its slowest lane. Almost every cell converges from
 * its warm start in a few Newton iterations, but a few cells per pass need the
 * fresh seed (3 x 60 bisection steps) and a long Newton, and they set the time
 * of their whole warp. So the recovery runs in two kernels:
 *   k_prim_fast  every cell; vacuum cells and warm starts that converge within
 *                FAST_BUDGET iterations finish here; every other cell is
 *                appended to a queue.
 *   k_prim_slow  one warp per queued cell runs the whole cons_to_prim_2d!
 *                from the start (recover_warp, coop.cuh).
 * A cell's result does not depend on which kernel computed it: the fast kernel
 * accepts only a first attempt whose Newton loop converged, which is exactly
 * what the full algorithm returns for it, and the slow kernel recomputes
 * everything else from scratch.
 * The stage is split the same way: k_faces (one thread per face, no block
 * barrier) writes the HLLE fluxes to planes, k_update combines and sanitises
 * each cell and queues the rare cells whose admissibility needs an inversion,
 * which k_adm_slow settles.
 * ====================================================================== */

#define FAST_BUDGET 6

/* _primitive_pass! body after the recovery (src2d/rhs2d.jl:89-155) */
template <int EOS>
__device__ __forceinline__ void store_recovery(const DevParams& d, const DevPrims& w, const DevHist& h,
                                               long long i, const Recovery& r) {
  double T = r.T, mu = r.mu, ux = r.ux, uy = r.uy, n = r.n, en = r.e, P = r.P;
  if (!r.ok) {
    T = FV_T_MIN; mu = 0.0; ux = 0.0; uy = 0.0;
    eos_Pne<EOS>(T, mu, d, &P, &n, &en);
    en = jmax(en, 0.0); n = 0.0;
  }
  double Tm = jmax(T, FV_T_MIN);
  double yT = fx_log(Tm);
  double phi = jclamp((mu - d.p.m_hq) / Tm, -FV_PHI_CAP, FV_PHI_CAP);
  w.yT[i] = yT; w.phi[i] = phi; w.mu[i] = mu; w.alpha[i] = mu / Tm;
  w.ux[i] = ux; w.uy[i] = uy; w.P[i] = P; w.n[i] = n; w.e[i] = en; w.ok[i] = r.ok;
  if (r.ok) { h.x0_yT[i] = yT; h.x0_phi[i] = phi; h.x0_ux[i] = ux; h.x0_uy[i] = uy; }
  else { double q = nan_(); h.x0_yT[i] = q; h.x0_phi[i] = q; h.x0_ux[i] = q; h.x0_uy[i] = q; }
}

__device__ __forceinline__ void load_cons(const DevParams& d, const DevState& U, long long i, double tau,
                                          CellCons& c) {
  c.D = safe_div(U.f[d.iDtau][i], tau);
  c.Sx = U.f[d.iSx][i]; c.Sy = U.f[d.iSy][i]; c.E = U.f[d.iE][i];
  double dis[7];
  load_dis(d, U, i, dis);
  c.nux = dis[0]; c.nuy = dis[1]; c.Pi = dis[2]; c.pixx = dis[3]; c.pixy = dis[4]; c.piyy = dis[5];
  c.pieta = dis[6];
}

template <int EOS, bool NCH>
__device__ __forceinline__ void prim_fast_body(const DevParams& d, const DevState& U, const DevPrims& w,
                                               const DevHist& h, double tau, DevFlags* fl, unsigned int* queue,
                                               long long i) {
  bool vac = false, defer = false;
  unsigned nit = 0, natt = 0;
  if (i < d.Ntot) {
    CellCons c;
    load_cons(d, U, i, tau, c);
    const double yT0 = h.x0_yT[i], ux0 = h.x0_ux[i], uy0 = h.x0_uy[i];
    if (is_vacuum(c)) {
      store_recovery<EOS>(d, w, h, i, vacuum_recovery<EOS>(c, d));
      vac = true;
    } else if (!(isfinite_(yT0) && isfinite_(ux0) && isfinite_(uy0))) {
      defer = true;
    } else {
      bool over = false;
      int it = 0;
      Recovery r = recover_fast<EOS, NCH>(c, d, yT0, h.x0_phi[i], ux0, uy0, d.p.primrec_maxit,
                                          d.p.primrec_tol, FAST_BUDGET, &over, 0x7fffffff, 0.0, &it);
      nit = (unsigned)it; natt = 1;
      if (over || !r.ok) defer = true;
      else store_recovery<EOS>(d, w, h, i, r);
    }
  }
  /* warp-aggregated counters and queue appends (the grid holds whole warps) */
  const unsigned lane = threadIdx.x & 31;
  {
    const unsigned si = __reduce_add_sync(0xffffffffu, nit), sa = __reduce_add_sync(0xffffffffu, natt);
    if (lane == 0 && sa) { atomicAdd(&fl->it_fast, (unsigned long long)si); atomicAdd(&fl->n_fast, (unsigned long long)sa); }
  }
  unsigned mv = __ballot_sync(0xffffffffu, vac);
  if (lane == 0 && mv) atomicAdd((unsigned long long*)&fl->nvacuum, (unsigned long long)__popc(mv));
  unsigned md = __ballot_sync(0xffffffffu, defer);
  if (md) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&fl->qcount_p, (unsigned)__popc(md));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (defer) queue[base + __popc(md & ((1u << lane) - 1u))] = (unsigned)i;
  }
}

template <int EOS, bool NCH>
__global__ void __launch_bounds__(128, FV_FAST_MINB) k_prim_fast(DevParams d, DevState U, DevPrims w, DevHist h, double tau,
                                                   DevFlags* fl, unsigned int* queue) {
  prim_fast_body<EOS, NCH>(d, U, w, h, tau, fl, queue, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

/* The warm pass with the learned guess in front of it. Every cell of a block of
 * 128 (one tensor-core tile) gets the MLP's (log T, u^x, u^y); the charm
 * chemical potential follows in closed form from N^tau = n u^tau + nu^tau with
 * the LatticeHRG charm density n = A T e^phi e^x K2(x) (x = m/T); for another
 * EOS it is the warm start's. Newton from that guess must reach residual 1e-10
 * within GUESS_CHECK_IT updates and then converge as usual; a cell that does not
 * falls back to the plain warm-started attempt (the FAST_BUDGET pass), and a
 * cell that fails that too is deferred to k_prim_slow like any other. */
#define GUESS_CHECK_IT 3
#define GUESS_CHECK_TOL 1e-10
template <int EOS, bool NCH>
__device__ __forceinline__ void prim_learned_body(const DevParams& d, const DevState& U, const DevPrims& w,
                                                  const DevHist& h, double tau, DevFlags* fl, unsigned int* queue,
                                                  const guess::Net& net, guess::FwdSmem& s, long long i) {
  const bool live = i < d.Ntot;
  CellCons c;
  bool vac = false;
  float xn[guess::NIN];
#pragma unroll
  for (int q = 0; q < guess::NIN; ++q) xn[q] = 0.0f;
  if (live) {
    load_cons(d, U, i, tau, c);
    vac = is_vacuum(c);
    if (!vac && c.E > 0.0) {
      float r[guess::NIN];
      guess::features(c.E, c.Sx, c.Sy, c.Pi, c.pixx, c.pixy, c.piyy, r);
#pragma unroll
      for (int q = 0; q < guess::NIN; ++q) xn[q] = guess::nrm_in(net.norm, q, r[q]);
    }
  }
  float y[guess::NOUT] = {0.0f, 0.0f, 0.0f};
  const bool net_ok = guess::forward_tile(s, net, xn, y);
  bool defer = false;
  unsigned it_l = 0, n_l = 0, ok_l = 0, it_f = 0, n_f = 0;
  if (live) {
    const double yTw = h.x0_yT[i], phw = h.x0_phi[i], uxw = h.x0_ux[i], uyw = h.x0_uy[i];
    const bool warm = isfinite_(yTw) && isfinite_(uxw) && isfinite_(uyw);
    if (vac) {
      store_recovery<EOS>(d, w, h, i, vacuum_recovery<EOS>(c, d));
    } else {
      double g[4];
      bool have_guess = net_ok && c.E > 0.0;
      if (have_guess) {
        g[0] = ((double)y[0] * (double)net.norm.out_std[0] + (double)net.norm.out_mean[0]) + 0.25 * log(c.E);
        g[2] = (double)y[1] * (double)net.norm.out_std[1] + (double)net.norm.out_mean[1];
        g[3] = (double)y[2] * (double)net.norm.out_std[2] + (double)net.norm.out_mean[2];
        g[1] = isfinite_(phw) ? phw : 0.0;
        if (NCH && EOS == FIVO_EOS_LATTICE_HRG) {
          const double T0 = jclamp(exp(g[0]), FV_T_MIN, FV_T_SOLVE_MAX);
          const double K2 = lhrg_K2(lhrg_x(T0, d));
          double Cn = (d.A_lhrg * T0) * K2;
          if (d.p.hq_times_fmGeV3) Cn *= d.fmgev3;
          const double ut = utau(g[2], g[3]);
          const double nt = (c.D - nu_tau(g[2], g[3], ut, c.nux, c.nuy)) / ut;
          if (nt > 0.0 && Cn > 0.0) g[1] = log(nt / Cn);
        }
        have_guess = isfinite_(g[0]) && isfinite_(g[1]) && isfinite_(g[2]) && isfinite_(g[3]);
      }
      /* pass 0: the learned guess; pass 1: the warm start (one call site) */
      bool done = false;
      for (int pass = have_guess ? 0 : 1; pass < 2 && !done; ++pass) {
        if (pass == 1 && !warm) break;
        const double a0 = pass == 0 ? g[0] : yTw, a1 = pass == 0 ? g[1] : phw;
        const double a2 = pass == 0 ? g[2] : uxw, a3 = pass == 0 ? g[3] : uyw;
        bool over = false;
        int it = 0;
        Recovery r = recover_fast<EOS, NCH>(c, d, a0, a1, a2, a3, d.p.primrec_maxit, d.p.primrec_tol,
                                            pass == 0 ? d.p.primrec_maxit : FAST_BUDGET, &over,
                                            pass == 0 ? GUESS_CHECK_IT : 0x7fffffff, GUESS_CHECK_TOL, &it);
        if (pass == 0) { it_l += (unsigned)it; n_l = 1; } else { it_f += (unsigned)it; n_f = 1; }
        if (!over && r.ok) {
          store_recovery<EOS>(d, w, h, i, r);
          done = true;
          if (pass == 0) ok_l = 1;
        }
      }
      defer = !done;
    }
  }
  const unsigned lane = threadIdx.x & 31;
  {
    const unsigned a = __reduce_add_sync(0xffffffffu, it_l), b = __reduce_add_sync(0xffffffffu, n_l);
    const unsigned e = __reduce_add_sync(0xffffffffu, ok_l), f = __reduce_add_sync(0xffffffffu, it_f);
    const unsigned g2 = __reduce_add_sync(0xffffffffu, n_f);
    if (lane == 0 && (b || g2)) {
      atomicAdd(&fl->it_learn, (unsigned long long)a); atomicAdd(&fl->n_learn, (unsigned long long)b);
      atomicAdd(&fl->ok_learn, (unsigned long long)e); atomicAdd(&fl->it_fb, (unsigned long long)f);
      atomicAdd(&fl->n_fb, (unsigned long long)g2);
    }
  }
  unsigned mv = __ballot_sync(0xffffffffu, live && vac);
  if (lane == 0 && mv) atomicAdd((unsigned long long*)&fl->nvacuum, (unsigned long long)__popc(mv));
  unsigned md = __ballot_sync(0xffffffffu, defer);
  if (md) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&fl->qcount_p, (unsigned)__popc(md));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (defer) queue[base + __popc(md & ((1u << lane) - 1u))] = (unsigned)i;
  }
  if (!net_ok && threadIdx.x == 0) atomicExch(&fl->status, 3);
}

template <int EOS, bool NCH>
__global__ void __launch_bounds__(128, 4) k_prim_learned(DevParams d, DevState U, DevPrims w, DevHist h,
                                                       double tau, DevFlags* fl, unsigned int* queue,
                                                       guess::Net net) {
  __shared__ __align__(128) guess::FwdSmem s;
  prim_learned_body<EOS, NCH>(d, U, w, h, tau, fl, queue, net, s, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

/* (features, targets) pairs of the interior cells whose recovery succeeded, every
 * stride-th cell from phase on: out[k][11], k < cap, *count counts every offered
 * pair (it may pass cap) */
template <int EOS>
__global__ void k_guess_harvest(DevParams d, DevState U, DevPrims w, double tau, float* out, unsigned long long cap,
                                unsigned long long* count, int stride, int phase) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= d.Ntot || ((i + phase) % stride) != 0) return;
  const int ix = (int)(i / d.Nytot), iy = (int)(i % d.Nytot);
  if (!(ix >= d.ng && ix < d.ng + d.Nx && iy >= d.ng && iy < d.ng + d.Ny) || !w.ok[i]) return;
  CellCons c;
  load_cons(d, U, i, tau, c);
  if (is_vacuum(c) || !(c.E > 0.0)) return;
  float f[guess::NSAMP];
  guess::features(c.E, c.Sx, c.Sy, c.Pi, c.pixx, c.pixy, c.piyy, f);
  guess::targets(w.yT[i], w.ux[i], w.uy[i], c.E, f + guess::NIN);
  for (int q = 0; q < guess::NSAMP; ++q) if (!isfinite(f[q])) return;
  const unsigned long long k = atomicAdd(count, 1ULL);
  if (k < cap)
    for (int q = 0; q < guess::NSAMP; ++q) out[k * guess::NSAMP + q] = f[q];
}

/* The learned guess for the deferred cells only (FIVO_GUESS_DEFERRED): the fast pass
 * ran the warm starts as in the plain path; CTA b takes the 128 cells b*128 .. of its
 * queue (the cells without a warm start, and the warm attempts over budget or failed),
 * infers their starting points with the network on the tensor cores and runs the
 * Newton from there with the guess check (GUESS_CHECK_IT, GUESS_CHECK_TOL). A cell
 * that converges is stored; the rest go on to a second queue, which the full
 * recovery (k_prim_slow) then takes. The grid covers the largest possible queue and
 * the CTAs past its end return at once (all threads alike). One tile per CTA: the
 * forward pass gives up the CTA's tensor-memory allocation permit after its one
 * allocation, so a CTA cannot allocate for a second tile. */
/* a deferred cell from the network's output y: its starting point (log T, u from the
 * network, the charm chemical potential in closed form from N^tau), then the Newton
 * with the guess check; true when the cell converged and is stored */
template <int EOS, bool NCH>
__device__ __forceinline__ bool guess_and_recover(const DevParams& d, const DevPrims& w, const DevHist& h,
                                                  const CellCons& c, const float y[guess::NOUT],
                                                  const guess::Net& net, long long i, unsigned* it_l, unsigned* n_l,
                                                  unsigned* ok_l) {
  double g[4];
  g[0] = ((double)y[0] * (double)net.norm.out_std[0] + (double)net.norm.out_mean[0]) + 0.25 * log(c.E);
  g[2] = (double)y[1] * (double)net.norm.out_std[1] + (double)net.norm.out_mean[1];
  g[3] = (double)y[2] * (double)net.norm.out_std[2] + (double)net.norm.out_mean[2];
  const double phw = h.x0_phi[i];
  g[1] = isfinite_(phw) ? phw : 0.0;
  if (NCH && EOS == FIVO_EOS_LATTICE_HRG) {
    const double T0 = jclamp(exp(g[0]), FV_T_MIN, FV_T_SOLVE_MAX);
    const double K2 = lhrg_K2(lhrg_x(T0, d));
    double Cn = (d.A_lhrg * T0) * K2;
    if (d.p.hq_times_fmGeV3) Cn *= d.fmgev3;
    const double ut = utau(g[2], g[3]);
    const double nt = (c.D - nu_tau(g[2], g[3], ut, c.nux, c.nuy)) / ut;
    if (nt > 0.0 && Cn > 0.0) g[1] = log(nt / Cn);
  }
  if (!(isfinite_(g[0]) && isfinite_(g[1]) && isfinite_(g[2]) && isfinite_(g[3]))) return false;
  bool over = false;
  int it = 0;
  Recovery r = recover_fast<EOS, NCH>(c, d, g[0], g[1], g[2], g[3], d.p.primrec_maxit, d.p.primrec_tol,
                                      d.p.primrec_maxit, &over, GUESS_CHECK_IT, GUESS_CHECK_TOL, &it);
  *it_l = (unsigned)it; *n_l = 1;
  if (over || !r.ok) return false;
  store_recovery<EOS>(d, w, h, i, r);
  *ok_l = 1;
  return true;
}

template <int EOS, bool NCH>
__global__ void __launch_bounds__(128, 4) k_prim_learned_retry(DevParams d, DevState U, DevPrims w, DevHist h,
                                                             double tau, DevFlags* fl, const unsigned int* queue,
                                                             unsigned int* queue2, guess::Net net) {
  __shared__ __align__(128) guess::FwdSmem s;
  const unsigned n = *(volatile unsigned int*)&fl->qcount_p;
  const unsigned lane = threadIdx.x & 31;
  bool net_ok = true;
  {
    const unsigned base = blockIdx.x * 128u;
    if (base >= n) return;
    const unsigned qi = base + threadIdx.x;
    const bool live = qi < n;
    const long long i = live ? (long long)queue[qi] : 0;
    CellCons c;
    float xn[guess::NIN];
#pragma unroll
    for (int q = 0; q < guess::NIN; ++q) xn[q] = 0.0f;
    if (live) {
      load_cons(d, U, i, tau, c);
      if (c.E > 0.0) {
        float r[guess::NIN];
        guess::features(c.E, c.Sx, c.Sy, c.Pi, c.pixx, c.pixy, c.piyy, r);
#pragma unroll
        for (int q = 0; q < guess::NIN; ++q) xn[q] = guess::nrm_in(net.norm, q, r[q]);
      }
    }
    float y[guess::NOUT] = {0.0f, 0.0f, 0.0f};
    const bool tile_ok = guess::forward_tile(s, net, xn, y);
    net_ok = net_ok && tile_ok;
    bool pass_on = live, done = false;
    unsigned it_l = 0, n_l = 0, ok_l = 0;
    if (live && tile_ok && c.E > 0.0) done = guess_and_recover<EOS, NCH>(d, w, h, c, y, net, i, &it_l, &n_l, &ok_l);
    pass_on = live && !done;
    {
      const unsigned a = __reduce_add_sync(0xffffffffu, it_l), b = __reduce_add_sync(0xffffffffu, n_l);
      const unsigned e = __reduce_add_sync(0xffffffffu, ok_l);
      if (lane == 0 && b) {
        atomicAdd(&fl->it_learn, (unsigned long long)a); atomicAdd(&fl->n_learn, (unsigned long long)b);
        atomicAdd(&fl->ok_learn, (unsigned long long)e);
      }
    }
    const unsigned md = __ballot_sync(0xffffffffu, pass_on);
    if (md) {
      unsigned b2 = 0;
      if (lane == 0) b2 = atomicAdd(&fl->qcount_q, (unsigned)__popc(md));
      b2 = __shfl_sync(0xffffffffu, b2, 0);
      if (pass_on) queue2[b2 + __popc(md & ((1u << lane) - 1u))] = (unsigned)i;
    }
  }
  if (!net_ok && threadIdx.x == 0) atomicExch(&fl->status, 3);
}

/* Barrier of the two warps of pair p of a block (named barrier 1 + p, 64 threads). */
__device__ __forceinline__ void pair_sync(int p) {
  asm volatile("bar.sync %0, 64;" :: "r"(1 + p) : "memory");
}

/* The deferred cells. Each cell is taken by a pair of warps: the first runs the
 * warm-started attempt, the second at the same time the cold (seeded) attempt
 * that cons_to_prim_2d! runs when the warm one fails; the second stops early
 * when the first succeeds. The pair takes cells from the queue one at a time so
 * that long and short recoveries balance over the pairs. */
/* one queued cell i, taken by the warp pair `pair` of the block (both warps call it) */
template <int EOS, bool NCH>
__device__ __forceinline__ void slow_item(const DevParams& d, const DevState& U, const DevPrims& w, const DevHist& h,
                                          double tau, DevFlags* fl, long long i, int lane, bool lead, int pair,
                                          int* s_stop, Recovery* s_cold) {
    CellCons c;
    load_cons(d, U, i, tau, c);
    const double yT0 = h.x0_yT[i], phi0 = h.x0_phi[i], ux0 = h.x0_ux[i], uy0 = h.x0_uy[i];
    const bool warm = isfinite_(yT0) && isfinite_(ux0) && isfinite_(uy0);
    Recovery r;
    r.ok = 0; r.reason = PRR_UNSET;
    if (!lead || warm) {   /* one call site: the lead's warm attempt or the partner's cold one */
      r = attempt_warp<EOS, NCH>(c, d, lead ? yT0 : nan_(), lead ? phi0 : nan_(), lead ? ux0 : nan_(),
                                 lead ? uy0 : nan_(), d.p.primrec_maxit, d.p.primrec_tol, lane,
                                 lead ? nullptr : &s_stop[pair]);
      if (lead && lane == 0 && (r.ok || r.reason == PRR_VACUUM)) *(volatile int*)&s_stop[pair] = 1;
      if (!lead && lane == 0) s_cold[pair] = r;
    }
    pair_sync(pair);
    if (lead && lane == 0) {
      /* cons_to_prim_2d!: the warm result if it succeeded (or found vacuum), else the cold one */
      if (!(warm && (r.ok || r.reason == PRR_VACUUM))) r = s_cold[pair];
      if (!r.ok) {
        if (r.reason == PRR_VACUUM) atomicAdd((unsigned long long*)&fl->nvacuum, 1ULL);
        else {
          atomicAdd((unsigned long long*)&fl->nprimfail, 1ULL);
          atomicMin(&fl->rep, ((unsigned long long)i << 8) | r.reason);
        }
      }
      store_recovery<EOS>(d, w, h, i, r);
    }
}

template <int EOS, bool NCH>
__global__ void __launch_bounds__(128) k_prim_slow(DevParams d, DevState U, DevPrims w, DevHist h, double tau,
                                                   DevFlags* fl, const unsigned int* queue, const unsigned int* qcount,
                                                   unsigned int* qnext) {
  __shared__ unsigned int s_q[2];
  __shared__ int s_stop[2];
  __shared__ Recovery s_cold[2];
  const unsigned n = *(volatile const unsigned int*)qcount;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&fl->tot_p, (unsigned long long)n);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pair = warp >> 1;
  const bool lead = (warp & 1) == 0;
  while (true) {
    if (lead && lane == 0) {
      s_q[pair] = atomicAdd(qnext, 1u);
      s_stop[pair] = 0;
    }
    pair_sync(pair);
    const unsigned q = *(volatile unsigned int*)&s_q[pair];
    if (q >= n) break;
    slow_item<EOS, NCH>(d, U, w, h, tau, fl, (long long)queue[q], lane, lead, pair, s_stop, s_cold);
  }
}

/* One face, computed by a pair of lanes: lane side 0 owns the left state (cell
 * i), side 1 the right state (cell i + st). Each lane reconstructs, maps to
 * conserved variables (EOS with c_s^2), applies the fallbacks and evaluates the
 * physical flux and wave speeds of its own state; the pair then exchanges them
 * by shuffle and both lanes form the HLLE flux. The operations on each state are
 * those of face_flux (the same expressions, the same order), so the fluxes have
 * its bits; a lane does half the EOS work, which halves the dependent chain of a
 * face and the registers it needs. All lanes of the warp must call it.
 * Returns max(|sL|, |sR|); stores each row of the HLLE flux into its plane of
 * Fh (the lane of side a % 2 stores plane a) unless Fh is null. */
/* Where a face reads its stencil: the cells i - st, i, i + st, i + 2 st around the
 * face between i and i + st, named by their position p = -1, 0, 1, 2. The
 * primitives q = 0..3 are (yT, phi, u^x, u^y). FaceSrcGlobal reads the planes in
 * global memory; k_faces_tile's source reads a tile staged in shared memory. */
struct FaceSrcGlobal {
  const DevParams& d;
  const DevState& U;
  const DevPrims& w;
  long long i, st;
  __device__ __forceinline__ double prim(int q, int p) const {
    const double* f = q == 0 ? w.yT : (q == 1 ? w.phi : (q == 2 ? w.ux : w.uy));
    return f[i + p * st];
  }
  __device__ __forceinline__ double mu(int p) const { return w.mu[i + p * st]; }
  __device__ __forceinline__ void dis(int p, double out[7]) const { load_dis(d, U, i + p * st, out); }
};

template <int EOS, bool XDIR, class Src>
__device__ __forceinline__ double face_flux_pair(const DevParams& d, const Src& src, long long i, long long st,
                                                 int k, int kmax, double tau, const uint8_t* ffo, int side,
                                                 double* Fh) {
  const long long ip = i + st;
  const int p0 = side;             /* this lane's own cell: i (left) or i + st (right) */
  /* the two lanes of this pair; every branch below is taken by both or neither */
  const unsigned pm = 3u << (threadIdx.x & 30);
  const int ng = d.ng;
  double dis[7];
  src.dis(p0, dis);
  const bool forced = ffo != nullptr && (ffo[i] || ffo[ip]);
  Prim p;
  double uc[4];
  bool good = false, floored = false;
  if (!forced) {
    double v[4];
    const bool first = (k + 1 <= ng) || (k + 1 >= kmax - ng);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      /* left: (vm, vi, vp) around vi; right: (vi, vp, vpp) around vp */
      const double c = src.prim(q, p0);
      if (first) { v[q] = c; continue; }
      const double a = src.prim(q, side ? 0 : -1);
      const double b = src.prim(q, side ? 2 : 1);
      const double sl = mc_limiter(c - a, b - c);
      const double h = 0.5 * sl;
      const double val = side ? c - h : c + h;
      v[q] = jclamp(val, jmin(jmin(a, c), b), jmax(jmax(a, c), b));
    }
    const double T = fx_exp(v[0]);
    const double mu = d.p.m_hq + (T * v[1]);
    const bool ok = prim_to_cons<EOS>(uc, p, T, mu, v[2], v[3], dis, tau, d);
    const bool mine = ok && uc[0] >= 0.0 && uc[3] >= FV_E_FLOOR;
    const int theirs = __shfl_xor_sync(pm, (int)mine, 1);
    good = mine && theirs;
  }
  if (!good) {
    const double Tc = fx_exp(src.prim(0, p0)), muc = src.mu(p0);
    const bool ok = prim_to_cons<EOS>(uc, p, Tc, muc, src.prim(2, p0), src.prim(3, p0), dis, tau, d);
    const int theirs = __shfl_xor_sync(pm, (int)ok, 1);
    const bool both = ok && theirs;
    if (!both && !ok) {
      /* _floor_prim_2d!, src2d/rhs2d.jl:259-268 */
      floored = true;
      uc[0] = 0.0; uc[1] = 0.0; uc[2] = 0.0; uc[3] = FV_E_FLOOR;
      p.T = FV_T_MIN; p.mu = 0.0; p.ux = 0.0; p.uy = 0.0; p.n = 0.0; p.e = FV_E_FLOOR; p.P = 0.0;
      p.nux = p.nuy = p.Pi = p.pixx = p.pixy = p.piyy = p.pieta = 0.0;
    }
  }
  if (floored) p.cs2 = eos_cs2<EOS>(FV_T_MIN, d);
  double F4[4], v;
  flux_cons4<XDIR>(F4, p, tau, &v);
  double lm, lp;
  wavespeeds<XDIR>(p, XDIR ? p.pixx : p.piyy, &lm, &lp);
  const double lmo = __shfl_xor_sync(pm, lm, 1), lpo = __shfl_xor_sync(pm, lp, 1);
  const double lmL = side ? lmo : lm, lmR = side ? lm : lmo;
  const double lpL = side ? lpo : lp, lpR = side ? lp : lpo;
  const double sL = jmin(lmL, lmR), sR = jmax(lpL, lpR);
  const bool an = d.hasNu && d.p.advect_nu, aP = d.hasPi && d.p.advect_Pi, ap = d.hasShear && d.p.advect_pi;
  const double inv = 1.0 / ((sR - sL) + FV_TINY);
#pragma unroll
  for (int s = 0; s < 11; ++s) {
    /* row s of this state: the conserved column (its stored dissipatives, zero
     * when floored) and the flux of flux_cell_2d!, whose advected rows are that
     * same dissipative times v */
    double cs, Fs;
    if (s < 4) { cs = uc[s]; Fs = F4[s]; }
    else {
      cs = floored ? 0.0 : dis[s - 4];
      const bool adv = s < 6 ? an : (s == 6 ? aP : ap);
      Fs = adv ? cs * v : 0.0;
    }
    const double Fo = __shfl_xor_sync(pm, Fs, 1);
    const double co = __shfl_xor_sync(pm, cs, 1);
    const double FLs = side ? Fo : Fs, FRs = side ? Fs : Fo;
    const double cls = side ? co : cs, crs = side ? cs : co;
    double h;
    if (sL >= 0) h = FLs;
    else if (sR <= 0) h = FRs;
    else h = (((sR * FLs) - (sL * FRs)) + ((sR * sL) * (crs - cls))) * inv;
    const int a = plane_of(d, s);
    if (Fh && a >= 0 && (a & 1) == side) Fh[(size_t)a * d.Ntot + i] = h;
  }
  return jmax(fabs_(sL), fabs_(sR));
}

/* two lanes per face of one direction, every face of the (ghost-inclusive) grid;
 * the lane of the left state stores the even rows, its partner the odd ones */
template <int EOS, bool XDIR>
__device__ __forceinline__ void faces_body(const DevParams& d, const DevState& Ub, const DevPrims& w, double tau,
                                           const uint8_t* ffo, double* Fh, DevFlags* fl, long long t) {
  const long long nf = XDIR ? (long long)(d.Nxtot - 1) * d.Nytot : (long long)d.Nxtot * (d.Nytot - 1);
  const int side = (int)(t & 1);
  long long f = t >> 1;
  const bool valid = f < nf;
  if (!valid) f = nf - 1;          /* a spare pair repeats the last face and stores nothing */
  long long i;
  int k, kmax;
  if (XDIR) { i = f; k = (int)(f / d.Nytot); kmax = d.Nxtot; }
  else {
    int ix = (int)(f / (d.Nytot - 1)), iy = (int)(f % (d.Nytot - 1));
    i = (long long)ix * d.Nytot + iy; k = iy; kmax = d.Nytot;
  }
  const long long st = XDIR ? d.Nytot : 1;
  const FaceSrcGlobal src{d, Ub, w, i, st};
  double amax = face_flux_pair<EOS, XDIR>(d, src, i, st, k, kmax, tau, ffo, side, valid ? Fh : nullptr);
  for (int o = 16; o > 0; o >>= 1) amax = jmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  __shared__ double red[4];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = jmax(jmax(red[0], red[1]), jmax(red[2], red[3]));
    atomic_max_pos(&fl->amax_bits, m);
  }
}

template <int EOS, bool XDIR>
__global__ void __launch_bounds__(128, FV_FACE_MINB) k_faces(DevParams d, DevState Ub, DevPrims w, double tau,
                                               const uint8_t* ffo, double* Fh, DevFlags* fl) {
  faces_body<EOS, XDIR>(d, Ub, w, tau, ffo, Fh, fl, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

/* cell_admissible_2d up to (not including) the inversion: 0 inadmissible,
 * 1 admissible, 2 settle by inverting (src2d/floors2d.jl:281-337) */
__device__ __forceinline__ int adm_prefilter(const DevParams& d, const double u[FV_MAXV], bool okw, double ux,
                                             double uy, double Pw) {
  const double Emin = FV_E_FLOOR;
  double E = u[d.iE], Sx = u[d.iSx], Sy = u[d.iSy], Dt = u[d.iDtau];
  if (!(isfinite_(E) && isfinite_(Sx) && isfinite_(Sy) && isfinite_(Dt))) return 0;
  if (!(E >= Emin)) return 0;
  if (!(Dt >= 0.0)) return 0;
  for (int a = 4; a < d.nvf; ++a) if (!isfinite_(u[a])) return 0;
  if (E <= 1e6 * Emin) return 1;
  if (okw) {
    double ut = utau(ux, uy);
    double iu = safe_inv(ut);
    double vx = ux * iu, vy = uy * iu;
    if (!(isfinite_(vx) && isfinite_(vy))) return 0;
    double lim = (1.0 - 1e-12) * (1.0 - 1e-12);
    if (!((vx * vx) + (vy * vy) < lim)) return 0;
  }
  double Peff = peff_of(d, u, Pw);
  if (fx_hypot(Sx, Sy) <= ((FV_SR_MARGIN * FV_CHI_SRE) * (E + Peff))) return 1;
  return 2;
}

/* per interior cell: flux divergence + source (rhs_2d! assembly), the stage
 * combination, sanitize_stage_2d!'s floors and bounds, and the admissibility
 * test up to the inversion */
/* FT: the type of the face-flux planes (double; float for the mixed-precision face pass).
 * FULL: the layout carries charge, bulk and shear (the viscous event's), so every row
 * index is a compile-time constant and the per-cell row arrays live in registers; the
 * arithmetic is the same. */
template <int EOS, bool NCH, typename FT = double, bool FULL = false>
__device__ __forceinline__ void update_body(const DevParams& d0, const StageArgs& s, const FT* Fhx, const FT* Fhy,
                                            unsigned int* aqueue, long long t) {
  DevParams d = d0;
  if (FULL) {
    d.iDtau = 0; d.iSx = 1; d.iSy = 2; d.iE = 3; d.iNux = 4; d.iNuy = 5; d.iPi = 6;
    d.iPixx = 7; d.iPixy = 8; d.iPiyy = 9; d.iPieta = 10; d.nvf = 11;
    d.hasNu = 1; d.hasPi = 1; d.hasShear = 1;
  }
  int verdict = 1;
  long long i = 0;
  if (t < (long long)d.Nx * d.Ny) {
    const int ix = d.ng + (int)(t / d.Ny), iy = d.ng + (int)(t % d.Ny);
    i = (long long)ix * d.Nytot + iy;
    const int nv = d.nvf;
    const size_t N = (size_t)d.Ntot;
    const double invdx = 1.0 / d.dx, invdy = 1.0 / d.dy;
    double ub[FV_MAXV];
    for (int a = 0; a < nv; ++a) ub[a] = s.Ub.f[a][i];
    const double Pw = s.w.P[i];
    /* source_cell_2d!, src2d/fluxes2d.jl:166-177 (+ the advected-scalar divv terms) */
    double Sr[FV_MAXV];
    for (int a = 0; a < nv; ++a) Sr[a] = 0.0;
    {
      double itau = safe_inv(s.tau);
      double Pi = d.hasPi ? ub[d.iPi] : 0.0, pieta = d.hasShear ? ub[d.iPieta] : 0.0;
      Sr[d.iSx] = (-ub[d.iSx]) * itau;
      Sr[d.iSy] = (-ub[d.iSy]) * itau;
      Sr[d.iE] = (-((ub[d.iE] + (Pw + Pi)) + pieta)) * itau;
      bool an = d.hasNu && d.p.advect_nu, aP = d.hasPi && d.p.advect_Pi, ap = d.hasShear && d.p.advect_pi;
      if (an || aP || ap) {
        /* compute_divv_2d!, src2d/rhs2d.jl:29-41 */
        const long long ixm = i - d.Nytot, ixp = i + d.Nytot;
        double vxp = s.w.ux[ixp] * safe_inv(utau(s.w.ux[ixp], s.w.uy[ixp]));
        double vxm = s.w.ux[ixm] * safe_inv(utau(s.w.ux[ixm], s.w.uy[ixm]));
        double vyp = s.w.uy[i + 1] * safe_inv(utau(s.w.ux[i + 1], s.w.uy[i + 1]));
        double vym = s.w.uy[i - 1] * safe_inv(utau(s.w.ux[i - 1], s.w.uy[i - 1]));
        double divv = ((0.5 * (vxp - vxm)) * invdx) + ((0.5 * (vyp - vym)) * invdy);
        if (an) { Sr[d.iNux] += ub[d.iNux] * divv; Sr[d.iNuy] += ub[d.iNuy] * divv; }
        if (aP) Sr[d.iPi] += ub[d.iPi] * divv;
        if (ap) {
          Sr[d.iPixx] += ub[d.iPixx] * divv; Sr[d.iPixy] += ub[d.iPixy] * divv;
          Sr[d.iPiyy] += ub[d.iPiyy] * divv; Sr[d.iPieta] += ub[d.iPieta] * divv;
        }
      }
    }
    double u[FV_MAXV];
    for (int a = 0; a < nv; ++a) {
      const FT* fx = Fhx + (size_t)a * N;
      const FT* fy = Fhy + (size_t)a * N;
      double k = (((-((double)fx[i] - (double)fx[i - d.Nytot])) * invdx) -
                  (((double)fy[i] - (double)fy[i - 1]) * invdy)) + Sr[a];
      if (s.dU) s.dU[(size_t)a * N + i] = k;
      if (s.mode == COMB_EULER) u[a] = ub[a] + (s.dt * k);
      else if (s.mode == COMB_BLEND) u[a] = (s.wold * s.Uold.f[a][i]) + (s.wnew * (ub[a] + (s.dt * k)));
      else if (s.mode == COMB_THIRD) u[a] = (s.Uold.f[a][i] + (2.0 * (ub[a] + (s.dt * k)))) / 3.0;
    }
    if (d.hasM2) stage_m2_rows(d, s, i);
    if (s.mode != COMB_RHS_ONLY) {
      sanitize_cell(d, u, ix, iy, s.tau_state, Pw, true, FV_E_FLOOR);
      verdict = adm_prefilter(d, u, s.w.ok[i] != 0, s.w.ux[i], s.w.uy[i], Pw);
      s.bad[i] = verdict == 0 ? 1 : 0;
      for (int a = 0; a < nv; ++a) s.Uout.f[a][i] = u[a];
    }
  }
  const unsigned lane = threadIdx.x & 31;
  unsigned mb = __ballot_sync(0xffffffffu, verdict == 0);
  if (lane == 0 && mb) atomicAdd((unsigned long long*)&s.fl->nbad, (unsigned long long)__popc(mb));
  unsigned mq = __ballot_sync(0xffffffffu, verdict == 2);
  if (mq) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(&s.fl->qcount_a, (unsigned)__popc(mq));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (verdict == 2) aqueue[base + __popc(mq & ((1u << lane) - 1u))] = (unsigned)i;
  }
}

template <int EOS, bool NCH, typename FT = double, bool FULL = false>
__global__ void __launch_bounds__(128) k_update(DevParams d0, StageArgs s, const FT* Fhx, const FT* Fhy,
                                                unsigned int* aqueue) {
  update_body<EOS, NCH, FT, FULL>(d0, s, Fhx, Fhy, aqueue, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

/* the inversion of cell_admissible_2d for one queued cell i (src2d/floors2d.jl:329-335), by one warp */
template <int EOS, bool NCH>
__device__ __forceinline__ void adm_item(const DevParams& d, const DevState& Uout, double tau_state, uint8_t* bad,
                                         DevFlags* fl, long long i, int lane) {
  CellCons c;
  load_cons(d, Uout, i, tau_state, c);
  Recovery r = recover_warp<EOS, NCH>(c, d, nan_(), nan_(), nan_(), nan_(), 80, 1e-12, lane);
  if (lane == 0) {
    bool adm = r.ok || r.reason == PRR_VACUUM;
    bad[i] = adm ? 0 : 1;
    if (!adm) atomicAdd((unsigned long long*)&fl->nbad, 1ULL);
  }
}

/* the inversion of cell_admissible_2d for the queued cells (src2d/floors2d.jl:329-335),
 * one warp per cell */
template <int EOS, bool NCH>
__global__ void __launch_bounds__(128) k_adm_slow(DevParams d, DevState Uout, double tau_state, uint8_t* bad,
                                                  DevFlags* fl, const unsigned int* aqueue) {
  const unsigned n = *(volatile unsigned int*)&fl->qcount_a;
  if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&fl->tot_a, (unsigned long long)n);
  const int lane = threadIdx.x & 31;
  while (true) {
    unsigned q = 0;
    if (lane == 0) q = atomicAdd(&fl->qnext_a, 1u);
    q = __shfl_sync(FV_FULL, q, 0);
    if (q >= n) break;
    adm_item<EOS, NCH>(d, Uout, tau_state, bad, fl, (long long)aqueue[q], lane);
  }
}

}  // namespace fv
#endif
