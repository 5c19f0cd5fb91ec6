/*
 * freezeout.cuh — the 2-D freeze-out surface and its Cooper-Frye pion yield
 * (freezeout2d.jl), the step after the hydrodynamic stage.
 *
 * The surface is boost invariant and parameterised as tau = tau_fo(x, y): for
 * each interior cell the last time T crosses T_fo downwards, the crossing
 * interpolated linearly between two records, with the flow at that record
 * (record!, freezeout2d.jl:94-115). The yield integrates
 *     dN/dy = f_yield / (2 pi hbar c)^3  sum dSigma_mu p^mu f(Estar / T_fo)
 * with dSigma_mu p^mu = tau_fo (m_T cosh eta - d_x tau_fo p_x - d_y tau_fo p_y) and
 * Estar = u^tau m_T cosh eta - u^x p_x - u^y p_y, over a (p_T, phi, eta) grid, Boltzmann
 * and Bose both (pion_yield, freezeout2d.jl:144-190).
 */
#pragma once

namespace fo {

/* the surface over the Nx x Ny interior cells, cell (a, b) at a * ny + b */
struct Surf {
  double *tau_fo, *uxf, *uyf, *Tprev;
  uint8_t* above;                 /* wasabove */
  unsigned long long* refroze;    /* cells that re-heated above T_fo after freezing */
  int nx, ny;
};

/* record!(tau), freezeout2d.jl:94-115: one interior cell per thread */
__global__ void k_record(fv::DevParams d, fv::DevPrims w, double tau, double tau_prev, double T_fo, Surf s) {
  const long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (long long)s.nx * s.ny) return;
  const int a = (int)(k / s.ny), b = (int)(k % s.ny);
  const long long i = (long long)(d.ng + a) * d.Nytot + (d.ng + b);
  const double T = fx::fx_exp(w.yT[i]);
  if (T > T_fo) {
    if (!isnan(s.tau_fo[k])) atomicAdd(s.refroze, 1ULL);
    s.above[k] = 1;
    s.tau_fo[k] = fx::nan_();                        /* still hot */
  } else if (s.above[k] && isnan(s.tau_fo[k])) {
    const double Tp = s.Tprev[k];
    s.tau_fo[k] = (isnan(Tp) || Tp <= T_fo) ? tau : tau_prev + ((tau - tau_prev) * (Tp - T_fo)) / (Tp - T);
    s.uxf[k] = w.ux[i];
    s.uyf[k] = w.uy[i];
  }
  s.Tprev[k] = T;
}

/* grad1, freezeout2d.jl:132-141: central where both neighbours froze, one-sided
 * where one did, NaN where neither did */
__device__ __forceinline__ double grad1(const double* A, int ny, int a, int b, int dir, double dx) {
  const double lo = dir == 1 ? A[(a - 1) * ny + b] : A[a * ny + b - 1];
  const double hi = dir == 1 ? A[(a + 1) * ny + b] : A[a * ny + b + 1];
  const double c = A[a * ny + b];
  if (!isnan(lo) && !isnan(hi)) return (hi - lo) / (2.0 * dx);
  if (!isnan(hi)) return (hi - c) / dx;
  if (!isnan(lo)) return (c - lo) / dx;
  return fx::nan_();
}

struct CF {
  double T_fo, m, pt_lo, pt_hi, eta_max;
  int n_eta, n_pt, n_phi;
};

/* One thread per (surface cell, p_T, phi), the eta sum in the thread; per block
 * the sums of w f_Boltzmann, w f_Bose and the negative and positive parts of the
 * Boltzmann integrand, reduced in a fixed tree into part[block][4]. */
__global__ void __launch_bounds__(256) k_cooper_frye(Surf s, double dx, CF p, double* part) {
  __shared__ double red[4][256];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)s.nx * s.ny * p.n_pt * p.n_phi;
  double acc = 0.0, accB = 0.0, neg = 0.0, pos = 0.0;
  if (t < total) {
    const int iphi = (int)(t % p.n_phi);
    const long long r = t / p.n_phi;
    const int ipt = (int)(r % p.n_pt);
    const long long k = r / p.n_pt;
    const int a = (int)(k / s.ny), b = (int)(k % s.ny);
    if (a >= 1 && a <= s.nx - 2 && b >= 1 && b <= s.ny - 2 && !isnan(s.tau_fo[k])) {
      const double gx = grad1(s.tau_fo, s.ny, a, b, 1, dx), gy = grad1(s.tau_fo, s.ny, a, b, 2, dx);
      if (!isnan(gx) && !isnan(gy)) {
        const double tau = s.tau_fo[k], ux = s.uxf[k], uy = s.uyf[k];
        const double ut = sqrt((1.0 + (ux * ux)) + (uy * uy));
        const double dpt = (p.pt_hi - p.pt_lo) / (double)(p.n_pt - 1);
        const double pt = p.pt_lo + (double)ipt * dpt;
        const double dphi = (2.0 * M_PI) / (double)p.n_phi;
        const double phi = (double)iphi * dphi;
        const double deta = (2.0 * p.eta_max) / (double)(p.n_eta - 1);
        const double mT = sqrt((pt * pt) + (p.m * p.m));
        const double px = pt * cos(phi), py = pt * sin(phi);
        for (int ie = 0; ie < p.n_eta; ++ie) {
          const double eta = -p.eta_max + (double)ie * deta;
          const double ch = cosh(eta);
          const double dSp = tau * (((mT * ch) - (gx * px)) - (gy * py));
          const double Es = (((ut * mT) * ch) - (ux * px)) - (uy * py);
          const double x = Es / p.T_fo;
          const double fB = exp(-x);
          const double fb = x > 1e-8 ? 1.0 / (exp(x) - 1.0) : 0.0;
          const double w = (((((dSp * pt) * dpt) * dphi) * deta) * dx) * dx;
          acc += w * fB;
          accB += w * fb;
          if (dSp < 0.0) neg += -(w * fB); else pos += w * fB;
        }
      }
    }
  }
  red[0][threadIdx.x] = acc; red[1][threadIdx.x] = accB; red[2][threadIdx.x] = neg; red[3][threadIdx.x] = pos;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o)
      for (int q = 0; q < 4; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 4; ++q) part[(size_t)blockIdx.x * 4 + q] = red[q][0];
}

}  // namespace fo
