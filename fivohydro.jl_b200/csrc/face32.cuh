/*
 * face32.cuh — the mixed-precision face pass: reconstruction, the map to
 * conserved variables with the EOS, the physical fluxes, the wave speeds and the
 * HLLE combination of rhs_2d!'s face loop (src2d/rhs2d.jl:286-371,
 * src2d/reconstruction2d.jl:27-103, src2d/fluxes2d.jl:24-113) in FP32, with the
 * face fluxes stored as FP32 planes. The primitive recovery, the flux
 * divergence, the sources, the SSPRK combination and the floors stay FP64
 * (k_update reads the FP32 planes into FP64 sums).
 *
 * The operations and fallbacks are those of face_flux_pair (kernels.cuh) in the
 * same order; only the arithmetic type differs. e^x K2(x) of the charm density is
 * the same Chebyshev series (piece B, 2 <= x < 1e4) summed in FP32 from the FP64
 * coefficients rounded once; outside that range the FP64 function is used.
 */
#pragma once

namespace f32 {

__constant__ float K0B_F[FX_CHEB_NB] = FX_CHEB_K0B;
__constant__ float K1B_F[FX_CHEB_NB] = FX_CHEB_K1B;

constexpr float TINY_F = 1e-30f;

/* Julia's min / max / clamp (a NaN operand propagates) in FP32 */
__device__ __forceinline__ float jminf(float a, float b) { return (a != a || b != b) ? a + b : (a < b ? a : b); }
__device__ __forceinline__ float jmaxf(float a, float b) { return (a != a || b != b) ? a + b : (a > b ? a : b); }
__device__ __forceinline__ float jclampf(float x, float lo, float hi) { return x > hi ? hi : (x < lo ? lo : x); }
__device__ __forceinline__ float jsignf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : x); }
__device__ __forceinline__ float utauf(float ux, float uy) { return sqrtf((1.0f + ux * ux) + uy * uy); }
__device__ __forceinline__ float safe_invf(float x) { return fabsf(x) > TINY_F ? 1.0f / x : 0.0f; }

__device__ __forceinline__ float mc_limiter_f(float a, float b) {
  if (jsignf(a) != jsignf(b)) return 0.0f;
  const float s = jsignf(a), aa = fabsf(a), bb = fabsf(b);
  return s * jminf(2.0f * aa, jminf(2.0f * bb, 0.5f * (aa + bb)));
}

/* light_P, light_dP_dT, light_d2P_dT2 (src/eos.jl:357-463) in FP32, from one exp */
__device__ __forceinline__ void light_eos_f(float T, const fv::DevParams& d, float* P, float* dP, float* d2P) {
  const fivo_params& e = d.p;
  const float A = (float)d.lA, B = (float)d.lB;
  const float a0 = (float)e.lhrg_a[0], a1 = (float)e.lhrg_a[1], a2 = (float)e.lhrg_a[2], a3 = (float)e.lhrg_a[3];
  const float b0 = (float)e.lhrg_b[0], b1 = (float)e.lhrg_b[1], b2 = (float)e.lhrg_b[2], b3 = (float)e.lhrg_b[3];
  const float k0 = (float)LK0, k1 = (float)LK1, k2 = (float)LK2, k3 = (float)LK3, k4 = (float)LK4;
  const float T2 = T * T, T3 = T2 * T, T4 = T2 * T2;
  const float E = jclampf((-(A / T2)) - (B / T), -700.0f, 700.0f);
  const float expE = expf(E);
  const float N = (((k0 * a3) + ((k1 * a2) * T)) + ((k2 * a1) * T2)) + ((k3 * a0) * T3) + (k4 * T4);
  const float D = (((k0 * b3) + ((k1 * b2) * T)) + ((k2 * b1) * T2)) + ((k3 * b0) * T3) + T4;
  const float C = (float)d.fmgev3 * expE;
  *P = (C * T4) * (N / D);
  const float Ep = ((2.0f * A) / T3) + (B / T2);
  const float Np = ((k1 * a2) + (((2.0f * k2) * a1) * T)) + (((3.0f * k3) * a0) * T2) + ((4.0f * k4) * T3);
  const float Dp = ((k1 * b2) + (((2.0f * k2) * b1) * T)) + (((3.0f * k3) * b0) * T2) + (4.0f * T3);
  const float G = T4 * N, H = D;
  const float Gp = ((4.0f * T3) * N) + (T4 * Np);
  const float F = G / H;
  const float Fp = ((Gp * H) - (G * Dp)) / (H * H);
  *dP = C * (Fp + (F * Ep));
  const float Epp = ((-6.0f * A) / T4) - ((2.0f * B) / T3);
  const float Npp = (((2.0f * k2) * a1) + (((6.0f * k3) * a0) * T)) + ((12.0f * k4) * T2);
  const float Dpp = (((2.0f * k2) * b1) + (((6.0f * k3) * b0) * T)) + (12.0f * T2);
  const float Gpp = (((12.0f * T2) * N) + ((8.0f * T3) * Np)) + (T4 * Npp);
  const float Q = (Gp * H) - (G * Dp);
  const float Qp = (Gpp * H) - (G * Dpp);
  const float Fpp = ((Qp * H) - ((2.0f * Q) * Dp)) / ((H * H) * H);
  *d2P = C * ((Fpp + ((2.0f * Fp) * Ep)) + (F * (Epp + (Ep * Ep))));
}

/* e^x K2(x) (the LatticeHRG charm density's, 0 off the domain) */
__device__ __forceinline__ float k2x_f(float x) {
  if (x >= 2.0f && x < 1.0e4f) {
    const float u = (4.0f / x) - 1.0f, tu = 2.0f * u;
    float p1 = 0.0f, p2 = 0.0f, q1 = 0.0f, q2 = 0.0f;
#pragma unroll
    for (int k = FX_CHEB_NB - 1; k >= 1; --k) {
      const float p = fmaf(tu, p1, K0B_F[k] - p2);
      const float q = fmaf(tu, q1, K1B_F[k] - q2);
      p2 = p1; p1 = p; q2 = q1; q1 = q;
    }
    const float rs = rsqrtf(x);
    const float k0 = fmaf(u, p1, K0B_F[0] - p2) * rs, k1 = fmaf(u, q1, K1B_F[0] - q2) * rs;
    return k0 + (2.0f / x) * k1;
  }
  return (float)fv::lhrg_K2((double)x);
}

struct PrimF { float T, mu, ux, uy, n, e, P, cs2, nux, nuy, Pi, pixx, pixy, piyy, pieta; };
struct PiCF { float tt, tx, ty, xx, xy, yy; };

__device__ __forceinline__ PiCF shear_tensor_f(float ux, float uy, float ut, float pixx, float pixy, float piyy) {
  const float iu = safe_invf(ut);
  const float tx = ((ux * pixx) + (uy * pixy)) * iu;
  const float ty = ((ux * pixy) + (uy * piyy)) * iu;
  const float tt = ((ux * tx) + (uy * ty)) * iu;
  return PiCF{tt, tx, ty, pixx, pixy, piyy};
}

/* eos_Pne + eos_cs2 at one T, FP32 */
template <int EOS>
__device__ __forceinline__ void eos_Pne_cs2_f(float T, float mu, const fv::DevParams& d, float* P, float* n,
                                              float* en, float* cs2) {
  if (EOS == FIVO_EOS_CONFORMAL_HQ) {
    double Pd, nd, ed;
    fv::conformal_Pne((double)T, (double)mu, d, &Pd, &nd, &ed);
    *P = (float)Pd; *n = (float)nd; *en = (float)ed; *cs2 = 1.0f / 3.0f;
    return;
  }
  T = jmaxf(T, (float)FV_T_MIN);
  float Pl, dP, d2P;
  light_eos_f(T, d, &Pl, &dP, &d2P);
  const float el = (-Pl) + (T * dP);
  const float x = jminf((float)d.p.m_hq / T, 100000.0f);
  const bool off = !(x == x) || isinf(x) || x <= 0.0f;
  const float z = jclampf((mu - (float)d.p.m_hq) / T, -700.0f, 700.0f);
  float n_hq = (((float)d.A_lhrg * T) * expf(z)) * (off ? 0.0f : k2x_f(x));
  if (d.p.hq_times_fmGeV3) n_hq *= (float)d.fmgev3;
  *P = Pl;
  *n = off ? 0.0f : n_hq;
  *en = el;
  *cs2 = (d2P == 0.0f) ? (1.0f / 3.0f) : (dP / (T * d2P));
}

template <int EOS>
__device__ __forceinline__ bool prim_to_cons_f(float uc[4], PrimF& pr, float T, float mu, float ux, float uy,
                                               const float dis[7], float tau, const fv::DevParams& d) {
  const float Tc = jmaxf(T, (float)FV_T_MIN);
  const float ut = utauf(ux, uy);
  float P, n, en, cs2;
  eos_Pne_cs2_f<EOS>(Tc, mu, d, &P, &n, &en, &cs2);
  pr.T = Tc; pr.mu = mu;
  pr.nux = dis[0]; pr.nuy = dis[1]; pr.Pi = dis[2]; pr.pixx = dis[3]; pr.pixy = dis[4]; pr.piyy = dis[5];
  pr.pieta = dis[6];
  if (!(isfinite(P) && isfinite(n) && isfinite(en)) || en <= 0.0f) {
    pr.ux = 0.0f; pr.uy = 0.0f; pr.n = 0.0f; pr.e = 0.0f; pr.P = 0.0f; pr.cs2 = cs2;
    return false;
  }
  const float weff = (en + P) + dis[2];
  const float Ptot = P + dis[2];
  const PiCF pc = shear_tensor_f(ux, uy, ut, dis[3], dis[4], dis[5]);
  const float Jt = (n * ut) + ((ux * dis[0]) + (uy * dis[1])) * safe_invf(ut);
  uc[0] = tau * Jt;
  uc[1] = ((weff * ut) * ux) + pc.tx;
  uc[2] = ((weff * ut) * uy) + pc.ty;
  uc[3] = (((weff * ut) * ut) - Ptot) + pc.tt;
  pr.ux = ux; pr.uy = uy; pr.n = n; pr.e = en; pr.P = P; pr.cs2 = cs2;
  return true;
}

template <bool XDIR>
__device__ __forceinline__ void wavespeeds_f(const PrimF& p, float pinn, float* lm, float* lp) {
  float cs2 = jclampf(p.cs2, 0.0f, 0.999f);
  const float w = p.e + p.P;
  if (w > TINY_F) cs2 = jminf(cs2 + ((fabsf(p.Pi) + fabsf(pinn)) / w), 0.999f);
  const float ut = utauf(p.ux, p.uy);
  const float iu = safe_invf(ut);
  const float vx = p.ux * iu, vy = p.uy * iu;
  const float v2 = (vx * vx) + (vy * vy);
  const float vn = XDIR ? vx : vy;
  const float den = 1.0f - (v2 * cs2);
  if (den <= TINY_F) { *lm = -1.0f; *lp = 1.0f; return; }
  const float cs = sqrtf(jmaxf(cs2, 0.0f));
  const float rad = (1.0f - v2) * (den - ((vn * vn) * (1.0f - cs2)));
  const float disc = cs * sqrtf(jmaxf(rad, 0.0f));
  *lm = jclampf(((vn * (1.0f - cs2)) - disc) / den, -1.0f, 1.0f);
  *lp = jclampf(((vn * (1.0f - cs2)) + disc) / den, -1.0f, 1.0f);
}

/* the conserved four rows of flux_cell_2d! and the normal velocity */
template <bool XDIR>
__device__ __forceinline__ void flux_cons4_f(float F[4], const PrimF& p, float tau, float* vn) {
  const float ux = p.ux, uy = p.uy, ut = utauf(ux, uy), iu = safe_invf(ut);
  const float vx = ux * iu, vy = uy * iu;
  const float Ptot = p.P + p.Pi, weff = (p.e + p.P) + p.Pi;
  const PiCF pc = shear_tensor_f(ux, uy, ut, p.pixx, p.pixy, p.piyy);
  const float Jx = (p.n * ux) + p.nux, Jy = (p.n * uy) + p.nuy;
  float v;
  if (XDIR) {
    F[0] = tau * Jx; F[1] = (((weff * ux) * ux) + Ptot) + pc.xx; F[2] = ((weff * ux) * uy) + pc.xy;
    F[3] = ((weff * ut) * ux) + pc.tx; v = vx;
  } else {
    F[0] = tau * Jy; F[1] = ((weff * ux) * uy) + pc.xy; F[2] = (((weff * uy) * uy) + Ptot) + pc.yy;
    F[3] = ((weff * ut) * uy) + pc.ty; v = vy;
  }
  *vn = v;
}

/* face_flux_pair in FP32 (two lanes per face; see kernels.cuh) */
template <int EOS, bool XDIR>
__device__ __forceinline__ float face_flux_pair_f(const fv::DevParams& d, const fv::DevState& U, const fv::DevPrims& w,
                                                  long long i, long long st, int k, int kmax, double tau_d,
                                                  const uint8_t* ffo, int side, float* Fh) {
  const long long ip = i + st;
  const long long c0 = side ? ip : i;
  const unsigned pm = 3u << (threadIdx.x & 30);
  const int ng = d.ng;
  const float tau = (float)tau_d;
  double disd[7];
  fv::load_dis(d, U, c0, disd);
  float dis[7];
#pragma unroll
  for (int q = 0; q < 7; ++q) dis[q] = (float)disd[q];
  const bool forced = ffo != nullptr && (ffo[i] || ffo[ip]);
  PrimF p;
  float uc[4];
  bool good = false, floored = false;
  if (!forced) {
    float v[4];
    const double* fld[4] = {w.yT, w.phi, w.ux, w.uy};
    const bool first = (k + 1 <= ng) || (k + 1 >= kmax - ng);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const double* f = fld[q];
      const float c = (float)f[c0];
      if (first) { v[q] = c; continue; }
      const float a = (float)(side ? f[i] : f[i - st]);
      const float b = (float)(side ? f[ip + st] : f[ip]);
      const float h = 0.5f * mc_limiter_f(c - a, b - c);
      const float val = side ? c - h : c + h;
      v[q] = jclampf(val, jminf(jminf(a, c), b), jmaxf(jmaxf(a, c), b));
    }
    const float T = expf(v[0]);
    const float mu = (float)d.p.m_hq + (T * v[1]);
    const bool ok = prim_to_cons_f<EOS>(uc, p, T, mu, v[2], v[3], dis, tau, d);
    const bool mine = ok && uc[0] >= 0.0f && uc[3] >= (float)FV_E_FLOOR;
    const int theirs = __shfl_xor_sync(pm, (int)mine, 1);
    good = mine && theirs;
  }
  if (!good) {
    const float Tc = (float)fx::fx_exp(w.yT[c0]), muc = (float)w.mu[c0];
    const bool ok = prim_to_cons_f<EOS>(uc, p, Tc, muc, (float)w.ux[c0], (float)w.uy[c0], dis, tau, d);
    const int theirs = __shfl_xor_sync(pm, (int)ok, 1);
    if (!(ok && theirs) && !ok) {
      floored = true;
      uc[0] = 0.0f; uc[1] = 0.0f; uc[2] = 0.0f; uc[3] = (float)FV_E_FLOOR;
      p.T = (float)FV_T_MIN; p.mu = 0.0f; p.ux = 0.0f; p.uy = 0.0f; p.n = 0.0f; p.e = (float)FV_E_FLOOR; p.P = 0.0f;
      p.nux = p.nuy = p.Pi = p.pixx = p.pixy = p.piyy = p.pieta = 0.0f;
    }
  }
  if (floored) p.cs2 = (float)fv::eos_cs2<EOS>(FV_T_MIN, d);
  float F4[4], v;
  flux_cons4_f<XDIR>(F4, p, tau, &v);
  float lm, lp;
  wavespeeds_f<XDIR>(p, XDIR ? p.pixx : p.piyy, &lm, &lp);
  const float lmo = __shfl_xor_sync(pm, lm, 1), lpo = __shfl_xor_sync(pm, lp, 1);
  const float lmL = side ? lmo : lm, lmR = side ? lm : lmo;
  const float lpL = side ? lpo : lp, lpR = side ? lp : lpo;
  const float sL = jminf(lmL, lmR), sR = jmaxf(lpL, lpR);
  const bool an = d.hasNu && d.p.advect_nu, aP = d.hasPi && d.p.advect_Pi, ap = d.hasShear && d.p.advect_pi;
  const float inv = 1.0f / ((sR - sL) + TINY_F);
#pragma unroll
  for (int s = 0; s < 11; ++s) {
    /* row s: conserved column and flux (advected rows = stored dissipative * v) */
    float cs, Fs;
    if (s < 4) { cs = uc[s]; Fs = F4[s]; }
    else {
      cs = floored ? 0.0f : dis[s - 4];
      const bool adv = s < 6 ? an : (s == 6 ? aP : ap);
      Fs = adv ? cs * v : 0.0f;
    }
    const float Fo = __shfl_xor_sync(pm, Fs, 1);
    const float co = __shfl_xor_sync(pm, cs, 1);
    const float FLs = side ? Fo : Fs, FRs = side ? Fs : Fo;
    const float cls = side ? co : cs, crs = side ? cs : co;
    float h;
    if (sL >= 0.0f) h = FLs;
    else if (sR <= 0.0f) h = FRs;
    else h = (((sR * FLs) - (sL * FRs)) + ((sR * sL) * (crs - cls))) * inv;
    const int a = fv::plane_of(d, s);
    if (Fh && a >= 0 && (a & 1) == side) Fh[(size_t)a * d.Ntot + i] = h;
  }
  return jmaxf(fabsf(sL), fabsf(sR));
}

template <int EOS, bool XDIR>
__device__ __forceinline__ void faces32_body(const fv::DevParams& d, const fv::DevState& Ub, const fv::DevPrims& w,
                                             double tau, const uint8_t* ffo, float* Fh, fv::DevFlags* fl,
                                             long long t) {
  const long long nf = XDIR ? (long long)(d.Nxtot - 1) * d.Nytot : (long long)d.Nxtot * (d.Nytot - 1);
  const int side = (int)(t & 1);
  long long f = t >> 1;
  const bool valid = f < nf;
  if (!valid) f = nf - 1;
  long long i;
  int k, kmax;
  if (XDIR) { i = f; k = (int)(f / d.Nytot); kmax = d.Nxtot; }
  else {
    const int ix = (int)(f / (d.Nytot - 1)), iy = (int)(f % (d.Nytot - 1));
    i = (long long)ix * d.Nytot + iy; k = iy; kmax = d.Nytot;
  }
  float amax = face_flux_pair_f<EOS, XDIR>(d, Ub, w, i, XDIR ? d.Nytot : 1, k, kmax, tau, ffo, side,
                                            valid ? Fh : nullptr);
  for (int o = 16; o > 0; o >>= 1) amax = jmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  __shared__ float red[4];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
  __syncthreads();
  if (threadIdx.x == 0) {
    const float m = jmaxf(jmaxf(red[0], red[1]), jmaxf(red[2], red[3]));
    fv::atomic_max_pos(&fl->amax_bits, (double)m);
  }
}

template <int EOS, bool XDIR>
__global__ void __launch_bounds__(128, 8) k_faces32(fv::DevParams d, fv::DevState Ub, fv::DevPrims w, double tau,
                                                   const uint8_t* ffo, float* Fh, fv::DevFlags* fl) {
  faces32_body<EOS, XDIR>(d, Ub, w, tau, ffo, Fh, fl, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

}  // namespace f32
