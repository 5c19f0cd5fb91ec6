/*
 * guess.cuh — the learned starting guess of the primitive recovery: an MLP
 * 8 -> 64 -> 64 -> 3 (GELU), BF16 weights and activations on the tensor cores
 * with FP32 accumulation in tensor memory, mapping a cell's normalised
 * conserved and dissipative components to (log T, u^x, u^y). The charm
 * chemical potential of the guess then follows in closed form from N^tau, so
 * the Newton iteration of cons_to_prim_2d! (src2d/primrec2d.jl:465-742) starts
 * next to its root in all four unknowns.
 *
 * Everything the network needs is here: the feature map, the forward tile
 * shared by inference and training, the training kernel (forward and backward
 * for 128 samples per CTA on the tensor cores, one set of partial gradients per
 * CTA), Adam over the summed partials, the packing of the FP32 master weights
 * into BF16 operand images, and the harvest of (features, primitives) pairs
 * from a solver's own recovered states. The recovery kernel that uses the guess
 * is k_prim_learned (kernels.cuh).
 */
#pragma once
#include <cuda_bf16.h>
#include "tc05.cuh"

namespace guess {

constexpr int NIN = 8, K0 = 16, NH = 64, NOUT = 3, N3 = 16;
constexpr int NSAMP = NIN + NOUT;                  /* floats per training sample */
/* flat FP32 parameter vector: W1[64][16] b1[64] W2[64][64] b2[64] W3[16][64] b3[16]
 * (W[out][in]); the padding columns of W1 and rows of W3 stay zero */
constexpr int P_W1 = 0, P_B1 = P_W1 + NH * K0, P_W2 = P_B1 + NH, P_B2 = P_W2 + NH * NH, P_W3 = P_B2 + NH,
              P_B3 = P_W3 + N3 * NH, NPARAM = P_B3 + N3;
/* BF16 operand images, canonical K-major (tc05.cuh): W1 (64 x 16), W2 (64 x 64),
 * W3 (16 x 64), and for the backward pass W3^T (64 x 16), W2^T (64 x 64) */
constexpr int I_W1 = 0, I_W2 = I_W1 + NH * K0 * 2, I_W3 = I_W2 + NH * NH * 2, I_W3T = I_W3 + N3 * NH * 2,
              I_W2T = I_W3T + NH * K0 * 2, IMG_BYTES = I_W2T + NH * NH * 2;
constexpr uint32_t WAIT_LIMIT = 1u << 22;          /* mbarrier polls before a wait gives up */

/* input / output normalisation: x_n = (r - mean) * istd, r_out = y_n * std + mean */
struct Norm { float in_mean[NIN], in_istd[NIN], out_mean[NOUT], out_std[NOUT]; };

struct Net {
  const uint8_t* img;     /* IMG_BYTES of BF16 operand images */
  const float* params;    /* NPARAM FP32 master weights (the biases are read from here) */
  Norm norm;
};

/* raw features of a non-vacuum cell (E > 0): log E, S/E, Pi/E, pi^{ij}/E, |S|/E */
FX_HD void features(double E, double Sx, double Sy, double Pi, double pixx, double pixy, double piyy,
                    float r[NIN]) {
  const double iE = 1.0 / E;
  r[0] = (float)log(E);
  r[1] = (float)(Sx * iE);
  r[2] = (float)(Sy * iE);
  r[3] = (float)(Pi * iE);
  r[4] = (float)(pixx * iE);
  r[5] = (float)(pixy * iE);
  r[6] = (float)(piyy * iE);
  r[7] = (float)(sqrt(Sx * Sx + Sy * Sy) * iE);
}
/* the regression targets: log T relative to the conformal scaling E^(1/4), u^x, u^y */
FX_HD void targets(double yT, double ux, double uy, double E, float t[NOUT]) {
  t[0] = (float)(yT - 0.25 * log(E));
  t[1] = (float)ux;
  t[2] = (float)uy;
}

/* splitmix64: the hash of the sample draws and the seeded initial weights */
FX_HD uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

#if defined(__CUDACC__)

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}
__device__ __forceinline__ uint32_t pack2(float a, float b) {
  return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(a)) |
         ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(b)) << 16);
}
/* row r of a canonical tile of R rows, columns k0 .. k0+7 from v[0..7] (one 16-byte store) */
__device__ __forceinline__ void st_row8(uint8_t* tile, uint32_t R, uint32_t r, uint32_t k0, const float* v) {
  uint4 q;
  q.x = pack2(v[0], v[1]); q.y = pack2(v[2], v[3]); q.z = pack2(v[4], v[5]); q.w = pack2(v[6], v[7]);
  *reinterpret_cast<uint4*>(tile + tc05::kmaj_off(R, r, k0)) = q;
}
/* element (r, k) of a canonical tile */
__device__ __forceinline__ void st_el(uint8_t* tile, uint32_t R, uint32_t r, uint32_t k, float v) {
  *reinterpret_cast<__nv_bfloat16*>(tile + tc05::kmaj_off(R, r, k)) = __float2bfloat16_rn(v);
}
__device__ __forceinline__ void copy16(uint8_t* dst, const uint8_t* src, int bytes, int tid, int nthr) {
  for (int o = tid * 16; o < bytes; o += nthr * 16)
    *reinterpret_cast<uint4*>(dst + o) = *reinterpret_cast<const uint4*>(src + o);
}
__device__ __forceinline__ uint32_t lane_addr(uint32_t tbase, int warp, uint32_t col) {
  return tbase + ((uint32_t)(32 * warp) << 16) + col;
}

/* Shared memory of the forward tile (inference). */
struct FwdSmem {
  uint8_t X[128 * K0 * 2];      /* A of layer 1 */
  uint8_t H[128 * NH * 2];      /* A of layers 2 and 3 (H1, then H2) */
  uint8_t W1[NH * K0 * 2];
  uint8_t W2[NH * NH * 2];
  uint8_t W3[N3 * NH * 2];
  uint64_t mbar;
  uint32_t tbase;
  int err;
};

/* One issue of a chain of MMAs by thread 0 after all threads' operand writes,
 * then the wait of every thread for its completion. Returns false when the wait
 * gave up (the caller skips the epilogue and unwinds). */
__device__ __forceinline__ bool run_chain(uint64_t* mbar, uint32_t& phase, uint32_t d_tmem, uint32_t a_saddr,
                                          uint32_t a_rows, uint32_t b_saddr, uint32_t b_rows, uint32_t nk16,
                                          uint32_t n, bool commit) {
  if (threadIdx.x == 0) {
    tc05::fence_after_sync();
    const uint32_t id = tc05::idesc_bf16_f32(128, n);
    for (uint32_t k = 0; k < nk16; ++k)
      tc05::mma_bf16(d_tmem, tc05::tile_desc(a_saddr, a_rows, k), tc05::tile_desc(b_saddr, b_rows, k), id,
                     k > 0 ? 1u : 0u);
    if (commit) tc05::mma_commit(mbar);
  }
  if (!commit) return true;
  const bool ok = tc05::mbar_wait(mbar, phase, WAIT_LIMIT);
  phase ^= 1u;
  tc05::fence_after_sync();
  return ok;
}
/* operand writes (generic proxy) made visible to the MMA, and every thread's
 * tensor-memory reads finished, before thread 0 issues the next chain */
__device__ __forceinline__ void to_mma() {
  tc05::fence_smem_to_async();
  tc05::fence_before_sync();
  __syncthreads();
}

/* Forward pass of the 128 rows of a CTA of 128 threads: row t = threadIdx.x,
 * normalised features xn[8] in, normalised outputs y[3] out. Every thread of the
 * CTA must call it. Tensor memory: 128 columns (layer 1 in 0-63, layer 2 in
 * 64-127, layer 3 again in 0-15). Returns false when a wait gave up (then y is
 * not set and the tensor memory is freed all the same). */
__device__ __forceinline__ bool forward_tile(FwdSmem& s, const Net& net, const float xn[NIN], float y[NOUT]) {
  const int t = threadIdx.x, warp = t >> 5;
  if (warp == 0) { tc05::tmem_alloc(&s.tbase, 128); tc05::tmem_relinquish(); }
  if (t == 0) { tc05::mbar_init(&s.mbar, 1); s.err = 0; }
  copy16(s.W1, net.img + I_W1, NH * K0 * 2, t, 128);
  copy16(s.W2, net.img + I_W2, NH * NH * 2, t, 128);
  copy16(s.W3, net.img + I_W3, N3 * NH * 2, t, 128);
  {
    float v[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = xn[q];
    st_row8(s.X, 128, t, 0, v);
#pragma unroll
    for (int q = 0; q < 8; ++q) v[q] = 0.0f;
    st_row8(s.X, 128, t, 8, v);
  }
  to_mma();
  tc05::fence_after_sync();
  const uint32_t tb = s.tbase;
  uint32_t phase = 0;
  bool ok = run_chain(&s.mbar, phase, tb, tc05::smem_u32(s.X), 128, tc05::smem_u32(s.W1), NH, 1, NH, true);
  ok = __syncthreads_and(ok);
  const float* b1 = net.params + P_B1;
  const float* b2 = net.params + P_B2;
  const float* b3 = net.params + P_B3;
  if (ok) {
#pragma unroll
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tc05::tmem_ld16(lane_addr(tb, warp, c), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = gelu(v[q] + b1[c + q]);
      st_row8(s.H, 128, t, c, v);
      st_row8(s.H, 128, t, c + 8, v + 8);
    }
  }
  to_mma();
  if (ok) ok = run_chain(&s.mbar, phase, tb + 64, tc05::smem_u32(s.H), 128, tc05::smem_u32(s.W2), NH, 4, NH, true);
  ok = __syncthreads_and(ok);
  /* every thread has read layer 2 before H is overwritten: the MMA that read H has completed */
  if (ok) {
#pragma unroll
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tc05::tmem_ld16(lane_addr(tb, warp, 64 + c), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = gelu(v[q] + b2[c + q]);
      st_row8(s.H, 128, t, c, v);
      st_row8(s.H, 128, t, c + 8, v + 8);
    }
  }
  to_mma();
  if (ok) ok = run_chain(&s.mbar, phase, tb, tc05::smem_u32(s.H), 128, tc05::smem_u32(s.W3), N3, 4, N3, true);
  ok = __syncthreads_and(ok);
  if (ok) {
    float v[16];
    tc05::tmem_ld16(lane_addr(tb, warp, 0), v);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) y[o] = v[o] + b3[o];
  }
  if (!ok && t == 0) s.err = 1;
  tc05::fence_before_sync();
  __syncthreads();
  const bool all_ok = s.err == 0;
  if (warp == 0) { tc05::fence_after_sync(); tc05::tmem_dealloc(tb, 128); }
  return all_ok;
}

/* ---- training: 128 samples per CTA, forward and backward on the tensor cores ---- */
struct TrainSmem {
  uint8_t X[128 * K0 * 2];          /* A of fwd 1 */
  uint8_t W1[NH * K0 * 2];
  uint8_t H1[128 * NH * 2];         /* A of fwd 2 */
  uint8_t W2[NH * NH * 2];
  uint8_t H2[128 * NH * 2];         /* A of fwd 3 */
  uint8_t W3[N3 * NH * 2];
  uint8_t dY[128 * N3 * 2];         /* A of dH2 = dY W3 */
  uint8_t W3T[NH * N3 * 2];
  uint8_t dZ2[128 * NH * 2];        /* A of dH1 = dZ2 W2 */
  uint8_t W2T[NH * NH * 2];
  uint8_t AS[128 * 128 * 2];        /* [dZ2^T; dZ1^T], then [H2^T; 0]: A of the weight gradients */
  uint8_t BS[80 * 128 * 2];         /* [H1^T; X^T]: B of dW2 and dW1 */
  uint8_t BY[N3 * 128 * 2];         /* dY^T: B of dW3^T */
  float Z1[128][NH + 1];            /* pre-activations of layers 1, 2 (padded rows) */
  float Z2[128][NH + 1];
  float gb3[4][N3];                 /* per-warp sums of dY (bias of layer 3) */
  float lossw[4];                   /* per-warp sums of the squared error */
  uint64_t mbar;
  uint32_t tbase;
};

/* TMEM columns of the training kernel (512 allocated; one CTA per SM) */
constexpr uint32_t TC_D1 = 0, TC_D2 = 64, TC_D3 = 128, TC_DH2 = 144, TC_DH1 = 208, TC_GA = 272, TC_GB = 352;

__device__ __forceinline__ float nrm_in(const Norm& nm, int q, float r) {
  return fminf(fmaxf((r - nm.in_mean[q]) * nm.in_istd[q], -8.0f), 8.0f);
}

/* 128 samples per CTA (row t = threadIdx.x; sample (start + 128 b + t) mod n in
 * order when seed == 0, else a seeded hash of that position mod n):
 * the forward pass, the mean-squared error of the normalised outputs and its
 * gradient with respect to every parameter, written as this CTA's partial sums
 * part[b][NPARAM] (the caller sums them over b); loss_part[b] = the CTA's sum of
 * squared errors. inv_batch = 1 / (samples of the whole step). */
__global__ void __launch_bounds__(128, 1) k_train(Net net, const float* __restrict__ samples,
                                                  long long n, unsigned long long seed, long long start,
                                                  float inv_batch, float* __restrict__ part,
                                                  float* __restrict__ loss_part, int* err) {
  extern __shared__ __align__(128) uint8_t smem_raw[];
  TrainSmem& s = *reinterpret_cast<TrainSmem*>(smem_raw);
  const int t = threadIdx.x, warp = t >> 5;
  if (warp == 0) { tc05::tmem_alloc(&s.tbase, 512); tc05::tmem_relinquish(); }
  if (t == 0) tc05::mbar_init(&s.mbar, 1);
  copy16(s.W1, net.img + I_W1, NH * K0 * 2, t, 128);
  copy16(s.W2, net.img + I_W2, NH * NH * 2, t, 128);
  copy16(s.W3, net.img + I_W3, N3 * NH * 2, t, 128);
  copy16(s.W3T, net.img + I_W3T, NH * N3 * 2, t, 128);
  copy16(s.W2T, net.img + I_W2T, NH * NH * 2, t, 128);
  const long long gi = start + (long long)blockIdx.x * 128 + t;
  const unsigned long long ks = seed == 0 ? (unsigned long long)gi % (unsigned long long)n
                                           : mix64(seed ^ (unsigned long long)gi) % (unsigned long long)n;
  const float* smp = samples + (size_t)ks * NSAMP;
  float xn[8], tn[NOUT];
#pragma unroll
  for (int q = 0; q < NIN; ++q) xn[q] = nrm_in(net.norm, q, smp[q]);
#pragma unroll
  for (int o = 0; o < NOUT; ++o) tn[o] = (smp[NIN + o] - net.norm.out_mean[o]) / net.norm.out_std[o];
  {
    float z8[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    st_row8(s.X, 128, t, 0, xn);
    st_row8(s.X, 128, t, 8, z8);
    /* X^T: rows 64 .. 79 of BS, column t */
#pragma unroll
    for (int k = 0; k < K0; ++k) st_el(s.BS, 80, 64 + k, t, k < NIN ? xn[k] : 0.0f);
  }
  to_mma();
  tc05::fence_after_sync();
  const uint32_t tb = s.tbase;
  uint32_t ph = 0;
  const float* b1 = net.params + P_B1;
  const float* b2 = net.params + P_B2;
  const float* b3 = net.params + P_B3;
  bool ok = run_chain(&s.mbar, ph, tb + TC_D1, tc05::smem_u32(s.X), 128, tc05::smem_u32(s.W1), NH, 1, NH, true);
  ok = __syncthreads_and(ok);
  if (ok) {
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tc05::tmem_ld16(lane_addr(tb, warp, TC_D1 + c), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float z = v[q] + b1[c + q];
        s.Z1[t][c + q] = z;
        v[q] = gelu(z);
        st_el(s.BS, 80, c + q, t, v[q]);                /* H1^T: rows 0 .. 63 of BS */
      }
      st_row8(s.H1, 128, t, c, v);
      st_row8(s.H1, 128, t, c + 8, v + 8);
    }
  }
  to_mma();
  if (ok) ok = run_chain(&s.mbar, ph, tb + TC_D2, tc05::smem_u32(s.H1), 128, tc05::smem_u32(s.W2), NH, 4, NH, true);
  ok = __syncthreads_and(ok);
  if (ok) {
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tc05::tmem_ld16(lane_addr(tb, warp, TC_D2 + c), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float z = v[q] + b2[c + q];
        s.Z2[t][c + q] = z;
        v[q] = gelu(z);
      }
      st_row8(s.H2, 128, t, c, v);
      st_row8(s.H2, 128, t, c + 8, v + 8);
    }
  }
  to_mma();
  if (ok) ok = run_chain(&s.mbar, ph, tb + TC_D3, tc05::smem_u32(s.H2), 128, tc05::smem_u32(s.W3), N3, 4, N3, true);
  ok = __syncthreads_and(ok);
  float dy[N3];
  float se = 0.0f;
#pragma unroll
  for (int o = 0; o < N3; ++o) dy[o] = 0.0f;
  if (ok) {
    float v[16];
    tc05::tmem_ld16(lane_addr(tb, warp, TC_D3), v);
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      const float e = (v[o] + b3[o]) - tn[o];
      se += e * e;
      dy[o] = 2.0f * e * inv_batch;
    }
  }
  st_row8(s.dY, 128, t, 0, dy);
  st_row8(s.dY, 128, t, 8, dy + 8);
#pragma unroll
  for (int o = 0; o < N3; ++o) st_el(s.BY, N3, o, t, dy[o]);   /* dY^T */
  /* per-warp sums of the squared error and of dY (bias of layer 3), in a fixed order */
  for (int o = 16; o > 0; o >>= 1) se += __shfl_xor_sync(0xffffffffu, se, o);
#pragma unroll
  for (int q = 0; q < NOUT; ++q) {
    float g = dy[q];
    for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
    if ((t & 31) == 0) s.gb3[warp][q] = g;
  }
  if ((t & 31) == 0) s.lossw[warp] = se;
  to_mma();
  if (ok) ok = run_chain(&s.mbar, ph, tb + TC_DH2, tc05::smem_u32(s.dY), 128, tc05::smem_u32(s.W3T), NH, 1, NH, true);
  ok = __syncthreads_and(ok);
  if (ok) {
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tc05::tmem_ld16(lane_addr(tb, warp, TC_DH2 + c), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float g = v[q] * gelu_d(s.Z2[t][c + q]);
        v[q] = g;
        s.Z2[t][c + q] = g;                             /* dZ2, kept in FP32 for the bias sum */
        st_el(s.AS, 128, c + q, t, g);                  /* dZ2^T: rows 0 .. 63 of AS */
      }
      st_row8(s.dZ2, 128, t, c, v);
      st_row8(s.dZ2, 128, t, c + 8, v + 8);
    }
  }
  to_mma();
  if (ok) ok = run_chain(&s.mbar, ph, tb + TC_DH1, tc05::smem_u32(s.dZ2), 128, tc05::smem_u32(s.W2T), NH, 4, NH, true);
  ok = __syncthreads_and(ok);
  if (ok) {
    for (int c = 0; c < NH; c += 16) {
      float v[16];
      tc05::tmem_ld16(lane_addr(tb, warp, TC_DH1 + c), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const float g = v[q] * gelu_d(s.Z1[t][c + q]);
        s.Z1[t][c + q] = g;                             /* dZ1 */
        st_el(s.AS, 128, 64 + c + q, t, g);             /* dZ1^T: rows 64 .. 127 of AS */
      }
    }
  }
  to_mma();
  /* dW2 and dW1 in one chain: [dZ2^T; dZ1^T] (128 x K=128) times [H1^T; X^T] (80 x K=128) */
  if (ok) ok = run_chain(&s.mbar, ph, tb + TC_GA, tc05::smem_u32(s.AS), 128, tc05::smem_u32(s.BS), 80, 8, 80, true);
  ok = __syncthreads_and(ok);
  float* pp = part + (size_t)blockIdx.x * NPARAM;
  if (ok) {
    if (t < 64) {          /* warps 0, 1: dW2 rows */
      for (int c = 0; c < NH; c += 16) {
        float v[16];
        tc05::tmem_ld16(lane_addr(tb, warp, TC_GA + c), v);
#pragma unroll
        for (int q = 0; q < 16; ++q) pp[P_W2 + t * NH + c + q] = v[q];
      }
    } else {               /* warps 2, 3: dW1 rows */
      float v[16];
      tc05::tmem_ld16(lane_addr(tb, warp, TC_GA + 64), v);
#pragma unroll
      for (int q = 0; q < 16; ++q) pp[P_W1 + (t - 64) * K0 + q] = v[q];
    }
  }
  /* the chain above has completed, so AS may be rewritten: rows 0 .. 63 := H2^T,
   * copied as BF16 bits from row t of the H2 tile (rows 64 .. 127 only feed
   * accumulator rows that are not read) */
  for (int j = 0; j < NH; ++j)
    *reinterpret_cast<uint16_t*>(s.AS + tc05::kmaj_off(128, j, t)) =
        *reinterpret_cast<const uint16_t*>(s.H2 + tc05::kmaj_off(128, t, j));
  to_mma();
  /* dW3^T = H2^T dY: (128 x K=128) times dY^T (16 x K=128) */
  if (ok) ok = run_chain(&s.mbar, ph, tb + TC_GB, tc05::smem_u32(s.AS), 128, tc05::smem_u32(s.BY), N3, 8, N3, true);
  ok = __syncthreads_and(ok);
  if (ok && t < 64) {
    float v[16];
    tc05::tmem_ld16(lane_addr(tb, warp, TC_GB), v);
#pragma unroll
    for (int o = 0; o < N3; ++o) pp[P_W3 + o * NH + t] = v[o];
  }
  /* bias gradients: thread j sums column j of dZ1 / dZ2 over the 128 rows, in order */
  if (t < NH) {
    float g1 = 0.0f, g2 = 0.0f;
    for (int r = 0; r < 128; ++r) { g1 += s.Z1[r][t]; g2 += s.Z2[r][t]; }
    pp[P_B1 + t] = g1;
    pp[P_B2 + t] = g2;
  }
  if (t < N3) pp[P_B3 + t] = t < NOUT ? ((s.gb3[0][t] + s.gb3[1][t]) + s.gb3[2][t]) + s.gb3[3][t] : 0.0f;
  if (t == 0) {
    loss_part[blockIdx.x] = ((s.lossw[0] + s.lossw[1]) + s.lossw[2]) + s.lossw[3];
    if (!ok) atomicExch(err, 1);
  }
  tc05::fence_before_sync();
  __syncthreads();
  if (warp == 0) { tc05::fence_after_sync(); tc05::tmem_dealloc(tb, 512); }
}

/* Adam over the summed partial gradients (summed over the CTAs in order, so a
 * training run is reproducible); the padding entries stay zero */
__device__ __forceinline__ bool is_pad(int p) {
  if (p >= P_W1 && p < P_B1) return ((p - P_W1) % K0) >= NIN;
  if (p >= P_W3 && p < P_B3) return (p - P_W3) / NH >= NOUT;
  if (p >= P_B3) return (p - P_B3) >= NOUT;
  return false;
}
__global__ void k_adam(float* __restrict__ params, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ part, int nparts, float lr, float b1, float b2, float eps,
                       float c1, float c2, float* __restrict__ grad_out) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NPARAM) return;
  float g = 0.0f;
  for (int b = 0; b < nparts; ++b) g += part[(size_t)b * NPARAM + p];
  if (grad_out) grad_out[p] = g;
  if (lr == 0.0f || is_pad(p)) return;
  const float mm = b1 * m[p] + (1.0f - b1) * g;
  const float vv = b2 * v[p] + (1.0f - b2) * g * g;
  m[p] = mm; v[p] = vv;
  params[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

/* per-block sums of each sample column and of its square (for the normalisation);
 * part[b][2 * NSAMP]; 256 threads */
__global__ void __launch_bounds__(256) k_moments(const float* __restrict__ smp, long long n, double* part) {
  __shared__ double red[256];
  double acc[2 * NSAMP];
#pragma unroll
  for (int q = 0; q < 2 * NSAMP; ++q) acc[q] = 0.0;
  for (long long k = (long long)blockIdx.x * 256 + threadIdx.x; k < n; k += (long long)gridDim.x * 256)
#pragma unroll
    for (int q = 0; q < NSAMP; ++q) {
      const double x = smp[(size_t)k * NSAMP + q];
      acc[q] += x;
      acc[NSAMP + q] += x * x;
    }
  for (int q = 0; q < 2 * NSAMP; ++q) {
    red[threadIdx.x] = acc[q];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
      if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * 2 * NSAMP + q] = red[0];
    __syncthreads();
  }
}

/* BF16 operand images from the FP32 master weights: one thread per image element */
__global__ void k_pack(const float* __restrict__ P, uint8_t* __restrict__ img) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  auto put = [&](int off, uint32_t R, uint32_t r, uint32_t k, float v) {
    *reinterpret_cast<__nv_bfloat16*>(img + off + tc05::kmaj_off(R, r, k)) = __float2bfloat16_rn(v);
  };
  int q = e;
  if (q < NH * K0) { int j = q / K0, k = q % K0; put(I_W1, NH, j, k, P[P_W1 + j * K0 + k]); return; }
  q -= NH * K0;
  if (q < NH * NH) { int j = q / NH, k = q % NH; put(I_W2, NH, j, k, P[P_W2 + j * NH + k]); return; }
  q -= NH * NH;
  if (q < N3 * NH) { int o = q / NH, k = q % NH; put(I_W3, N3, o, k, P[P_W3 + o * NH + k]); return; }
  q -= N3 * NH;
  /* W3^T: (n = j, k = o) = W3[o][j] */
  if (q < NH * N3) { int j = q / N3, o = q % N3; put(I_W3T, NH, j, o, P[P_W3 + o * NH + j]); return; }
  q -= NH * N3;
  /* W2^T: (n = k, k = j) = W2[j][k] */
  if (q < NH * NH) { int kk = q / NH, j = q % NH; put(I_W2T, NH, kk, j, P[P_W2 + j * NH + kk]); return; }
}
constexpr int PACK_ELEMS = NH * K0 + NH * NH + N3 * NH + NH * N3 + NH * NH;

/* Inference on raw features (tests and the harvest check): out[i][3] = the
 * normalised outputs of row i. Blocks of 128 threads. */
__global__ void __launch_bounds__(128) k_infer(Net net, const float* __restrict__ raw, long long n,
                                              float* __restrict__ out, int* err) {
  __shared__ __align__(128) FwdSmem s;
  const long long i = (long long)blockIdx.x * 128 + threadIdx.x;
  float xn[NIN], y[NOUT] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int q = 0; q < NIN; ++q) xn[q] = i < n ? nrm_in(net.norm, q, raw[(size_t)i * NIN + q]) : 0.0f;
  const bool ok = forward_tile(s, net, xn, y);
  if (!ok) { if (threadIdx.x == 0) atomicExch(err, 1); return; }
  if (i < n)
    for (int o = 0; o < NOUT; ++o) out[(size_t)i * NOUT + o] = y[o];
}

#endif  /* __CUDACC__ */

}  // namespace guess
