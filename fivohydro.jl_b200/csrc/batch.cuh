/* Lockstep event batches: every kernel of an SSPRK step launched ONCE over all
 * events of a batch.
 *
 * The events of a batch share the model and differ in their grids, states, time
 * steps and control flow (event-by-event hydro). In lockstep mode the host
 * takes every event's step at the same time: for each kernel of the optimistic
 * step (the stages without a host read in between) one launch covers the blocks
 * of every event, and a block learns its event from a per-shape block table.
 * The per-cell work of a block is the single-event kernel's own body
 * (prim_fast_body, faces_body, update_body, ...), called with the event's grid
 * and buffers, so every cell gets the same arithmetic on the same inputs as in
 * a separate run: results are bitwise those of fivo_run on each event.
 *
 * The deferred passes (the warp-pair recovery of the cells the fast pass left,
 * and the admissibility inversions) are persistent kernels over the union of
 * all events' queues: a one-block scan turns the per-event queue lengths into
 * offsets, and each warp (pair) takes the next item of the batch from one
 * counter, so the long serial chains of one event run beside the other events'
 * chains.
 *
 * Reference: the per-event loop these launches serve is run_sim_2d!
 * (main2D.jl:436-513) around step_ssprk2_2d! / step_ssprk3_2d!
 * (src2d/timestepper2d.jl:74-103, 148-188); the reference itself runs one
 * event at a time and spreads a grid's columns over threads (src2d/rhs2d.jl:69-74).
 */
#ifndef FIVO_BATCH_CUH
#define FIVO_BATCH_CUH

#include "kernels.cuh"
#include "face32.cuh"
#include "relax32.cuh"

namespace fv {
namespace bt {

/* the units one 128-thread block covers, per event: cells of the whole grid,
 * ghost cells, x-face lane pairs, y-face lane pairs, interior cells, and both
 * face directions in one launch (the event's x-face blocks, then its y-face blocks) */
enum { SH_CELL = 0, SH_FRAME = 1, SH_FACEX = 2, SH_FACEY = 3, SH_INT = 4, SH_FACEXY = 5, NSHAPE = 6 };

/* an event's grid (the DevParams fields that differ between events) and the
 * first block of the event in each shape's launch */
struct Geo {
  int Nx, Ny, Nxtot, Nytot;
  long long Ntot;
  double dx, dy, xmin, ymin;
  int b0[NSHAPE];
  int nbx;                  /* x-face blocks of the event (the first ones of its SH_FACEXY range) */
};

/* one event's arguments for a step and for the pass after it (host-built) */
struct Ev {
  int active;               /* 0: every launch skips the event */
  int snap;                 /* the step starts with k_snapshot's copy */
  int spec;                 /* the post-step pass follows in the same sequence: save the
                               history planes it overwrites (for an undone step) */
  DevPrims w;
  DevHist h;
  DevFlags* fl;
  unsigned int* qp;         /* deferred recoveries */
  unsigned int* qa;         /* deferred admissibility inversions */
  unsigned int* qq;         /* what the learned retry leaves for the full recovery */
  double* fhx;
  double* fhy;
  float* fhx32;
  float* fhy32;
  double* x0save;           /* the warm starts before the step */
  double* hsave;            /* ux_prev, uy_prev, nux_prev, nuy_prev before the step */
  DevState cp_dst, cp_src;  /* copy_state(U2 <- U) before the step */
  StageArgs st[3];          /* the step's stages */
  DevState pU[4];           /* recovery input: stage 0..2's Ub; 3 = the step's result */
  double ptau[4];
  DevState rq, ro;          /* relaxation input and output */
  double rtau, rD;
  int do_relax, do_project;
};

/* batch-wide control of a deferred pass */
struct Ctl {
  unsigned int total, next;
};

__device__ __forceinline__ void with_geo(DevParams& d, const Geo& g) {
  d.Nx = g.Nx; d.Ny = g.Ny; d.Nxtot = g.Nxtot; d.Nytot = g.Nytot; d.Ntot = g.Ntot;
  d.dx = g.dx; d.dy = g.dy; d.xmin = g.xmin; d.ymin = g.ymin;
}

/* block-wide copy of a POD (multiple of 8 bytes) into shared memory; the caller syncs */
template <class T>
__device__ __forceinline__ void to_shared(T* dst, const T* src) {
  static_assert(sizeof(T) % 8 == 0, "8-byte multiple");
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* o = reinterpret_cast<unsigned long long*>(dst);
  for (int k = threadIdx.x; k < (int)(sizeof(T) / 8); k += blockDim.x) o[k] = s[k];
}

/* The block's event (from the shape's block table) and its block index within
 * the event; the event's grid and `active` land in shared memory. Returns false
 * (uniformly over the block) when the event sits this launch out. */
struct BlockHead {
  Geo g;
  int e, active;
};

__device__ __forceinline__ bool block_head(BlockHead* sh, const Geo* geo, const Ev* tab, const unsigned short* eob,
                                           int shape, long long* blk) {
  const int e = eob[blockIdx.x];
  to_shared(&sh->g, &geo[e]);
  if (threadIdx.x == 0) { sh->e = e; sh->active = tab[e].active; }
  __syncthreads();
  *blk = (long long)blockIdx.x - sh->g.b0[shape];
  return sh->active != 0;
}

/* ----------------------------------------------------------------- kernels */

/* per event, before the step: k_snapshot (when due), save_warm (x0 -> x0save),
 * copy_state (U2 <- U) and, when the post-step pass follows in the same
 * sequence, the history planes it overwrites (-> hsave), fused over the cells
 * (disjoint data) */
__global__ void __launch_bounds__(128) kb_pre_step(DevParams d0, const Geo* __restrict__ geo,
                                                   const Ev* __restrict__ tab, const unsigned short* __restrict__ eob) {
  __shared__ BlockHead sh;
  __shared__ DevState sdst, ssrc;
  __shared__ DevPrims sw;
  __shared__ DevHist shh;
  __shared__ double* sx0;
  __shared__ double* shs;
  __shared__ int ssnap, sspec;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, SH_CELL, &blk)) return;
  const Ev& ev = tab[sh.e];
  to_shared(&sdst, &ev.cp_dst);
  to_shared(&ssrc, &ev.cp_src);
  to_shared(&sw, &ev.w);
  to_shared(&shh, &ev.h);
  if (threadIdx.x == 0) { sx0 = ev.x0save; shs = ev.hsave; ssnap = ev.snap; sspec = ev.spec; }
  __syncthreads();
  const long long N = sh.g.Ntot;
  const long long i = blk * 128 + threadIdx.x;
  if (i >= N) return;
  if (ssnap) snapshot_cell(sw, shh, i);
  sx0[i] = shh.x0_yT[i]; sx0[N + i] = shh.x0_phi[i]; sx0[2 * N + i] = shh.x0_ux[i]; sx0[3 * N + i] = shh.x0_uy[i];
  if (sspec) {
    shs[i] = shh.ux_prev[i]; shs[N + i] = shh.uy_prev[i]; shs[2 * N + i] = shh.nux_prev[i];
    shs[3 * N + i] = shh.nuy_prev[i];
  }
  for (int a = 0; a < d0.nv; ++a) sdst.f[a][i] = ssrc.f[a][i];
}

/* k_reset_flags on every active event (one thread per event) */
__global__ void kb_reset(const Ev* __restrict__ tab, int nev, int what) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < nev && tab[e].active) reset_flags_dev(tab[e].fl, what, 0ULL);
}

/* apply_bc_2d! on a state of each event: which = 0 stage 0's input, 1..3 stage
 * which-1's output */
__global__ void __launch_bounds__(128) kb_bc(DevParams d0, const Geo* __restrict__ geo, const Ev* __restrict__ tab,
                                             const unsigned short* __restrict__ eob, int which, int bc) {
  __shared__ BlockHead sh;
  __shared__ DevState sU;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, SH_FRAME, &blk)) return;
  const Ev& ev = tab[sh.e];
  to_shared(&sU, which == 0 ? &ev.st[0].Ub : &ev.st[which - 1].Uout);
  __syncthreads();
  DevParams d = d0;
  with_geo(d, sh.g);
  bc_body(d, sU, bc, blk * 128 + threadIdx.x);
}

/* the fast recovery pass on each event's state pU[which] */
template <int EOS, bool NCH>
__global__ void __launch_bounds__(128, FV_FAST_MINB) kb_prim_fast(DevParams d0, const Geo* __restrict__ geo,
                                                                  const Ev* __restrict__ tab,
                                                                  const unsigned short* __restrict__ eob, int which) {
  __shared__ BlockHead sh;
  __shared__ DevState sU;
  __shared__ DevPrims sw;
  __shared__ DevHist shh;
  __shared__ DevFlags* sfl;
  __shared__ unsigned int* sq;
  __shared__ double stau;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, SH_CELL, &blk)) return;
  const Ev& ev = tab[sh.e];
  to_shared(&sU, &ev.pU[which]);
  to_shared(&sw, &ev.w);
  to_shared(&shh, &ev.h);
  if (threadIdx.x == 0) { sfl = ev.fl; sq = ev.qp; stau = ev.ptau[which]; }
  __syncthreads();
  DevParams d = d0;
  with_geo(d, sh.g);
  prim_fast_body<EOS, NCH>(d, sU, sw, shh, stau, sfl, sq, blk * 128 + threadIdx.x);
}

/* the warm pass with the learned guess in front of it (k_prim_learned) on each
 * event's state pU[which]; one tensor-core tile per block (128 cells of one event) */
template <int EOS, bool NCH>
__global__ void __launch_bounds__(128, 4) kb_prim_learned(DevParams d0, const Geo* __restrict__ geo,
                                                        const Ev* __restrict__ tab,
                                                        const unsigned short* __restrict__ eob, int which,
                                                        guess::Net net) {
  __shared__ __align__(128) guess::FwdSmem s;
  __shared__ BlockHead sh;
  __shared__ DevState sU;
  __shared__ DevPrims sw;
  __shared__ DevHist shh;
  __shared__ DevFlags* sfl;
  __shared__ unsigned int* sq;
  __shared__ double stau;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, SH_CELL, &blk)) return;
  const Ev& ev = tab[sh.e];
  to_shared(&sU, &ev.pU[which]);
  to_shared(&sw, &ev.w);
  to_shared(&shh, &ev.h);
  if (threadIdx.x == 0) { sfl = ev.fl; sq = ev.qp; stau = ev.ptau[which]; }
  __syncthreads();
  DevParams d = d0;
  with_geo(d, sh.g);
  prim_learned_body<EOS, NCH>(d, sU, sw, shh, stau, sfl, sq, net, s, blk * 128 + threadIdx.x);
}

/* Offsets of every active event's queue in the batch's union of queues; pre[nev] =
 * total. kind 0: deferred recoveries (counted into tot_p, as k_prim_slow counts
 * them), 1: admissibility inversions (into tot_a), 2: the learned retry's leftovers
 * (into tot_p), 3: deferred recoveries without counting (the learned retry takes
 * them; k_prim_learned_retry counts nothing). One block. */
__global__ void __launch_bounds__(1024) kb_scan(const Ev* __restrict__ tab, int nev, int kind, unsigned int* pre,
                                                Ctl* ctl) {
  __shared__ unsigned int s_warp[32];
  __shared__ unsigned int s_carry;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int base = 0; base < nev; base += blockDim.x) {
    const int e = base + threadIdx.x;
    unsigned int cnt = 0;
    if (e < nev && tab[e].active) {
      DevFlags* fl = tab[e].fl;
      cnt = *(volatile unsigned int*)(kind == 1 ? &fl->qcount_a : (kind == 2 ? &fl->qcount_q : &fl->qcount_p));
      if (cnt && kind != 3) atomicAdd(kind == 1 ? &fl->tot_a : &fl->tot_p, (unsigned long long)cnt);
    }
    /* inclusive scan in the warp, then over the warps' totals */
    unsigned int v = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    if (lane == 31) s_warp[warp] = v;
    __syncthreads();
    if (warp == 0) {
      const int nw = blockDim.x >> 5;
      unsigned int x = lane < nw ? s_warp[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned int t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
      }
      if (lane < nw) s_warp[lane] = x;
    }
    __syncthreads();
    const unsigned int before = s_carry + (warp ? s_warp[warp - 1] : 0u) + (v - cnt);
    if (e < nev) pre[e] = before;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = before + cnt;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    pre[nev] = s_carry;
    ctl->total = s_carry;
    ctl->next = 0;
  }
}

/* the event of item q of the union: pre[e] <= q < pre[e + 1] (pre[nev] > q) */
__device__ __forceinline__ int item_event(const unsigned int* pre, int nev, unsigned int q) {
  int lo = 0, hi = nev;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= q) lo = mid;
    else hi = mid;
  }
  return lo;
}

/* k_prim_slow over the union of the events' deferred recoveries (persistent;
 * one item per warp pair at a time); left: the learned retry's leftovers instead */
template <int EOS, bool NCH>
__global__ void __launch_bounds__(128) kb_prim_slow(DevParams d0, const Geo* __restrict__ geo,
                                                    const Ev* __restrict__ tab, const unsigned int* __restrict__ pre,
                                                    int nev, Ctl* ctl, int which, int left) {
  __shared__ unsigned int s_q[2];
  __shared__ int s_stop[2];
  __shared__ Recovery s_cold[2];
  const unsigned n = *(volatile const unsigned int*)&ctl->total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int pair = warp >> 1;
  const bool lead = (warp & 1) == 0;
  while (true) {
    if (lead && lane == 0) {
      s_q[pair] = atomicAdd(&ctl->next, 1u);
      s_stop[pair] = 0;
    }
    pair_sync(pair);
    const unsigned q = *(volatile unsigned int*)&s_q[pair];
    if (q >= n) break;
    const int e = item_event(pre, nev, q);
    const Ev& ev = tab[e];
    DevParams d = d0;
    with_geo(d, geo[e]);
    const unsigned int* qe = left ? ev.qq : ev.qp;
    slow_item<EOS, NCH>(d, ev.pU[which], ev.w, ev.h, ev.ptau[which], ev.fl, (long long)qe[q - pre[e]], lane,
                        lead, pair, s_stop, s_cold);
  }
}

/* k_prim_learned_retry over the union of the events' deferred recoveries: CTA b
 * takes items b*128 .. of the union (cells of several events may share a tile:
 * the network does not depend on the grid), infers their starting points on the
 * tensor cores and runs the Newton with the guess check; a cell that converges is
 * stored, the rest go to its event's second queue. The grid covers the largest
 * possible union and the CTAs past its end return at once (all threads alike);
 * one tile per CTA, as in the single-event kernel. */
template <int EOS, bool NCH>
__global__ void __launch_bounds__(128, 4) kb_prim_learned_retry(DevParams d0, const Geo* __restrict__ geo,
                                                              const Ev* __restrict__ tab,
                                                              const unsigned int* __restrict__ pre, int nev,
                                                              const Ctl* ctl, int which, guess::Net net) {
  __shared__ __align__(128) guess::FwdSmem s;
  const unsigned n = *(volatile const unsigned int*)&ctl->total;
  const unsigned base = blockIdx.x * 128u;
  if (base >= n) return;
  const unsigned qi = base + threadIdx.x;
  const bool live = qi < n;
  int e = 0;
  long long i = 0;
  DevParams d = d0;
  CellCons c;
  float xn[guess::NIN];
#pragma unroll
  for (int q = 0; q < guess::NIN; ++q) xn[q] = 0.0f;
  if (live) {
    e = item_event(pre, nev, qi);
    with_geo(d, geo[e]);
    const Ev& ev = tab[e];
    i = (long long)ev.qp[qi - pre[e]];
    load_cons(d, ev.pU[which], i, ev.ptau[which], c);
    if (c.E > 0.0) {
      float r[guess::NIN];
      guess::features(c.E, c.Sx, c.Sy, c.Pi, c.pixx, c.pixy, c.piyy, r);
#pragma unroll
      for (int q = 0; q < guess::NIN; ++q) xn[q] = guess::nrm_in(net.norm, q, r[q]);
    }
  }
  float y[guess::NOUT] = {0.0f, 0.0f, 0.0f};
  const bool tile_ok = guess::forward_tile(s, net, xn, y);
  if (!live) return;
  const Ev& ev = tab[e];
  unsigned it_l = 0, n_l = 0, ok_l = 0;
  bool done = false;
  if (tile_ok && c.E > 0.0) done = guess_and_recover<EOS, NCH>(d, ev.w, ev.h, c, y, net, i, &it_l, &n_l, &ok_l);
  if (n_l) {
    atomicAdd(&ev.fl->it_learn, (unsigned long long)it_l);
    atomicAdd(&ev.fl->n_learn, (unsigned long long)n_l);
    atomicAdd(&ev.fl->ok_learn, (unsigned long long)ok_l);
  }
  if (!done) ev.qq[atomicAdd(&ev.fl->qcount_q, 1u)] = (unsigned)i;
  if (!tile_ok) atomicExch(&ev.fl->status, 3);
}

/* the face pass of stage k in one direction (FP64 or FP32 planes) */
template <int EOS, bool XDIR, bool F32>
__global__ void __launch_bounds__(128, FV_FACE_MINB) kb_faces(DevParams d0, const Geo* __restrict__ geo,
                                                              const Ev* __restrict__ tab,
                                                              const unsigned short* __restrict__ eob, int k) {
  __shared__ BlockHead sh;
  __shared__ DevState sU;
  __shared__ DevPrims sw;
  __shared__ DevFlags* sfl;
  __shared__ void* sF;
  __shared__ double stau;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, XDIR ? SH_FACEX : SH_FACEY, &blk)) return;
  const Ev& ev = tab[sh.e];
  to_shared(&sU, &ev.st[k].Ub);
  to_shared(&sw, &ev.w);
  if (threadIdx.x == 0) {
    sfl = ev.fl;
    stau = ev.st[k].tau;
    sF = F32 ? (void*)(XDIR ? ev.fhx32 : ev.fhy32) : (void*)(XDIR ? ev.fhx : ev.fhy);
  }
  __syncthreads();
  DevParams d = d0;
  with_geo(d, sh.g);
  const long long t = blk * 128 + threadIdx.x;
  if (F32) f32::faces32_body<EOS, XDIR>(d, sU, sw, stau, nullptr, (float*)sF, sfl, t);
  else faces_body<EOS, XDIR>(d, sU, sw, stau, nullptr, (double*)sF, sfl, t);
}

/* the face pass of stage k in both directions in one launch: an event's x-face
 * blocks and then its y-face blocks, so both read the event's planes at about the
 * same time (the second from L2 where the batch's planes do not fit in it) */
template <int EOS, bool F32>
__global__ void __launch_bounds__(128, FV_FACE_MINB) kb_faces_xy(DevParams d0, const Geo* __restrict__ geo,
                                                                 const Ev* __restrict__ tab,
                                                                 const unsigned short* __restrict__ eob, int k) {
  __shared__ BlockHead sh;
  __shared__ DevState sU;
  __shared__ DevPrims sw;
  __shared__ DevFlags* sfl;
  __shared__ void* sFx;
  __shared__ void* sFy;
  __shared__ double stau;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, SH_FACEXY, &blk)) return;
  const Ev& ev = tab[sh.e];
  to_shared(&sU, &ev.st[k].Ub);
  to_shared(&sw, &ev.w);
  if (threadIdx.x == 0) {
    sfl = ev.fl;
    stau = ev.st[k].tau;
    sFx = F32 ? (void*)ev.fhx32 : (void*)ev.fhx;
    sFy = F32 ? (void*)ev.fhy32 : (void*)ev.fhy;
  }
  __syncthreads();
  DevParams d = d0;
  with_geo(d, sh.g);
  const bool xdir = blk < sh.g.nbx;   /* uniform over the block */
  const long long t = (xdir ? blk : blk - sh.g.nbx) * 128 + threadIdx.x;
  if (F32) {
    if (xdir) f32::faces32_body<EOS, true>(d, sU, sw, stau, nullptr, (float*)sFx, sfl, t);
    else f32::faces32_body<EOS, false>(d, sU, sw, stau, nullptr, (float*)sFy, sfl, t);
  } else {
    if (xdir) faces_body<EOS, true>(d, sU, sw, stau, nullptr, (double*)sFx, sfl, t);
    else faces_body<EOS, false>(d, sU, sw, stau, nullptr, (double*)sFy, sfl, t);
  }
}

/* k_update of stage k */
template <int EOS, bool NCH, typename FT, bool FULL>
__global__ void __launch_bounds__(128) kb_update(DevParams d0, const Geo* __restrict__ geo, const Ev* __restrict__ tab,
                                                 const unsigned short* __restrict__ eob, int k) {
  __shared__ BlockHead sh;
  __shared__ StageArgs sa;
  __shared__ const FT* sfx;
  __shared__ const FT* sfy;
  __shared__ unsigned int* sq;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, SH_INT, &blk)) return;
  const Ev& ev = tab[sh.e];
  to_shared(&sa, &ev.st[k]);
  if (threadIdx.x == 0) {
    if (sizeof(FT) == 4) { sfx = (const FT*)ev.fhx32; sfy = (const FT*)ev.fhy32; }
    else { sfx = (const FT*)ev.fhx; sfy = (const FT*)ev.fhy; }
    sq = ev.qa;
  }
  __syncthreads();
  DevParams d = d0;
  with_geo(d, sh.g);
  update_body<EOS, NCH, FT, FULL>(d, sa, sfx, sfy, sq, blk * 128 + threadIdx.x);
}

/* k_adm_slow of stage k over the union of the events' queued inversions */
template <int EOS, bool NCH>
__global__ void __launch_bounds__(128) kb_adm_slow(DevParams d0, const Geo* __restrict__ geo,
                                                   const Ev* __restrict__ tab, const unsigned int* __restrict__ pre,
                                                   int nev, Ctl* ctl, int k) {
  const unsigned n = *(volatile const unsigned int*)&ctl->total;
  const int lane = threadIdx.x & 31;
  while (true) {
    unsigned q = 0;
    if (lane == 0) q = atomicAdd(&ctl->next, 1u);
    q = __shfl_sync(FV_FULL, q, 0);
    if (q >= n) break;
    const int e = item_event(pre, nev, q);
    const Ev& ev = tab[e];
    DevParams d = d0;
    with_geo(d, geo[e]);
    adm_item<EOS, NCH>(d, ev.st[k].Uout, ev.st[k].tau_state, ev.st[k].bad, ev.fl, (long long)ev.qa[q - pre[e]],
                       lane);
  }
}

/* relax_dissipative_2d! + project_shear! (FP64 or FP32 sources) */
template <int EOS, bool M2, bool F32>
__global__ void __launch_bounds__(128) kb_relax(DevParams d0, const Geo* __restrict__ geo, const Ev* __restrict__ tab,
                                                const unsigned short* __restrict__ eob) {
  __shared__ BlockHead sh;
  __shared__ DevState sq, so;
  __shared__ DevPrims sw;
  __shared__ DevHist shh;
  __shared__ DevFlags* sfl;
  __shared__ double stau, sD;
  __shared__ int srel, sproj;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, SH_CELL, &blk)) return;
  const Ev& ev = tab[sh.e];
  to_shared(&sq, &ev.rq);
  to_shared(&so, &ev.ro);
  to_shared(&sw, &ev.w);
  to_shared(&shh, &ev.h);
  if (threadIdx.x == 0) { sfl = ev.fl; stau = ev.rtau; sD = ev.rD; srel = ev.do_relax; sproj = ev.do_project; }
  __syncthreads();
  DevParams d = d0;
  with_geo(d, sh.g);
  const long long i = blk * 128 + threadIdx.x;
  if (F32) relax32_body<EOS>(d, sq, so, sw, shh, stau, sD, srel, sproj, sfl, i);
  else relax_body<EOS, M2>(d, sq, so, sw, shh, stau, sD, srel, sproj, sfl, i);
}

/* after a relaxation: ux_prev <- ux, uy_prev <- uy (the single-event path's two copies) */
__global__ void __launch_bounds__(128) kb_post_hist(const Geo* __restrict__ geo, const Ev* __restrict__ tab,
                                                    const unsigned short* __restrict__ eob) {
  __shared__ BlockHead sh;
  __shared__ double *sux, *suy, *spx, *spy;
  __shared__ int srel;
  long long blk;
  if (!block_head(&sh, geo, tab, eob, SH_CELL, &blk)) return;
  const Ev& ev = tab[sh.e];
  if (threadIdx.x == 0) { sux = ev.w.ux; suy = ev.w.uy; spx = ev.h.ux_prev; spy = ev.h.uy_prev; srel = ev.do_relax; }
  __syncthreads();
  const long long i = blk * 128 + threadIdx.x;
  if (!srel || i >= sh.g.Ntot) return;
  spx[i] = sux[i];
  spy[i] = suy[i];
}

/* every event's flag block into one array (one D2H copy for the batch) */
__global__ void kb_gather_flags(const Ev* __restrict__ tab, int nev, DevFlags* out) {
  constexpr int W = (int)(sizeof(DevFlags) / 8);
  static_assert(sizeof(DevFlags) % 8 == 0, "8-byte multiple");
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nev * W) return;
  const int e = (int)(t / W), k = (int)(t % W);
  if (!tab[e].active) return;
  reinterpret_cast<unsigned long long*>(out + e)[k] = reinterpret_cast<const unsigned long long*>(tab[e].fl)[k];
}

}  // namespace bt
}  // namespace fv

#endif
