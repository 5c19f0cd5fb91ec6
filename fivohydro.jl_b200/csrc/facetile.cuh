/*
 * facetile.cuh — the face pass of rhs_2d! (`_faces_2d!`, src2d/rhs2d.jl:282-371,
 * with `reconstruct_muscl_2d!`, src2d/reconstruction2d.jl:27-103) fed from
 * halo tiles staged in shared memory by the tensor memory accelerator.
 *
 * One CTA owns a tile of TX x TY faces of one direction. Before any arithmetic,
 * one thread issues a 2-D bulk tensor copy (cp.async.bulk.tensor, no multicast)
 * per plane the faces read: the four reconstructed primitives (yT, phi, u^x,
 * u^y), mu (the first-order fallback), and the dissipative rows the layout
 * carries. Each box covers the tile plus the stencil's halo: for x faces between
 * cells fx and fx + 1, fx in [X0, X0 + TX), the cells X0 - 1 .. X0 + TX + 1 in x
 * and Y0 .. Y0 + TY - 1 in y; for y faces the same with the roles swapped and the
 * box widened to TY + 4 in y so its start Y0 - 2 stays 16-byte aligned. Boxes
 * that reach past the grid are filled with zeros, which only faces outside the
 * grid or first-order faces (which read their own cell only) could see. The
 * threads wait on one mbarrier (a bounded wait: a copy that does not complete
 * sets status 4 and the CTA returns), then two lanes per face run
 * face_flux_pair on the tile: the same arithmetic as k_faces, so the same bits.
 *
 * Tensor maps need each plane's row pitch (Nytot doubles) and base to be
 * multiples of 16 bytes: the pass is used when Nytot is even. The tile shape is
 * chosen per context by timing the candidates (fivo2d.cu, tune_faces).
 */
#pragma once
#include <cuda.h>
#include "kernels.cuh"
#include "tc05.cuh"

namespace fv {

#define FT_MAXPL 12          /* 4 primitives + mu + up to 7 dissipative rows */
#define FT_WAIT_POLLS (1u << 22)

/* the tensor maps of one launch: plane k of the tile is map[k]; dis_plane[j] is
 * the tile plane of dissipative slot j (nux, nuy, Pi, pixx, pixy, piyy, pieta),
 * -1 when the layout does not carry it */
struct FaceTileMaps {
  CUtensorMap map[FT_MAXPL];
  int nplanes;
  int dis_plane[7];
};

__device__ __forceinline__ void tma_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
               :: "r"(tc05::smem_u32(mbar)), "r"(bytes) : "memory");
}

/* 2-D tiled bulk tensor copy global -> this CTA's shared memory, completion counted
 * on the mbarrier in bytes; c0 is the inner (y) coordinate, c1 the outer (x) one */
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
      :: "r"(tc05::smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(tc05::smem_u32(mbar)), "r"(c0),
         "r"(c1)
      : "memory");
}

/* bytes of one plane's box, padded to the 128-byte alignment of each box in shared memory */
FX_HD constexpr int ft_box_elems(bool xdir, int TX, int TY) { return xdir ? (TX + 3) * TY : TX * (TY + 4); }
FX_HD constexpr int ft_plane_bytes(bool xdir, int TX, int TY) { return ((ft_box_elems(xdir, TX, TY) * 8 + 127) / 128) * 128; }
/* dynamic shared memory of a launch: the boxes plus the 128-byte alignment slack */
FX_HD constexpr int ft_smem_bytes(bool xdir, int TX, int TY, int np) { return np * ft_plane_bytes(xdir, TX, TY) + 128; }

/* the stencil read from the tile: L is the tile index of the face's left cell, st the
 * tile stride along the face's direction, pl the plane stride in doubles */
struct FaceSrcTile {
  const double* sm;
  int pl, L, st;
  const int* dis_plane;
  __device__ __forceinline__ double prim(int q, int p) const { return sm[q * pl + L + p * st]; }
  __device__ __forceinline__ double mu(int p) const { return sm[4 * pl + L + p * st]; }
  __device__ __forceinline__ void dis(int p, double out[7]) const {
#pragma unroll
    for (int j = 0; j < 7; ++j) {
      const int k = dis_plane[j];
      out[j] = k >= 0 ? sm[k * pl + L + p * st] : 0.0;
    }
  }
};

template <int EOS, bool XDIR, int TX, int TY>
__global__ void __launch_bounds__(2 * TX * TY, 1024 / (2 * TX * TY)) k_faces_tile(DevParams d, const __grid_constant__ FaceTileMaps maps,
                                                           double tau, const uint8_t* ffo, double* Fh, DevFlags* fl) {
  static_assert(TY % 2 == 0, "the inner box extent must be a multiple of 16 bytes");
  extern __shared__ __align__(128) unsigned char ft_smem[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ double red[(2 * TX * TY) / 32];
  constexpr int PB = ft_plane_bytes(XDIR, TX, TY);
  constexpr int PL = PB / 8;
  /* the boxes start on a 128-byte boundary (the launch reserves 128 bytes of slack) */
  unsigned char* base = ft_smem + ((128u - (tc05::smem_u32(ft_smem) & 127u)) & 127u);
  double* sm = reinterpret_cast<double*>(base);
  const int Y0 = blockIdx.x * TY, X0 = blockIdx.y * TX;
  const int np = maps.nplanes;
  if (threadIdx.x == 0) {
    tc05::mbar_init(&bar, 1);
    tma_expect_tx(&bar, (uint32_t)(np * ft_box_elems(XDIR, TX, TY) * 8));
    for (int k = 0; k < np; ++k)
      tma_load_2d(base + k * PB, &maps.map[k], XDIR ? Y0 : Y0 - 2, XDIR ? X0 - 1 : X0, &bar);
  }
  __syncthreads();
  const bool arrived = tc05::mbar_wait(&bar, 0, FT_WAIT_POLLS);
  if (!__syncthreads_and(arrived ? 1 : 0)) {
    if (threadIdx.x == 0) fl->status = 4;
    return;
  }
  /* two lanes per face; consecutive faces run along y */
  const int side = threadIdx.x & 1;
  const int face = threadIdx.x >> 1;
  const int a = face / TY, b = face % TY;          /* tile face (x, y) */
  double amax = 0.0;
  long long i;
  int k, kmax, L;
  bool valid;
  if (XDIR) {
    const int fx = X0 + a, y = Y0 + b;
    valid = fx < d.Nxtot - 1 && y < d.Nytot;
    i = (long long)fx * d.Nytot + y;
    k = fx; kmax = d.Nxtot;
    L = (a + 1) * TY + b;
  } else {
    const int x = X0 + a, fy = Y0 + b;
    valid = x < d.Nxtot && fy < d.Nytot - 1;
    i = (long long)x * d.Nytot + fy;
    k = fy; kmax = d.Nytot;
    L = a * (TY + 4) + (b + 2);
  }
  if (valid) {   /* both lanes of a pair agree */
    const FaceSrcTile src{sm, PL, L, XDIR ? TY : 1, maps.dis_plane};
    amax = face_flux_pair<EOS, XDIR>(d, src, i, XDIR ? d.Nytot : 1, k, kmax, tau, ffo, side, Fh);
  }
  for (int o = 16; o > 0; o >>= 1) amax = jmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = amax;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (2 * TX * TY) / 32; ++w) m = jmax(m, red[w]);
    atomic_max_pos(&fl->amax_bits, m);
  }
}

}  // namespace fv
