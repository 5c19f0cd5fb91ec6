/* Host-only check of the tensor-core descriptor encoders of tc05.cuh against
 * CUTLASS's own bitfield definitions of the sm_100 UMMA descriptors
 * (cute/arch/mma_sm100_desc.hpp), and of the canonical-layout offsets against
 * the descriptor's (start, LBO, SBO) addressing. Built with nvcc as a host
 * program; runs without a GPU. Prints "ok" or the first mismatch. */
#include <cstdio>
#include <cstdint>
#include <cute/arch/mma_sm100_desc.hpp>
#include "../../fivohydro.jl_b200/csrc/tc05.cuh"

static int fails = 0;
#define EXPECT(c, ...) do { if (!(c)) { std::printf(__VA_ARGS__); std::printf("\n"); ++fails; } } while (0)

int main() {
  /* instruction descriptors: every (M = 128, N) the kernels use */
  const int Ns[] = {16, 64, 80};
  for (int N : Ns) {
    cute::UMMA::InstrDescriptor ref{};
    ref.c_format_ = 1;                         /* F32 */
    ref.a_format_ = 1;                         /* BF16 */
    ref.b_format_ = 1;
    ref.a_major_ = 0;                          /* K-major */
    ref.b_major_ = 0;
    ref.n_dim_ = N >> 3;
    ref.m_dim_ = 128 >> 4;
    EXPECT(ref.desc_ == tc05::idesc_bf16_f32(128, N), "idesc N=%d: ours %08x cute %08x", N,
           tc05::idesc_bf16_f32(128, N), ref.desc_);
  }
  /* shared-memory descriptors: field by field */
  const uint32_t addrs[] = {0u, 4096u, 79872u, 200000u};
  const uint32_t rows[] = {16u, 64u, 80u, 128u};
  for (uint32_t a : addrs)
    for (uint32_t R : rows)
      for (uint32_t k16 = 0; k16 < 8; ++k16) {
        cute::UMMA::SmemDescriptor ref;
        ref.desc_ = 0;
        ref.version_ = 1;
        ref.lbo_mode_ = 0;
        ref.layout_type_ = (uint8_t)cute::UMMA::LayoutType::SWIZZLE_NONE;
        ref.base_offset_ = 0;
        ref.start_address_ = (uint16_t)((a + k16 * 2u * R * 16u) >> 4);
        ref.leading_byte_offset_ = (uint16_t)((R * 16u) >> 4);
        ref.stride_byte_offset_ = (uint16_t)(128u >> 4);
        const uint64_t ours = tc05::tile_desc(a, R, k16);
        EXPECT(ref.desc_ == ours, "smem desc a=%u R=%u k16=%u: ours %016llx cute %016llx", a, R, k16,
               (unsigned long long)ours, (unsigned long long)ref.desc_);
      }
  /* the canonical K-major layout ((8,n),2):((1,SBO),LBO) in 16-byte units: element
   * (r, k) of the k16-th slice sits at start + (r%8)*16 + (r/8)*SBO + ((k%16)/8)*LBO
   * + (k%8)*2; kmaj_off must agree for every element of every tile shape */
  for (uint32_t R : rows)
    for (uint32_t r = 0; r < R; ++r)
      for (uint32_t k = 0; k < 128; ++k) {
        const uint32_t k16 = k / 16, kk = k % 16;
        const uint32_t start = k16 * 2u * R * 16u, lbo = R * 16u, sbo = 128u;
        const uint32_t via_desc = start + (r % 8) * 16u + (r / 8) * sbo + (kk / 8) * lbo + (kk % 8) * 2u;
        EXPECT(via_desc == tc05::kmaj_off(R, r, k), "offset R=%u r=%u k=%u", R, r, k);
        if (fails > 8) return 1;
      }
  if (fails) return 1;
  std::printf("ok\n");
  return 0;
}
