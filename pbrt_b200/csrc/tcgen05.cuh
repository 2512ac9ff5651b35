// tcgen05.cuh — the sm_100a tensor-core primitives the radiance-cache MLP uses, as inline
// PTX: TMEM allocation, tcgen05.mma (kind::f16, BF16 in, FP32 accumulate, one CTA),
// tcgen05.commit to an mbarrier, tcgen05.ld of the accumulator, and the fences that order
// them against ordinary shared-memory traffic; plus the mbarrier transaction counts and the
// plain bulk global-to-shared copy (cp.async.bulk) that the ray-cast cull stages rays with.
//
// Operand layout (both operands K-major, no swizzle): an R x K BF16 tile is stored as 8x8
// "core matrices" (8 rows x 16 bytes, 128 contiguous bytes); core matrix (row block rb,
// k block kb) sits at byte offset kb * (R/8 * 128) + rb * 128, and element (r, k) at
// + (r % 8) * 16 + (k % 8) * 2. In descriptor terms SBO = 128 bytes (next 8 rows) and
// LBO = R/8 * 128 bytes (next 8 columns of K); one MMA consumes K = 16, i.e. two k blocks.
#pragma once

#include <cstdint>
#include <cuda_bf16.h>

namespace pbrt {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (r, k) in an R-row tile of the layout above.
__host__ __device__ __forceinline__ uint32_t tile_offset(uint32_t r, uint32_t k, uint32_t rows) {
  return (k >> 3) * (rows >> 3) * 128u + (r >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Shared-memory matrix descriptor: start address, LBO, SBO (all >> 4), version 1 (sm_100),
// base offset 0, layout SWIZZLE_NONE.
__device__ __forceinline__ uint64_t make_desc(uint32_t smem_addr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= uint64_t((smem_addr >> 4) & 0x3FFFu);
  d |= uint64_t((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= uint64_t((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= uint64_t(1) << 46;  // version
  return d;
}

// Instruction descriptor of kind::f16: D = F32, A = B = BF16, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t m, uint32_t n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}
// The same with both operands MN-major (bit 15: A, bit 16: B). An MN-major operand without
// swizzle is built of the same 128-byte core matrices, read the other way round: 8 MN-
// consecutive elements per 16-byte row, 8 rows = 8 consecutive K; the descriptor's SBO is then
// the step between 8-element MN blocks and its LBO the step between 8-deep K blocks. So an
// R-row K-major tile of the layout above (element (r, c) at tile_offset(r, c, R)) is also
// the MN-major operand whose MN index is c and whose K index is r, with SBO = R/8 * 128 and
// LBO = 128: a product over the tile's rows needs no transposed copy.
__host__ __device__ constexpr uint32_t idesc_bf16_mn(uint32_t m, uint32_t n) {
  return idesc_bf16(m, n) | (1u << 15) | (1u << 16);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)), "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor cores' async proxy.
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* mbar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(smem_u32(mbar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Arrives on the barrier (one of its expected arrivals) and adds `bytes` to the transaction
// count its current phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
               : "memory");
}

// Bulk asynchronous copy of `bytes` (a multiple of 16) from global memory to this CTA's shared
// memory, both addresses 16-byte aligned; its bytes complete on `mbar`'s transaction count.
// Plain form: no tensor map, no multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(mbar))
               : "memory");
}

// Waits for phase `parity` of the barrier; gives up after `budget` polls and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t budget = 1u << 22) {
  for (uint32_t i = 0; i < budget; ++i)
    if (mbar_try_wait(mbar, parity)) return true;
  return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane (32x32b shape: the warp reads its
// own 32-lane quarter, lane = warp_quarter * 32 + lane id). An M = 128 accumulator has row r
// in lane r; an M = 64 one (one CTA) has row 16q + j in lane 32q + j (j < 16), so lanes 0-15
// of warp q hold rows 16q .. 16q + 15. The wait sits in the same asm
// statement, so no use of the registers can be scheduled before the data has arrived.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n\ttcgen05.wait::ld.sync.aligned;"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace tc
}  // namespace pbrt
