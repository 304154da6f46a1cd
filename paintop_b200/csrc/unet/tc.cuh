// tc.cuh -- thin wrappers over the sm_100a tensor-core (tcgen05) and mbarrier
// PTX used by the U-Net kernels. Formats follow the PTX ISA for tcgen05:
//
// Shared-memory matrix descriptor (64 bit), canonical layout without swizzle:
//   bits  0-13  start address >> 4
//   bits 16-29  leading-dimension byte offset >> 4: the stride between
//               core matrices that are adjacent along K
//   bits 32-45  stride-dimension byte offset >> 4: the stride between core
//               matrices that are adjacent along M/N
//   bits 46-47  descriptor version (1 on sm_100)
//   bits 61-63  layout type (0 = no swizzle)
// A "core matrix" is 128 contiguous bytes: 8 rows of 16 bytes. For a K-major
// operand a row is 8 K-consecutive elements of one M/N index; for an MN-major
// operand it is 8 M/N-consecutive elements of one K index. Without swizzling
// the two offsets mean the same in both majors (the interleaved canonical
// layouts ((8,m),(8,2)) and ((8,m),(8,k)) of the CuTe UMMA descriptor).
//
// Instruction descriptor (32 bit) for kind::f16:
//   bits 4-5 accumulator format (1 = f32), 7-9 A format (1 = bf16),
//   10-12 B format (1 = bf16), 15 A major (0 = K), 16 B major (0 = K),
//   17-22 N >> 3, 24-28 M >> 4.
#pragma once

#include <cstdint>

namespace unet {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__host__ __device__ constexpr uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// bf16 x bf16 -> f32, both operands of the given majors, M x N tile.
__host__ __device__ constexpr uint32_t instr_desc_bf16(int M, int N, bool a_mn_major, bool b_mn_major) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn_major ? 1u : 0u) << 15) |
         ((b_mn_major ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// ---- TMEM allocation (one full warp) -------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *smem_dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// ---- MMA (one thread) -----------------------------------------------------
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// Arrive on `mbar` once every tcgen05 op this thread issued has completed.
__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(mbar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
// generic-proxy shared-memory writes (st.shared, cp.async) -> visible to the tensor core
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- TMEM -> registers: 32 lanes x 16 columns of 32 bits per warp ---------
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
        "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// ---- mbarrier ---------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Bounded wait for the phase with the given parity to complete. Returns false
// if it did not within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t k = 0; k < limit; ++k) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}
// Arrive and add `bytes` to the transaction count the phase waits for.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
               : "memory");
}

// ---- TMA (tensor copies; never multicast) -----------------------------------
// One box of a 4-D tensor map into shared memory; completion is reported to
// `mbar` as transaction bytes. Coordinates are element indices, innermost
// first; out-of-range elements read as zero.
__device__ __forceinline__ void tma_load_4d(void *smem_dst, const void *tmap, int c0, int c1, int c2, int c3,
                                            uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(smem_dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(mbar))
      : "memory");
}

__device__ __forceinline__ void tma_load_5d(void *smem_dst, const void *tmap, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t *mbar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(smem_dst)),
      "l"(tmap), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(mbar))
      : "memory");
}

// ---- cp.async ---------------------------------------------------------------
__device__ __forceinline__ void cp16(void *smem_dst, const void *gmem_src, bool in) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(smem_dst)), "l"(gmem_src),
               "r"(in ? 16 : 0)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// K-major core-matrix tile offset in bytes: rows (M or N) of `rows8 * 8`, 8
// bf16 of K per 16-byte core-matrix row. Element (r, k) sits at
// ((k / 8) * rows8 + r / 8) * 128 + (r % 8) * 16 + (k % 8) * 2, so the leading
// (K) byte offset is rows8 * 128 and the stride (row-group) offset is 128.
__host__ __device__ constexpr uint32_t kmajor_off(uint32_t r, uint32_t k8, uint32_t rows8) {
  return (k8 * rows8 + (r >> 3)) * 128u + (r & 7u) * 16u;
}

}  // namespace unet
