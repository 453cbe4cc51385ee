// Blackwell (sm_100a) tensor-core building blocks: tcgen05 MMA with shared
// memory operands and a TMEM accumulator, TMEM allocation and loads,
// mbarrier completion with a bounded wait, and the shared-memory matrix and
// instruction descriptors.
//
// Operand layout used throughout: a "blocked" bf16 matrix of R rows x C
// columns (R, C multiples of 8) stored as 8 x 8 core matrices,
//   byte(r, c) = (r / 8) * (C / 8) * 128 + (c / 8) * 128 + (r % 8) * 16 + (c % 8) * 2,
// i.e. each 8-row group holds its C / 8 core matrices (8 rows of 16 bytes)
// one after another.  With no swizzle this is a canonical tcgen05 layout both
// ways round:
//   K-major  (rows = M or N, columns = K): leading byte offset 128 (next
//            8 columns), stride byte offset (C / 8) * 128 (next 8 rows);
//            a K step of 16 adds 256 bytes to the start address;
//   MN-major (columns = M or N, rows = K): stride byte offset 128 (next 8
//            columns), leading byte offset (C / 8) * 128 (next 8 rows); a K
//            step of 16 adds 2 * (C / 8) * 128 bytes.
// So one buffer serves a forward GEMM (activations K-major) and the weight
// gradient GEMM (the same activations as the MN-major operand) without a
// transposed copy.
#pragma once

#include <cstdint>

namespace xyzgpu {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle): start address, leading and
// stride byte offsets (all >> 4), version 1 at bit 46, layout type 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = static_cast<uint64_t>((addr >> 4) & 0x3FFFu);
  d |= static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16;
  d |= static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32;
  d |= uint64_t{1} << 46;
  return d;
}

__device__ __forceinline__ uint64_t desc_kmajor(uint32_t addr, int cols) {
  return smem_desc(addr, 128u, static_cast<uint32_t>(cols / 8) * 128u);
}
__device__ __forceinline__ uint64_t desc_mnmajor(uint32_t addr, int cols) {
  return smem_desc(addr, static_cast<uint32_t>(cols / 8) * 128u, 128u);
}

// Instruction descriptor, kind::f16: BF16 A and B, F32 accumulator, dense.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

// D[tmem] (+)= A * B, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate ? 1u : 0u));
}

// Arrives on the mbarrier once every MMA issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Makes this thread's generic-proxy shared-memory writes visible to the
// tensor core (async proxy).
__device__ __forceinline__ void fence_smem_to_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for the phase with the given parity to complete; gives up after
// `limit` polls and returns false (the caller records an error).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// TMEM allocation: one whole warp; the base address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive 32-bit columns of this thread's TMEM lane (warp-collective;
// the warp's lanes are 32 * (warp % 4) + lane).  Call tmem_wait_ld before use.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
      "%14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of element (r, c) in a blocked matrix of `cols` columns.
__host__ __device__ constexpr uint32_t blocked_offset(int r, int c, int cols) {
  return static_cast<uint32_t>((r >> 3) * (cols >> 3) * 128 + (c >> 3) * 128 + (r & 7) * 16 + (c & 7) * 2);
}

}  // namespace tc
}  // namespace xyzgpu
