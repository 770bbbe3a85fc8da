// Blackwell (sm_100a) tensor-core building blocks for the radiance cache's
// MLP: tcgen05.mma with operands in shared memory and the accumulator in
// tensor memory (TMEM), TMEM allocation, completion through an mbarrier and
// TMEM -> register loads, and the untiled bulk copy (TMA) that stages the
// weights.  Inline PTX only; one CTA, no clusters, no multicast.
//
// Operand tiles use the no-swizzle canonical layout: an R x C bf16 tile is
// stored as 8-row x 16-byte core matrices (128 contiguous bytes each), core
// matrix (r/8, c/8) at ((c/8) * (R/8) + r/8) * 128 bytes.  The same bytes
// serve as a K-major operand (rows = M or N, columns = K) and as an MN-major
// operand (columns = M or N, rows = K); in both cases the descriptor's
// stride byte offset is the distance between core matrices along M/N and the
// leading byte offset the distance along K.
#pragma once
#include <cstdint>

namespace pfxt {
namespace umma {

__device__ __forceinline__ uint32_t tile_offset(uint32_t r, uint32_t c, uint32_t R) {
  return ((c >> 3) * (R >> 3) + (r >> 3)) * 128u + (r & 7u) * 16u + (c & 7u) * 2u;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor: start address, leading (K) and stride
// (M/N) byte offsets, version 1, no swizzle, base offset 0.
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// K-major operand from an R-row tile at `base`, K step `s` (16 columns).
__device__ __forceinline__ uint64_t desc_k(uint32_t base, uint32_t R, uint32_t s) {
  return desc(base + s * 2u * (R * 16u), R * 16u, 128u);
}
// MN-major operand from an R-row tile at `base`, K step `s` (16 rows).
__device__ __forceinline__ uint64_t desc_mn(uint32_t base, uint32_t R, uint32_t s) {
  return desc(base + s * 256u, 128u, R * 16u);
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator.
__host__ __device__ constexpr uint32_t idesc(uint32_t M, uint32_t N, bool a_mn, bool b_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
         ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(id), "r"(accumulate));
}

// Arrive on the mbarrier when every MMA issued so far by this thread is done.
__device__ __forceinline__ void commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
               : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One plain arrival on the barrier (release semantics for this thread's writes).
__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}

// One arrival that also expects `bytes` of asynchronous copies on the barrier.
__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}

// Untiled bulk copy (TMA) of `bytes` from global memory into this CTA's shared
// memory, completing on `mbar`: both addresses 16-byte aligned, `bytes` a
// multiple of 16.  No multicast: the copy lands in the issuing CTA only.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// Tiled 4-D bulk tensor copy (TMA) of the box at coordinates (c0, c1, c2, c3)
// of the tensor map `map` (a __grid_constant__ kernel parameter) into this
// CTA's shared memory, completing on `mbar`.  No multicast.  Coordinates may
// lie outside the tensor (the box reads zeros there); c0, the innermost, must
// be a multiple of 16 bytes of elements.
__device__ __forceinline__ void tensor_load_4d(uint32_t dst, const void* map, int c0, int c1, int c2, int c3,
                                               uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(dst),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(mbar)
      : "memory");
}

// Bounded wait for the completion of phase `parity`; false when the limit ran out.
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

// TMEM allocation by one full warp; the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
               "r"(cols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t cols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(cols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes become visible to the tensor cores.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive 32-bit columns of this thread's TMEM lane.
__device__ __forceinline__ void ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// TMEM address of lane `lane`, column `col`.
__device__ __forceinline__ uint32_t taddr(uint32_t base, uint32_t lane, uint32_t col) {
  return base + (lane << 16) + col;
}

}  // namespace umma
}  // namespace pfxt
