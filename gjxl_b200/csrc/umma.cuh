// Fifth-generation tensor core (tcgen05) building blocks for sm_100a, as
// inline PTX: shared-memory matrix descriptors, tensor-memory allocation,
// single-thread MMA issue with mbarrier completion, and tensor-memory loads.
//
// Operand layouts are the canonical no-swizzle ("interleaved") forms: a
// core matrix is 8 x 8 bf16 stored as 8 rows of 16 contiguous bytes (128 B).
//  * K-major: a row holds 8 consecutive K elements; core matrices that are
//    adjacent along M/N lie SBO bytes apart, along K LBO bytes apart.
//  * MN-major: a row holds 8 consecutive M (or N) elements of one k; core
//    matrices adjacent along M/N lie SBO bytes apart, along K LBO bytes apart.
// One kind::f16 MMA consumes K = 16 (two core matrices along K).
#pragma once

#include <cstdint>

namespace gjxl_b200 {
namespace umma {

__device__ __forceinline__ uint32_t SmemAddress(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (no swizzle, sm_100 descriptor version 1):
// start address, leading (K) and stride (M/N) byte offsets, all in 16-byte
// units.
__device__ __forceinline__ uint64_t Descriptor(uint32_t address, uint32_t lbo_bytes,
                                               uint32_t sbo_bytes) {
  return static_cast<uint64_t>((address >> 4) & 0x3FFFu) |
         (static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32) |
         (static_cast<uint64_t>(1) << 46);
}

// Instruction descriptor of kind::f16 with bf16 operands and an f32
// accumulator: M = 64 or 128, N a multiple of 16 (M = 128) up to 256.
__host__ __device__ constexpr uint32_t InstrBf16F32(int m, int n, bool a_mn_major,
                                                    bool b_mn_major) {
  return (1u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(a_mn_major) << 15) |
         (static_cast<uint32_t>(b_mn_major) << 16) | (static_cast<uint32_t>(n >> 3) << 17) |
         (static_cast<uint32_t>(m >> 4) << 24);
}

// Tensor-memory allocation by one whole warp; the base address is written to
// `slot` in shared memory. `columns` is a power of two >= 32.
__device__ __forceinline__ void Allocate(uint32_t* slot, uint32_t columns) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
               :: "r"(SmemAddress(slot)), "r"(columns));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

__device__ __forceinline__ void Deallocate(uint32_t base, uint32_t columns) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
               :: "r"(base), "r"(columns));
}

// D (tensor memory) [+]= A (shared) x B (shared), issued by one thread.
__device__ __forceinline__ void Mma(uint32_t d, uint64_t a, uint64_t b, uint32_t instr,
                                    bool accumulate) {
  asm volatile(
    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
    :: "r"(d), "l"(a), "l"(b), "r"(instr), "r"(accumulate ? 1u : 0u));
}

// Arrives once on `barrier` when every MMA this thread issued so far is done.
__device__ __forceinline__ void Commit(uint64_t* barrier) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(SmemAddress(barrier)));
}

__device__ __forceinline__ void InitBarrier(uint64_t* barrier, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(SmemAddress(barrier)),
               "r"(count));
  asm volatile("fence.mbarrier_init.release.cluster;");
}

// Waits for the barrier phase with the given parity; gives up after `limit`
// polls (each poll may suspend the thread for a short time) and returns false.
__device__ __forceinline__ bool WaitParity(uint64_t* barrier, uint32_t parity, uint32_t limit) {
  const uint32_t address = SmemAddress(barrier);
  for (uint32_t i = 0; i < limit; ++i) {
    uint32_t done;
    asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done) : "r"(address), "r"(parity) : "memory");
    if (done) return true;
  }
  return false;
}

// Orders this thread's generic-proxy shared-memory writes before later
// tensor-core (async-proxy) reads of them.
__device__ __forceinline__ void FenceAsyncShared() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void FenceBeforeSync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void FenceAfterSync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 16 or 32 consecutive accumulator columns of this thread's lane
// (32x32b shape: warp w reads lanes 32w .. 32w + 31). `address` already
// carries the warp's lane offset in its upper half.
template <int kColumns>
__device__ __forceinline__ void Load(uint32_t address, float (&v)[kColumns]);

template <>
__device__ __forceinline__ void Load<16>(uint32_t address, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
    "%14,%15}, [%16];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
      "=r"(r[14]), "=r"(r[15])
    : "r"(address));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <>
__device__ __forceinline__ void Load<32>(uint32_t address, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
    "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
      "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
      "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
      "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
    : "r"(address));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace umma
}  // namespace gjxl_b200
