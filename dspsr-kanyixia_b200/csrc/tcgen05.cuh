// tcgen05.cuh -- the few Blackwell (sm_100a) tensor-core primitives the
// tensor-core kernels of this library use: shared-memory matrix and
// instruction descriptors, tcgen05.mma (BF16 in, FP32 accumulate in tensor
// memory) issued by one thread, tcgen05.commit to an mbarrier, bounded
// mbarrier waits, tensor-memory loads and the fences between them.
#pragma once

#include <cstdint>

namespace b200 {
namespace tc {

__device__ __forceinline__ uint32_t saddr (const void* p)
{
  return static_cast<uint32_t> (__cvta_generic_to_shared (p));
}

// shared memory matrix descriptor (sm_100): start, LBO, SBO in 16-byte
// units, descriptor version 1, no swizzle
__device__ __forceinline__ uint64_t sdesc (uint32_t start, uint32_t lbo, uint32_t sbo)
{
  return uint64_t ((start >> 4) & 0x3FFFu) | (uint64_t ((lbo >> 4) & 0x3FFFu) << 16)
         | (uint64_t ((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t (1) << 46);
}

// instruction descriptor: BF16 x BF16 -> F32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16 (unsigned M, unsigned N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16 (uint32_t d, uint64_t a, uint64_t b, uint32_t id,
                                          uint32_t acc)
{
  asm volatile (
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(id), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit (uint64_t* bar)
{
  asm volatile (
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          saddr (bar))
      : "memory");
}

__device__ __forceinline__ void fence_before () { asm volatile ("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after () { asm volatile ("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem () { asm volatile ("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void bar_init (uint64_t* bar, unsigned count)
{
  asm volatile ("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr (bar)), "r"(count) : "memory");
  asm volatile ("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool bar_try (uint64_t* bar, unsigned parity)
{
  uint32_t ok;
  asm volatile (
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(saddr (bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// bounded: about 2^21 polls (a second or so)
__device__ __forceinline__ bool bar_wait (uint64_t* bar, unsigned parity)
{
  for (int it = 0; it < (1 << 21); it++)
    if (bar_try (bar, parity)) return true;
  return false;
}

// 32 consecutive accumulator columns of this thread's lane
__device__ __forceinline__ void tmem_ld32 (uint32_t taddr, float* v)
{
  uint32_t r[32];
  asm volatile (
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile ("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; i++) v[i] = __uint_as_float (r[i]);
}


// tensor-memory allocation by one whole warp (ncols a power of two >= 32);
// the address lands in *slot
__device__ __forceinline__ void tmem_alloc (uint32_t* slot, uint32_t ncols)
{
  asm volatile ("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                    saddr (slot)),
                "r"(ncols)
                : "memory");
  asm volatile ("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free (uint32_t taddr, uint32_t ncols)
{
  asm volatile ("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                : "memory");
}

} // namespace tc
} // namespace b200
