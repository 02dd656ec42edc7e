// Blackwell (sm_100a) tensor-core building blocks in inline PTX: the 5th
// generation MMA (tcgen05.mma, kind::f16 with BF16 operands and an FP32
// accumulator in tensor memory), TMEM allocation and loads, and mbarrier
// completion with bounded waits. Used by the warm-start network's kernels.
//
// Operand tiles live in shared memory in the canonical no-swizzle layouts:
//   K-major  (element (r, k) of an R x K tile, r along M or N):
//     byte (r/8)*SBO + (k/8)*LBO + (r%8)*16 + (k%8)*2
//   MN-major (element (r, k), r contiguous):
//     byte (r/8)*SBO + (k/8)*LBO + (k%8)*16 + (r%8)*2
// i.e. 8 x 16-byte "core matrices" of 128 bytes each. One MMA consumes
// K = 16 (two core matrices along K for K-major, two 8-row K groups for
// MN-major); successive K steps advance the descriptor's start address.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qesb {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor (sm100 version 1, no swizzle).
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;  // version 1 (Blackwell)
  // base offset 0, LBO mode 0, layout type 0 = SWIZZLE_NONE
  return d;
}

// Instruction descriptor: kind::f16, A = B = BF16, D = FP32, dense.
// a_mn / b_mn: 1 if the operand is MN-major, 0 if K-major.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn)
{
  return (1u << 4)                      // D format F32
         | (1u << 7)                    // A format BF16
         | (1u << 10)                   // B format BF16
         | ((uint32_t)a_mn << 15)       // A major
         | ((uint32_t)b_mn << 16)       // B major
         | ((uint32_t)(N >> 3) << 17)   // N / 8
         | ((uint32_t)(M >> 4) << 24);  // M / 16
}

// TMEM allocation by one full warp; the TMEM address lands in *smem_dst.
__device__ __forceinline__ void tmem_alloc(uint32_t *smem_dst, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

// Arrive on the mbarrier once all previously issued MMAs of this thread complete.
__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Generic-proxy shared-memory writes -> visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Waits for the mbarrier phase `parity` to complete; gives up after
// `limit` polls and returns false (the caller records an error and stops).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, uint32_t limit)
{
  const uint32_t a = smem_u32(mbar);
  for (uint32_t i = 0; i < limit; ++i) {
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

// A bounded wait whose first poll does not block (mbarrier.test_wait), then up
// to limit - 1 potentially suspending polls: with limit 1 it gives up unless
// the phase has already completed, so a timeout can be reached on demand.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *mbar, uint32_t parity, uint32_t limit)
{
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(smem_u32(mbar)), "r"(parity)
      : "memory");
  return done || (limit > 1 && mbar_wait(mbar, parity, limit - 1));
}

// After a wait gave up: the issuing thread makes `drain` (an mbarrier
// initialised with count 1 and not used otherwise) track every MMA it has
// started, and every thread waits for it, at most `limit` polls, so that TMEM
// and the operand tiles are not released under a running MMA. Every thread of
// the CTA that gave up calls it.
__device__ __forceinline__ void mma_drain(uint64_t *drain, bool issuer, uint32_t limit)
{
  if (issuer) mma_commit(drain);
  mbar_wait(drain, 0, limit);
}

// Expect `bytes` of asynchronous copies on the mbarrier, counting this
// thread's arrival; a plain arrival (no copies) for the same phase bookkeeping.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *mbar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *mbar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

// 4-D tiled tensor copy global -> shared through a tensor map (a
// __grid_constant__ kernel parameter or global memory), completing on the
// mbarrier; this GPU's own memory only (no multicast).
__device__ __forceinline__ void tma_load4(void *dst, const void *map, int c0, int c1, int c2, int c3, uint64_t *mbar)
{
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(mbar))
      : "memory");
}

// 32 lanes x 8 consecutive 32-bit columns of TMEM into 8 registers per thread
// (warp w of a warpgroup reads lanes 32*(w%4) .. +31).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8])
{
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

// 32 lanes x 16 consecutive 32-bit columns of TMEM into 16 registers per
// thread, without waiting: call tmem_wait_ld() before reading them.
__device__ __forceinline__ void tmem_ld16_async(uint32_t taddr, uint32_t (&r)[16])
{
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace umma
}  // namespace qesb
