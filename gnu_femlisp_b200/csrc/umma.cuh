// umma.cuh -- minimal tcgen05 (5th-generation tensor core) helpers: shared
// memory matrix descriptors without swizzle, the BF16 x BF16 -> FP32
// instruction descriptor, tensor-memory allocation and loads, and the
// mbarrier the MMA completion is committed to.
//
// Shared-memory operands use the no-swizzle canonical layouts, whose unit is
// the core matrix: 8 rows of 16 contiguous bytes (8 BF16 values), rows 16
// bytes apart (128 contiguous bytes).
//   K-major (the 8 values of a row run along K): core matrices of one 8-row
//     group are `lbo` bytes apart along K, 8-row groups `sbo` bytes apart.
//   MN-major (the 8 values run along M or N): core matrices adjacent along
//     M/N are `sbo` bytes apart, along K `lbo` bytes apart.
// Neither needs the groups to be contiguous: any 16-byte multiple works, which
// lets a convolution address a shifted halo window by its start address alone.
//
// Waits are bounded: mbar_wait returns false after kSpinLimit polls and the
// caller records an error and stops issuing work.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace fmg {
namespace umma {

constexpr int kSpinLimit = 1 << 24;  // mbarrier polls before a wait gives up (well over a second)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// byte offset of element (r, k) in a K-major no-swizzle tile with K columns,
// K chunks of an 8-row group adjacent (lbo = 128), groups (K/8)*128 apart
__host__ __device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int K) {
  return (uint32_t)((r & 7) * 16 + (k >> 3) * 128 + (r >> 3) * (K >> 3) * 128 + (k & 7) * 2);
}

// shared-memory matrix descriptor, no swizzle (layout type 0), sm_100 version 1
__device__ __forceinline__ uint64_t make_desc(uint32_t start_bytes, uint32_t lbo_bytes, uint32_t sbo_bytes) {
  uint64_t d = 0;
  d |= (uint64_t)((start_bytes >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, dense
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, bool a_mn_major, bool b_mn_major) {
  return (1u << 4)                            // D format F32
         | (1u << 7)                          // A format BF16
         | (1u << 10)                         // B format BF16
         | ((a_mn_major ? 1u : 0u) << 15)     // A major
         | ((b_mn_major ? 1u : 0u) << 16)     // B major
         | ((uint32_t)(N >> 3) << 17)         // N / 8
         | ((uint32_t)(M >> 4) << 24);        // M / 16
}

// whole warp: allocate ncols (power of two >= 32) tensor-memory columns,
// address written to *slot_smem
__device__ __forceinline__ void tmem_alloc(uint32_t* slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot_smem)),
               "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {  // whole warp
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// this thread's generic-proxy shared-memory writes -> visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// an mbarrier whose phase completes after `count` arrivals
__device__ __forceinline__ void mbar_init_count(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival on the mbarrier that also expects `bytes` of asynchronous
// transactions (the TMA copies that complete on it)
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// tiled TMA load of a 5D box into this CTA's shared memory, completing on
// the mbarrier (no multicast); tmap: the address of a __grid_constant__
// CUtensorMap parameter
__device__ __forceinline__ void tma_load_5d(void* dst, const void* tmap, uint64_t* bar, int c0, int c1, int c2,
                                            int c3, int c4) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}

// tiled TMA loads of a 1D / 3D box, completing on the mbarrier (no multicast);
// the innermost coordinate times the element size must be a multiple of 16
__device__ __forceinline__ void tma_load_1d(void* dst, const void* tmap, uint64_t* bar, int c0) {
  asm volatile(
      "cp.async.bulk.tensor.1d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2}], [%3];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const void* tmap, uint64_t* bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// D[tmem] (+)= A * B^T; issued by one thread
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// arrive once on the mbarrier when all MMAs issued so far by this thread are done
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// bounded wait for the completion of the mbarrier phase with this parity:
// gives up after kWaitNs of global time or kSpinLimit polls, whichever first
constexpr uint64_t kWaitNs = 2000000000ull;
// the same wait with explicit limits (max_polls polls, max_ns of global time)
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, int max_polls, uint64_t max_ns) {
  const uint32_t a = smem_u32(bar);
  const uint64_t t0 = global_ns();
  for (int it = 0; it < max_polls; ++it) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255) == 255 && global_ns() - t0 > max_ns) return false;
  }
  return false;
}
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  return mbar_wait_for(bar, parity, kSpinLimit, kWaitNs);
}
// one test of the phase (no wait loop, no clock read): the fast path of a
// wait whose phase has usually completed already
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// one plain arrival on the mbarrier
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// whole warp: 32 (x32) or 16 (x16) consecutive FP32 columns of this thread's
// lane; warp w of the CTA may read lanes 32(w%4) .. 32(w%4)+31
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

template <int N>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float* v) {
  static_assert(N == 16 || N == 32, "16 or 32 columns");
  if constexpr (N == 32) tmem_ld32(taddr, v);
  else tmem_ld16(taddr, v);
}

}  // namespace umma
}  // namespace fmg
