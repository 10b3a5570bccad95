// Building blocks of the sm_100a tensor-core kernels: mbarriers, TMA loads, shared-memory
// and instruction descriptors of tcgen05.mma kind::tf32, TMEM loads.  Every wait built on
// these is bounded by the caller.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace hprmat {
namespace tc {

constexpr unsigned kWaitLimit = 1u << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: false if the limit was reached or another role already gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int* err,
                                          int site) {
  for (unsigned it = 0; it < kWaitLimit; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if ((it & 1023u) == 1023u && *abort_flag) return false;
  }
  *abort_flag = 1;
  atomicCAS(err, 0, site);
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}


// Prefetch of one TMA box into L2 (no shared-memory destination, no completion).
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap* map, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global.tile [%0, {%1, %2, %3}];" ::"l"(
                   reinterpret_cast<uint64_t>(map)),
               "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}

// Shared-memory matrix descriptor, K-major, 64-byte swizzle: rows of 64 bytes, 8-row
// groups 512 bytes apart (stride byte offset), leading byte offset unused (1), version 1.
__device__ __forceinline__ uint64_t sdesc_k_sw64(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
  d |= (uint64_t)1 << 16;                 // LBO (ignored for swizzled K-major)
  d |= (uint64_t)(512 >> 4) << 32;        // SBO
  d |= (uint64_t)1 << 46;                 // descriptor version (sm_100)
  d |= (uint64_t)4 << 61;                 // SWIZZLE_64B
  return d;
}

// Instruction descriptor: kind::tf32, D = F32, A = B = TF32, both K-major, M = 128, N = BN.
template <int BN>
__host__ __device__ constexpr uint32_t idesc_tf32(bool neg_a) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((neg_a ? 1u : 0u) << 13) | ((uint32_t)(BN >> 3) << 17) |
         ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 3xTF32 complex product of one K-step of 8 into the Re/Im accumulators t_re, t_im:
//   Re += Ar Br - Ai Bi,  Im += Ar Bi + Ai Br,  each real product as hi*lo + lo*hi + hi*hi.
// a[0..3] / b[0..3] are the descriptors of the Re-hi, Re-lo, Im-hi, Im-lo planes.  With
// negate = true the whole product is subtracted instead.
template <int BN>
__device__ __forceinline__ void cmma_3xtf32(uint32_t t_re, uint32_t t_im, const uint64_t* a, const uint64_t* b,
                                            uint32_t first, bool negate) {
  const uint32_t pos = idesc_tf32<BN>(negate), neg = idesc_tf32<BN>(!negate);
  mma_tf32(t_re, a[0], b[1], pos, first);
  mma_tf32(t_re, a[1], b[0], pos, 1u);
  mma_tf32(t_re, a[2], b[3], neg, 1u);
  mma_tf32(t_re, a[3], b[2], neg, 1u);
  mma_tf32(t_re, a[0], b[0], pos, 1u);
  mma_tf32(t_re, a[2], b[2], neg, 1u);
  mma_tf32(t_im, a[0], b[3], pos, first);
  mma_tf32(t_im, a[1], b[2], pos, 1u);
  mma_tf32(t_im, a[2], b[1], pos, 1u);
  mma_tf32(t_im, a[3], b[0], pos, 1u);
  mma_tf32(t_im, a[0], b[2], pos, 1u);
  mma_tf32(t_im, a[2], b[0], pos, 1u);
}

}  // namespace tc
}  // namespace hprmat
