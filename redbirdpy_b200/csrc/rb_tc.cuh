// tcgen05 / mbarrier building blocks shared by the tensor-core kernels
// (rb_gram.cu: J J^T; rb_jac.cu: the Jacobian's per-node pair products).
//
// Operands are K-major with the 128-byte swizzle: a row of an operand tile
// holds 128 bytes of K (32 TF32 or 64 BF16 elements), rows come in groups of
// 8 that are 1024 bytes apart, and inside a group the 16-byte chunk c of row
// r sits at chunk position c ^ (r % 8) (what a TMA copy with
// CU_TENSOR_MAP_SWIZZLE_128B writes).  An MMA consumes 32 bytes of K per
// instruction, at a descriptor start address advanced by 32 bytes per step.
#pragma once

#include <cstdint>

namespace rb {

constexpr long long kTcWaitLimit = 1LL << 24;  // polls before a wait gives up (about a second)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// bounded parity wait: false (and *err set to code) when the phase never
// completes within the limit
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err, int code,
                                          long long limit = kTcWaitLimit) {
  for (long long i = 0; i < limit; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  atomicExch(err, code);
  return false;
}

// shared-memory matrix descriptor: K-major operand, 128-byte swizzle,
// 8-row groups 1024 bytes apart (stride byte offset), descriptor version 1
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1u << 16;                    // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1u << 46;                    // version
  d |= (uint64_t)2u << 61;                    // SWIZZLE_128B
  return d;
}

// instruction descriptor of an MMA with FP32 accumulation and K-major A and
// B: fmt 2 = TF32 (kind::tf32), fmt 1 = BF16 (kind::f16); m = 64 or 128,
// n a multiple of 16 (m = 128) up to 256
__host__ __device__ constexpr uint32_t umma_idesc(uint32_t fmt, uint32_t m, uint32_t n) {
  return (1u << 4) | (fmt << 7) | (fmt << 10) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

// D (tensor memory) (+)= A B^T, A and B TF32 from shared memory
__device__ __forceinline__ void umma_tf32_i(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// both operands BF16 (one type for A and B, as kind::f16 requires)
__device__ __forceinline__ void umma_bf16_i(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(tmem_d),
      "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// arrive on a shared-memory mbarrier once every MMA issued before completes
__device__ __forceinline__ void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

}  // namespace rb
