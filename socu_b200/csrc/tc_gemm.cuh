// Blackwell 5th-generation tensor cores (tcgen05, sm_100a) for the float
// path: a CTA-level GEMM with FP32 operands split into TF32 pieces (3xTF32:
// a*b ~ ah*bh + ah*bl + al*bh with ah = tf32(a), al = tf32(a - ah)), FP32
// accumulation in tensor memory (TMEM), issued by one thread.
//
//   D (128 x N) (+)= A (128 x K) * B (N x K)^T
//
// Operands live in shared memory in the canonical K-major, no-swizzle
// tcgen05 layout: "core matrices" of 8 rows x 16 bytes (8 x 4 floats),
// stored row-group-major:
//   byte offset of (m, k) = (m / 8) * (K / 4) * 128 + (k / 4) * 128 + (m % 8) * 16 + (k % 4) * 4
// so one MMA (K = 8 tf32 elements = two 16-byte chunks) at k-step s starts at
// base + 2 s * 128, steps 128 bytes between its two K chunks (leading byte
// offset) and (K / 4) * 128 bytes between 8-row groups (stride byte offset).
// Each operand has a hi and a lo plane of that layout.
//
// The accumulator is 128 TMEM lanes (one per row) x N 32-bit columns; warp w
// of the CTA reads lanes 32 (w % 4) .. 32 (w % 4) + 31 with tcgen05.ld.
//
// Every wait here is bounded (%globaltimer): on timeout the caller's error
// word is set and the CTA carries on without the result, so a fault in the
// tensor-core path cannot hang the GPU.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace socu {
namespace tc {

__device__ __forceinline__ uint32_t saddr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Error word of the asynchronous units on one device: 1 a tensor-core wait
// ran out, 2 a TMA copy wait ran out (that kernel skipped its result).
__device__ int g_tc_error;

// ---- instruction / shared-memory descriptors --------------------------------
// kind::tf32 instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major (bits 15, 16 = 0), N >> 3 at bit 17,
// M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// K-major, no-swizzle shared-memory descriptor: start address, leading byte
// offset (between the two K chunks of one MMA) and stride byte offset
// (between 8-row groups), each >> 4 in 14 bits; version 1 at bit 46;
// base offset 0, legacy LBO mode, layout type 0 (no swizzle).
__host__ __device__ constexpr uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// byte offset of element (m, k) in an operand plane with K columns
__host__ __device__ constexpr uint32_t coff(int m, int k, int K) {
  return (uint32_t)((m >> 3) * (K >> 2) * 128 + (k >> 2) * 128 + (m & 7) * 16 + (k & 3) * 4);
}

// ---- mbarrier ----------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(saddr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long globaltimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for phase `parity` of `bar` to complete, at most timeout_ns; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, unsigned long long timeout_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer();
  while (!mbar_try_wait(bar, parity)) {
    if (globaltimer() - t0 > timeout_ns) return false;
  }
  return true;
}

// ---- fences ----------------------------------------------------------------
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// ---- tensor memory ----------------------------------------------------------
// warp-wide: allocate ncols (power of two >= 32) TMEM columns, address to *dst
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(saddr(dst)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}

// warp-wide
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// one thread: D (+)= A * B^T for one K = 8 step (tf32, cta_group::1)
__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

// one thread: arrive on `bar` when every MMA issued so far by this thread has completed
__device__ __forceinline__ void commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(saddr(bar))
               : "memory");
}

// warp-wide: 32 lanes x 8 consecutive 32-bit columns; thread t gets lane (taddr lane + t)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

// warp-wide: 32 lanes x 8 consecutive 32-bit columns from registers; thread t writes lane (taddr lane + t)
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const float (&v)[8]) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};\n" ::"r"(taddr),
               "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
               "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
               "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7]))
               : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// ---- TF32 split --------------------------------------------------------------
// round-to-nearest TF32 (10 explicit mantissa bits) of an FP32 value; the
// remainder a - hi is exact in FP32
__device__ __forceinline__ float tf32_hi(float a) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(a));
  return __uint_as_float(r);
}

// Store value v of operand element (m, k) into the hi / lo planes.  The
// remainder is rounded to TF32 as well (the tensor core would otherwise drop
// its low 13 mantissa bits, a truncation): each of the two pieces is then
// within half a TF32 unit, and a product of split operands misses only
// ~2^-23 of |a b| -- the FP32 rounding level.
__device__ __forceinline__ void put_split(unsigned char* hi, unsigned char* lo, int m, int k, int K, float v) {
  const uint32_t o = coff(m, k, K);
  const float h = tf32_hi(v);
  *reinterpret_cast<float*>(hi + o) = h;
  *reinterpret_cast<float*>(lo + o) = tf32_hi(v - h);
}

// One thread: the 3xTF32 MMAs of D (M x N) (+)= A * B^T over K (multiple of
// 8), operand planes at shared addresses a_hi, a_lo (M rows x K) and b_hi,
// b_lo (N rows x K) in the layout above; accumulate = 0 overwrites D first.
__device__ __forceinline__ void gemm_3xtf32(uint32_t d_tmem, uint32_t a_hi, uint32_t a_lo, uint32_t b_hi,
                                            uint32_t b_lo, int N, int K, uint32_t accumulate, int M = 128) {
  const uint32_t idesc = idesc_tf32(M, N);
  const uint32_t sbo = (uint32_t)(K >> 2) * 128u;
  for (int s = 0; s < K / 8; ++s) {
    const uint32_t off = (uint32_t)s * 256u;
    const uint64_t ah = sdesc(a_hi + off, 128u, sbo), al = sdesc(a_lo + off, 128u, sbo);
    const uint64_t bh = sdesc(b_hi + off, 128u, sbo), bl = sdesc(b_lo + off, 128u, sbo);
    // small cross terms first, the hi*hi term last
    mma_tf32(d_tmem, al, bh, idesc, (s > 0 || accumulate) ? 1u : 0u);
    mma_tf32(d_tmem, ah, bl, idesc, 1u);
    mma_tf32(d_tmem, ah, bh, idesc, 1u);
  }
}

}  // namespace tc
}  // namespace socu
