// Tensor-memory-accelerator (TMA) staging of the resident sweeps' tiles.
//
// A tensor map describes one of the problem arrays as a 4-D tensor
//   blocks:  {n columns, n rows, block index, batch}          (L, E)
//   vectors: {m columns, n rows, block index, batch}          (X)
// and one cp.async.bulk.tensor copies a whole tile -- a factor / coupling
// block, or a 32-column chunk of a node's vectors -- into shared memory, with
// the completion counted on an mbarrier (expect-tx bytes).  The box is wider
// than the tile (the padded shared row: res_ldm / res_ldy elements), so the
// padded layout the sweeps index comes straight out of the copy: columns
// past the tensor's extent are filled with zeros, columns of a next vector
// chunk land in the padding, which no product reads.
//
// Copies are unicast loads of this GPU's own memory (no cluster multicast).
// The maps are kernel parameters (__grid_constant__), encoded on the host per
// launch with cuTensorMapEncodeTiled.  Every wait is bounded (%globaltimer):
// on timeout the kernel sets g_tc_error = 2, waits once more (bounded) for
// the copies in flight and skips its result.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "tc_gemm.cuh"

namespace socu {

// bound of one TMA wait (0.2 s)
constexpr unsigned long long kTmaWaitNs = 200000000ull;

// Tensor maps of one sweep launch: L and E blocks, X vectors.  blocks / vecs
// say which maps are valid (alignment allowed the encoding).
struct alignas(64) SweepMaps {
  CUtensorMap L, E, X;
  int blocks, vecs;
};

namespace tma {

// one thread: arrive on bar and add `bytes` to the transaction count of its current phase
__device__ __forceinline__ void expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(tc::saddr(bar)), "r"(bytes)
               : "memory");
}

// one thread: tile (x, y, z, w) of the 4-D map into shared memory at dst (128-byte aligned),
// completion counted on bar
__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                        uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];\n" ::"r"(tc::saddr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(tc::saddr(bar))
      : "memory");
}

// earlier generic-proxy accesses of shared memory ordered before the async proxy's writes
__device__ __forceinline__ void fence_proxy() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// every thread: wait for phase `parity` of bar (bounded); false on timeout, the
// same answer in every thread of the CTA
__device__ __forceinline__ bool wait(uint64_t* bar, unsigned parity) {
  const bool done = tc::mbar_wait(bar, parity, kTmaWaitNs);
  const bool ok = __syncthreads_and(done) != 0;
  if (!ok) {
    tc::mbar_wait(bar, parity, kTmaWaitNs);   // copies still in flight into this CTA's shared memory
    if (threadIdx.x == 0) atomicExch(&tc::g_tc_error, 2);
  }
  return ok;
}

}  // namespace tma
}  // namespace socu
