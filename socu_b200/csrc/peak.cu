// Peak-throughput probe of the FP64 tensor-core pipe (DMMA, mma.sync m8n8k4
// .f64) on this device, for the FP64 roofline: MEASURED peaks of the device
// cover HBM bandwidth and BF16 GEMMs only.  Every warp runs kChains
// independent accumulator chains of `iters` m8n8k4 steps on register
// operands (no memory traffic); one step is 8 x 8 x 4 multiply-adds = 512
// flops.  The caller times the launch with CUDA events on `stream`.
#include <cuda_runtime.h>

#include "../../include/socu_b200.h"

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_dmma_peak(int iters, double* sink) {
  double a = 1.0 + 1e-3 * (threadIdx.x & 31), b = 1.0 - 1e-6 * (blockIdx.x & 1023);
  double c[kChains][2];
#pragma unroll
  for (int j = 0; j < kChains; ++j) c[j][0] = c[j][1] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < kChains; ++j)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(c[j][0]), "+d"(c[j][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int j = 0; j < kChains; ++j) s += c[j][0] + c[j][1];
  if (s == -1.0) sink[0] = s;   // keeps the chains live; never true for these operands
}

}  // namespace

extern "C" int socu_dmma_peak_launch(int64_t blocks, int threads, int iters, double* sink, void* stream,
                                     double* flops) {
  if (blocks <= 0 || blocks >= (1LL << 31) || threads <= 0 || threads > 256 || (threads & 31) != 0 || iters <= 0)
    return SOCU_ERR_INVALID_ARGUMENT;
  if (flops) *flops = (double)blocks * (threads / 32) * (double)iters * kChains * 512.0;
  k_dmma_peak<<<(unsigned)blocks, threads, 0, static_cast<cudaStream_t>(stream)>>>(iters, sink);
  return cudaGetLastError() == cudaSuccess ? SOCU_OK : SOCU_ERR_CUDA;
}
