// Self-test of the tcgen05 building block (tc_gemm.cuh): one CTA computes
// D (M x N) = A (M x K) * B (N x K)^T, M = 64 or 128, with the 3xTF32 split,
// FP32 accumulation in tensor memory, through exactly the staging,
// descriptor, MMA, commit and TMEM-load path the solver kernels use, and
// writes all 128 TMEM lanes of the accumulator's N columns to D (lane-major),
// so that the row-to-lane placement of an M = 64 accumulator can be checked
// too.  Exposed through the C ABI so that the path can be checked against a
// host reference in isolation.
#include <cuda_runtime.h>

#include "../../include/socu_b200.h"
#include "tc_gemm.cuh"

namespace {

using namespace socu;

constexpr unsigned long long kTcWaitNs = 200000000ull;   // 0.2 s bound of every tensor-core wait

__global__ void __launch_bounds__(256, 1) k_tc_selftest(const float* __restrict__ A, const float* __restrict__ B,
                                                         float* __restrict__ D, int M, int N, int K, int* err) {
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t ncols = N <= 32 ? 32u : (N <= 64 ? 64u : (N <= 128 ? 128u : 256u));
  unsigned char* a_hi = sm;
  unsigned char* a_lo = a_hi + 128 * K * 4;
  unsigned char* b_hi = a_lo + 128 * K * 4;
  unsigned char* b_lo = b_hi + N * K * 4;
  if (warp == 0) tc::tmem_alloc(&tbase, ncols);
  if (tid == 0) tc::mbar_init(&bar, 1);
  for (int e = tid; e < 128 * K; e += blockDim.x)
    tc::put_split(a_hi, a_lo, e / K, e % K, K, e / K < M ? A[e] : 0.0f);
  for (int e = tid; e < N * K; e += blockDim.x) tc::put_split(b_hi, b_lo, e / K, e % K, K, B[e]);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t d = tbase;
  if (tid == 0) {
    tc::gemm_3xtf32(d, tc::saddr(a_hi), tc::saddr(a_lo), tc::saddr(b_hi), tc::saddr(b_lo), N, K, 0u, M);
    tc::commit(&bar);
  }
  bool ok = tc::mbar_wait(&bar, 0, kTcWaitNs);
  tc::fence_after_sync();
  if (ok) {
    const int q = warp & 3, half = warp >> 2, nh = (N + 1) / 2;
    const int row = 32 * q + lane;
    for (int c0 = half * nh; c0 < min(N, (half + 1) * nh); c0 += 8) {
      float v[8];
      tc::tmem_ld8(d + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
      tc::tmem_wait_ld();
#pragma unroll
      for (int i = 0; i < 8; ++i)
        if (c0 + i < N) D[row * N + c0 + i] = v[i];
    }
  } else {
    atomicExch(err, 1);
    tc::mbar_wait(&bar, 0, kTcWaitNs);   // give MMAs still in flight a second bound before freeing TMEM
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(d, ncols);
}

}  // namespace

extern "C" int socu_tc_selftest(const float* A, const float* B, float* D, int64_t m_rows, int64_t n_cols,
                                int64_t k_depth, int* error_flag, void* stream) {
  if (A == nullptr || B == nullptr || D == nullptr || error_flag == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  if (m_rows != 64 && m_rows != 128) return SOCU_ERR_INVALID_ARGUMENT;
  if (n_cols < 16 || n_cols > 128 || n_cols % 16 != 0 || k_depth < 8 || k_depth % 8 != 0)
    return SOCU_ERR_INVALID_ARGUMENT;
  const size_t smem = (size_t)(128 + n_cols) * (size_t)k_depth * 4 * 2;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return SOCU_ERR_CUDA;
  if (smem + 1024 > (size_t)optin) return SOCU_ERR_UNSUPPORTED;
  if (cudaFuncSetAttribute(k_tc_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return SOCU_ERR_CUDA;
  k_tc_selftest<<<1, 256, smem, static_cast<cudaStream_t>(stream)>>>(A, B, D, (int)m_rows, (int)n_cols,
                                                                      (int)k_depth, error_flag);
  return cudaGetLastError() == cudaSuccess ? SOCU_OK : SOCU_ERR_CUDA;
}
