// Level node of a FLOAT factor for 64 < n <= 128 with the node's whole
// working set resident in tensor memory (TMEM) and the trailing updates of a
// right-looking blocked Cholesky on the tcgen05 tensor cores.
//
// socu: potrf K2 fused with trsm_rltn / trsm_llnn (K3/K4) and the forward
// step, socu/block_tridiag_solver.py:197-279, :108-110.  Same results layout
// as node_body (nd_kernels.cuh): lower(L_i) = C_i, zero strict upper triangle,
// R <- R C^{-T}, Lf <- C^{-1} Lf, y <- C^{-1} y.
//
// State, one TMEM lane per block row r (M = 128; rows n..127 unused):
//   columns [0, n)          the block L_i (lower triangle meaningful)
//   columns [VO, VO + NV)   the node's vectors, VO = n rounded up to 16:
//                           R^T (nr), Lf (nl), y (m) -- NV = nr + nl + m
// For each 32-column panel [P0, P1):
//   a. tcgen05.ld: the diagonal block A11 (rows P0..P1) into shared memory,
//      the panel below it transposed, and the vectors' rows P0..P1, side by
//      side in one shared array Vc (32 rows):
//         Vc = [ A21^T (n - P1 columns) | zeros (VO - n) | V1 (NV columns) ]
//      so that column j of Vc is TMEM column P1 + j;
//   b. the panel chain on SIMT cores (cta_chol_solve): C11 = chol(A11) and
//      Vc <- C11^{-1} Vc, i.e. A21 <- A21 C11^{-T} (the factor's panel P)
//      and V1 <- C11^{-1} V1 (final rows of the solved vectors);
//   c. C11, P and V1 go straight to global memory (final values);
//   d. trailing update of every remaining row in one MMA group per 256
//      columns, accumulating into TMEM:
//         D[r][P1 + j] += (-P)[r] . Vc[:, j]      (r >= P1)
//      which is A22 -= P P^T for j < n - P1 and V2 -= P V1 for the vector
//      columns.  Operands: A = -P (128 x 32, rows < P1 zero), B = Vc^T, each
//      split into TF32 hi/lo planes (3xTF32, FP32 accumulation).
// Waits on the tensor core are bounded (g_tc_error = 1 and the node stops).
// One CTA per SM (shared memory ~180 KB at n = 128, 32 right-hand sides).
#pragma once

#include "tc_update.cuh"

namespace socu {

constexpr int kTmPW = 32;   // panel width
__host__ __device__ inline int tm_vo(int n) { return ((n + 15) / 16) * 16; }
// vector columns of the largest node (both coupling slots, m right-hand sides)
__host__ __device__ inline int tm_nv_max(int n, int m) { return 2 * n + m; }
// shared row length of Vc (odd: the transposed stores hit distinct banks)
__host__ __device__ inline int tm_ldc(int n, int m) { return (tm_vo(n) - kTmPW + tm_nv_max(n, m)) | 1; }
__host__ __device__ inline long long tm_a11_bytes() { return round128((long long)kTmPW * (kTmPW + 1) * 4); }
__host__ __device__ inline long long tm_vc_bytes(int n, int m) { return round128((long long)kTmPW * tm_ldc(n, m) * 4); }
__host__ __device__ inline long long tm_ap_bytes() { return 128LL * kTmPW * 4; }   // one plane
__host__ __device__ inline long long tm_bp_bytes(int n, int m) {                    // one plane
  return (long long)tc_ncols(tm_vo(n) - kTmPW + tm_nv_max(n, m)) * kTmPW * 4;
}
__host__ __device__ inline long long smem_node_tm_bytes(int n, int m) {
  return tm_a11_bytes() + tm_vc_bytes(n, m) + 2 * tm_ap_bytes() + 2 * tm_bp_bytes(n, m);
}
// TMEM columns the node touches: the state plus the padding of the last MMA group
__host__ __device__ inline int tm_cols_used(int n, int nv) { return tm_vo(n) + nv + 16; }
__host__ __device__ inline bool node_tm_ok(int n, int m) {
  return n > 64 && n <= 128 && m >= 0 && tm_cols_used(n, tm_nv_max(n, m)) <= 512;
}

template <bool WITH_Y>
__device__ __forceinline__ void node_tm_body(const Problem<float>& p, const Level& lv, int b, int t,
                                             unsigned char* smem, uint32_t tm, uint64_t* bar) {
  const int n = p.n, s = lv.s, i = s - 1 + 2 * s * t, m = p.m;
  const bool right = i + s < p.N, left = t >= 1;
  const int nr = right ? n : 0, nl = left ? n : 0, ny = WITH_Y ? m : 0;
  const int NV = nr + nl + ny, VO = tm_vo(n);
  const int ldc = tm_ldc(n, ny);   // shared sizes follow the launch's m (0 without y)
  float* Li = p.Lb(b, i);
  float* R = right ? p.Eb(b, lv.oc + 2 * t) : nullptr;
  float* Lf = left ? p.Eb(b, lv.oc + 2 * t - 1) : nullptr;
  float* yi = WITH_Y ? p.Xb(b, i) : nullptr;
  float* A11 = reinterpret_cast<float*>(smem);
  float* Vc = reinterpret_cast<float*>(smem + tm_a11_bytes());
  unsigned char* a_hi = smem + tm_a11_bytes() + tm_vc_bytes(n, ny);
  unsigned char* a_lo = a_hi + tm_ap_bytes();
  unsigned char* b_hi = a_lo + tm_ap_bytes();
  unsigned char* b_lo = b_hi + tm_bp_bytes(n, ny);
  constexpr int lda = kTmPW + 1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, q = warp & 3, h = warp >> 2;
  const uint32_t lane_base = tm + ((uint32_t)(32 * q) << 16);

  // 0. state into TMEM (warp: lanes of its quadrant, half of the 8-column chunks)
  {
    const int r = 32 * q + lane;
    const int nch = (VO + NV + 7) / 8, half = (nch + 1) / 2;
    const int c_lo = h == 0 ? 0 : half, c_hi = h == 0 ? half : nch;
    if (32 * q < n) {
      for (int ch = c_lo; ch < c_hi; ++ch) {
        float v[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const int c = ch * 8 + e;
          float x = 0.0f;
          if (r < n) {
            if (c < n) {
              if (c <= r) x = Li[(long long)r * n + c];
            } else if (c >= VO && c < VO + NV) {
              const int v = c - VO;
              if (v < nr) x = R[(long long)v * n + r];
              else if (v < nr + nl) x = Lf[(long long)r * n + (v - nr)];
              else x = yi[(long long)r * m + (v - nr - nl)];
            }
          }
          v[e] = x;
        }
        tc::tmem_st8(lane_base + (uint32_t)(ch * 8), v);
      }
    }
    tc::tmem_wait_st();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();

  unsigned phase = 0;
  for (int P0 = 0; P0 < n; P0 += kTmPW) {
    const int P1 = min_i(P0 + kTmPW, n), pw = P1 - P0, nb = n - P1;
    const int vo = VO - P1;          // first vector column of Vc
    const int ncat = vo + NV;        // columns of Vc
    const int q0 = P0 / 32;
    const int nchp = (pw + 7) / 8;
    // a. TMEM -> shared memory
    if (q == q0) {
      for (int ch = h; ch < nchp; ch += 2) {
        float v[8];
        tc::tmem_ld8(lane_base + (uint32_t)(P0 + 8 * ch), v);
        tc::tmem_wait_ld();
        if (lane < pw) {
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (8 * ch + e < pw) A11[lane * lda + 8 * ch + e] = v[e];
        }
      }
      for (int ch = h; ch < (NV + 7) / 8; ch += 2) {
        float v[8];
        tc::tmem_ld8(lane_base + (uint32_t)(VO + 8 * ch), v);
        tc::tmem_wait_ld();
        if (lane < pw) {
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (8 * ch + e < NV) Vc[lane * ldc + vo + 8 * ch + e] = v[e];
        }
      }
    } else if (q > q0 && 32 * q < n) {
      const int j = 32 * q + lane - P1;   // row P1 + j of the panel below
      for (int ch = h; ch < nchp; ch += 2) {
        float v[8];
        tc::tmem_ld8(lane_base + (uint32_t)(P0 + 8 * ch), v);
        tc::tmem_wait_ld();
        if (j < nb) {
#pragma unroll
          for (int e = 0; e < 8; ++e)
            if (8 * ch + e < pw) Vc[(8 * ch + e) * ldc + j] = v[e];
        }
      }
    }
    // zero columns between the panel rows and the vectors (n not a multiple of 16)
    for (int e = threadIdx.x; e < pw * (vo - nb); e += blockDim.x) {
      const int k = e / (vo - nb), j = nb + e - k * (vo - nb);
      Vc[k * ldc + j] = 0.0f;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();

    // b. panel chain: C11 = chol(A11), Vc <- C11^{-1} Vc
    cta_chol_solve<float, true>(A11, lda, pw, Vc, ldc, ncat);
    if (p.info != nullptr) {
      bool bad = false;
      for (int r = threadIdx.x; r < pw; r += blockDim.x) {
        const float d = A11[r * lda + r];
        bad = bad || !(d > 0.0f) || isinf(d);
      }
      if (__syncthreads_or(bad) && threadIdx.x == 0) record_failure(p.info + b, i);
    }

    // c. final values of this panel to global memory
    for (int e = threadIdx.x; e < pw * n; e += blockDim.x) {   // rows P0..P1 of L_i: C11 and zeros
      const int r = e / n, c = e - r * n;
      if (c < P0) continue;                                    // written with earlier panels
      Li[(long long)(P0 + r) * n + c] = (c < P1 && c - P0 <= r) ? A11[r * lda + (c - P0)] : 0.0f;
    }
    for (int e = threadIdx.x; e < nb * pw; e += blockDim.x) {   // P: rows P1.., columns P0..P1
      const int j = e / pw, k = e - j * pw;
      Li[(long long)(P1 + j) * n + P0 + k] = Vc[k * ldc + j];
    }
    for (int e = threadIdx.x; e < nr * pw; e += blockDim.x) {   // F = R C^{-T}: row v, columns P0..P1
      const int v = e / pw, k = e - v * pw;
      R[(long long)v * n + P0 + k] = Vc[k * ldc + vo + v];
    }
    for (int e = threadIdx.x; e < pw * nl; e += blockDim.x) {   // G = C^{-1} Lf: rows P0..P1
      const int k = e / nl, v = e - k * nl;
      Lf[(long long)(P0 + k) * n + v] = Vc[k * ldc + vo + nr + v];
    }
    if (WITH_Y)
      for (int e = threadIdx.x; e < pw * ny; e += blockDim.x) {   // y rows P0..P1
        const int k = e / ny, v = e - k * ny;
        yi[(long long)(P0 + k) * m + v] = Vc[k * ldc + vo + nr + nl + v];
      }

    // d. trailing update of rows P1.. on the tensor cores
    if (P1 < n) {
      tc_stage_kc<kTmPW>(a_hi, a_lo, 128, 128, kTmPW, 0, [&](int r, int k) {
        return (r >= P1 && r < n && k < pw) ? -Vc[k * ldc + (r - P1)] : 0.0f;
      });
      const int ncp = tc_ncols(ncat);
      tc_stage_kc<kTmPW>(b_hi, b_lo, ncp, ncat, kTmPW, 0,
                         [&](int j, int k) { return k < pw ? Vc[k * ldc + j] : 0.0f; });
      tc::fence_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      tc::fence_after_sync();
      if (threadIdx.x == 0) {
        for (int g0 = 0; g0 < ncp; g0 += 256) {
          const int ng = min_i(256, ncp - g0);
          tc::gemm_3xtf32(tm + (uint32_t)(P1 + g0), tc::saddr(a_hi), tc::saddr(a_lo),
                          tc::saddr(b_hi) + (uint32_t)g0 * 128u, tc::saddr(b_lo) + (uint32_t)g0 * 128u, ng,
                          kTmPW, 1u, 128);
        }
        tc::commit(bar);
      }
      const bool done = tc::mbar_wait(bar, phase & 1u, kTcWaitNs);
      const bool ok = __syncthreads_and(done) != 0;
      tc::fence_after_sync();
      if (!ok) {
        tc::mbar_wait(bar, phase & 1u, kTcWaitNs);   // MMAs still in flight before TMEM is freed
        if (threadIdx.x == 0) atomicExch(&g_tc_error, 1);
        return;
      }
      ++phase;
    }
    __syncthreads();   // shared arrays are rewritten by the next panel
  }
}

template <bool WITH_Y>
__global__ void __launch_bounds__(256, 1) k_node_tm(Problem<float> p, Level lv) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  const int b = blockIdx.x / lv.d;
  const int t = blockIdx.x - b * lv.d;
  pdl_wait();
  pdl_trigger();
  if (!p.active(b)) return;
  const int i = lv.s - 1 + 2 * lv.s * t;
  const int nv = (i + lv.s < p.N ? p.n : 0) + (t >= 1 ? p.n : 0) + (WITH_Y ? p.m : 0);
  const int used = tm_cols_used(p.n, nv);
  const uint32_t ncols = used <= 32 ? 32u : (used <= 64 ? 64u : (used <= 128 ? 128u : (used <= 256 ? 256u : 512u)));
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tc::tmem_alloc(&tbase, ncols);
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  node_tm_body<WITH_Y>(p, lv, b, t, smem_raw, tbase, &bar);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tbase, ncols);
}

}  // namespace socu
