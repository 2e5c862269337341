// Device-side building blocks of the nested-dissection block-tridiagonal
// Cholesky (sm_100a).  Everything here works on one CTA's shared memory.
//
// Storage contract (identical to socu, socu/block_tridiag_solver.py:739-774):
//   L  (B, N, n, n)   diagonal blocks, lower triangle read, factor written
//   E  (B, S, n, n)   off-diagonal storage, S = off_diag_storage_len(N)
//   X  (B, N, n, m)   right-hand sides in, solution out
// Level l has stride s = 2^l and nodes i = s-1 + 2 s t, t < (N+s)/(2s)
// (socu/block_tridiag_solver.py:174).  Slot E[o_l + k] couples node
// p = (k+1)s-1 (columns) with q = p+s (rows).
//
// After a factor the upper triangle of every L block holds the strictly
// upper part of C^{-T} (C = lower Cholesky factor of that block).  The
// reference leaves that triangle unspecified; the substitution sweeps here
// only ever read the lower triangle, so factors are interchangeable with the
// reference's.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace socu {

template <typename T> __device__ __forceinline__ T rsqrt_t(T x);
template <> __device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float rsqrt_t<float>(float x) { return rsqrtf(x); }

template <typename T> __device__ __forceinline__ T rcp_t(T x) { return T(1) / x; }

template <typename T>
struct Problem {
  T* L;
  T* E;
  T* X;                  // may be null (factor only)
  const uint8_t* mask;   // may be null: all batch entries active
  int B, N, n, m, S;
  long long sL, sE, sX;  // per-batch strides in elements

  __device__ __forceinline__ T* Lb(int b, int i) const {
    return L + (long long)b * sL + (long long)i * n * n;
  }
  __device__ __forceinline__ T* Eb(int b, int slot) const {
    return E + (long long)b * sE + (long long)slot * n * n;
  }
  __device__ __forceinline__ T* Xb(int b, int i) const {
    return X + (long long)b * sX + (long long)i * n * m;
  }
  __device__ __forceinline__ bool active(int b) const { return mask == nullptr || mask[b] != 0; }
};

// One nested-dissection level (socu/block_tridiag_solver.py:869-914).
struct Level {
  int s;    // stride 2^l
  int d;    // nodes at this level, (N+s)/(2s)
  int oc;   // offset of this level's slots
  int on;   // offset of the next level's slots
};

// ---------------------------------------------------------------------------
// Register-tiled CTA GEMM on accessor functors.
//   acc(r,c) = sum_k a(r,k) * b(k,c) for 0<=r<M, 0<=c<N, k in [k0(r0,c0), K)
//   then out(r, c, acc) for every valid entry (and c <= r if LOWER).
// Threads own TM x TN micro-tiles; consecutive threads own consecutive
// column tiles so that row operands are broadcast within a warp.
// ---------------------------------------------------------------------------
template <typename T, int TM, int TN, bool LOWER, class FA, class FB, class FO>
__device__ __forceinline__ void cta_gemm(int M, int N, int K, FA a, FB b, FO out) {
  const int tm = (M + TM - 1) / TM;
  const int tn = (N + TN - 1) / TN;
  for (int t = threadIdx.x; t < tm * tn; t += blockDim.x) {
    const int r0 = (t / tn) * TM;
    const int c0 = (t % tn) * TN;
    if (LOWER && c0 > r0 + TM - 1) continue;
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
    for (int k = 0; k < K; ++k) {
      T av[TM], bv[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) av[i] = (r0 + i < M) ? a(r0 + i, k) : T(0);
#pragma unroll
      for (int j = 0; j < TN; ++j) bv[j] = (c0 + j < N) ? b(k, c0 + j) : T(0);
#pragma unroll
      for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) {
        const int r = r0 + i, c = c0 + j;
        if (r < M && c < N && (!LOWER || c <= r)) out(r, c, acc[i][j]);
      }
  }
}

// ---------------------------------------------------------------------------
// Global <-> shared block copies (row-major, contiguous rows of length cols).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void load_block(T* __restrict__ dst, int ld, const T* __restrict__ src,
                                           int rows, int cols, int src_ld) {
  const int total = rows * cols;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int r = e / cols, c = e - r * cols;
    dst[r * ld + c] = src[(long long)r * src_ld + c];
  }
}

template <typename T>
__device__ __forceinline__ void store_block(T* __restrict__ dst, int dst_ld, const T* __restrict__ src,
                                            int ld, int rows, int cols) {
  const int total = rows * cols;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int r = e / cols, c = e - r * cols;
    dst[(long long)r * dst_ld + c] = src[r * ld + c];
  }
}

// ---------------------------------------------------------------------------
// One warp: in-place lower Cholesky of a kb x kb diagonal block (kb <= 32)
// followed by the inverse of that factor.
//   on exit: lower(A) = C, A[c*ld + r] = (C^{-1})[r][c] for r > c,
//            dinv[r] = 1 / C[r][r].
// Right-looking column steps; lane r owns row r.
// ---------------------------------------------------------------------------
template <typename T>
__device__ void warp_chol_inv(T* A, int ld, int kb, T* dinv) {
  const int lane = threadIdx.x & 31;
  for (int j = 0; j < kb; ++j) {
    const T ajj = A[j * ld + j];
    const T rs = rsqrt_t(ajj);
    if (lane > j && lane < kb) A[lane * ld + j] *= rs;
    __syncwarp();
    if (lane == j) {
      A[j * ld + j] = ajj * rs;
      dinv[j] = rs;
    }
    if (lane > j && lane < kb) {
      const T lrj = A[lane * ld + j];
      for (int c = j + 1; c <= lane; ++c) A[lane * ld + c] = fma(-lrj, A[c * ld + j], A[lane * ld + c]);
    }
    __syncwarp();
  }
  // inverse W = C^{-1} (lower); S[r][c] = sum_{k=c}^{r-1} C[r][k] W[k][c]
  // accumulates in A[c*ld + r]; W[r][c] = -dinv[r] * S[r][c].
  if (lane < kb)
    for (int r = lane + 1; r < kb; ++r) A[lane * ld + r] = T(0);
  __syncwarp();
  for (int k = 0; k < kb; ++k) {
    if (lane < k) A[lane * ld + k] = -dinv[k] * A[lane * ld + k];
    __syncwarp();
    if (lane <= k) {
      const T wkc = (lane == k) ? dinv[k] : A[lane * ld + k];
      for (int r = k + 1; r < kb; ++r) A[lane * ld + r] = fma(A[r * ld + k], wkc, A[lane * ld + r]);
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------------------
// CTA: blocked right-looking Cholesky of the n x n block in A (lower read)
// plus the full inverse of the factor.
//   on exit: lower(A) = C, strict upper(A) = strict upper of C^{-T},
//            dinv[r] = 1 / C[r][r].
// P is scratch of n * BS elements.
// ---------------------------------------------------------------------------
template <typename T, int BS>
__device__ void cta_chol_inv(T* A, int ld, int n, T* dinv, T* P) {
  const int warp = threadIdx.x >> 5;
  for (int K = 0; K < n; K += BS) {
    const int kb = min(BS, n - K);
    if (warp == 0) warp_chol_inv<T>(A + K * ld + K, ld, kb, dinv + K);
    __syncthreads();
    const int R0 = K + kb, rows = n - R0;
    if (rows > 0) {
      // panel: C[R0+r][K+c] = sum_{k<=c} A[R0+r][K+k] * W_KK[c][k]
      cta_gemm<T, 2, 2, false>(
          rows, kb, kb,
          [&](int r, int k) { return A[(R0 + r) * ld + K + k]; },
          [&](int k, int c) { return k < c ? A[(K + k) * ld + K + c] : (k == c ? dinv[K + c] : T(0)); },
          [&](int r, int c, T v) { P[r * BS + c] = v; });
      __syncthreads();
      for (int e = threadIdx.x; e < rows * kb; e += blockDim.x) {
        const int r = e / kb, c = e - r * kb;
        A[(R0 + r) * ld + K + c] = P[r * BS + c];
      }
      // trailing: A[R0+r][R0+c] -= sum_k P[r][k] P[c][k]  (lower)
      cta_gemm<T, 2, 2, true>(
          rows, rows, kb,
          [&](int r, int k) { return P[r * BS + k]; },
          [&](int k, int c) { return P[c * BS + k]; },
          [&](int r, int c, T v) { A[(R0 + r) * ld + R0 + c] -= v; });
      __syncthreads();
    }
  }
  // off-diagonal blocks of W, block row by block row
  for (int I = BS; I < n; I += BS) {
    const int ib = min(BS, n - I);
    // Tm[r][c] = sum_{k=c}^{I-1} C[I+r][k] W[k][c]
    cta_gemm<T, 2, 2, false>(
        ib, I, I,
        [&](int r, int k) { return A[(I + r) * ld + k]; },
        [&](int k, int c) { return k > c ? A[c * ld + k] : (k == c ? dinv[c] : T(0)); },
        [&](int r, int c, T v) { P[r * I + c] = v; });
    __syncthreads();
    // W[I+r][c] = - sum_{k<=r} W_II[r][k] Tm[k][c], stored at A[c*ld + I + r]
    cta_gemm<T, 2, 2, false>(
        ib, I, ib,
        [&](int r, int k) { return k < r ? A[(I + k) * ld + I + r] : (k == r ? dinv[I + r] : T(0)); },
        [&](int k, int c) { return P[k * I + c]; },
        [&](int r, int c, T v) { A[c * ld + I + r] = -v; });
    __syncthreads();
  }
}

}  // namespace socu
