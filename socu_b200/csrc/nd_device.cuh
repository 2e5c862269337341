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
// Factor output: lower(L_i) = C_i (lower Cholesky factor).  The strict upper
// triangle is 0, or holds W_i^T with W_i = C_i^{-1} where a path keeps the
// diagonal inverses (factor_and_solve, the internal float factor of the mixed
// solve).  The reference leaves the upper triangle unspecified and every
// kernel here that is given a factor from outside reads only lower(L_i), so
// factors are interchangeable with socu's.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace socu {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBS = 32;  // row block of the blocked triangular solves

template <typename T> __device__ __forceinline__ T rsqrt_t(T x);
template <> __device__ __forceinline__ double rsqrt_t<double>(double x) { return rsqrt(x); }
template <> __device__ __forceinline__ float rsqrt_t<float>(float x) { return rsqrtf(x); }

template <typename T>
struct Problem {
  T* L;
  T* E;
  T* X;                  // may be null (factor only)
  const uint8_t* mask;   // may be null: all batch entries active
  int* info;             // may be null: per batch entry, 0 or 1 + the first node whose pivot failed
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

// Numerical status of one batch entry: node i failed to factor (a pivot
// <= 0, or a non-finite value).  info keeps the failing node that comes first
// in elimination order -- lowest level ctz(i+1), then lowest index -- so the
// result does not depend on which node of a level reports first.  LAPACK's
// potrf reports the failing column the same way (info > 0); the reference
// reports nothing (socu/blas/potrf.py:97-117 takes the square root of
// whatever pivot it meets).
__device__ __forceinline__ void record_failure(int* info, int i) {
  const int mine = i + 1;
  int cur = *reinterpret_cast<volatile int*>(info);
  while (true) {
    if (cur != 0) {
      const int lc = __ffs(cur) - 1, lm = __ffs(mine) - 1;
      if (lc < lm || (lc == lm && cur <= mine)) return;
    }
    const int prev = atomicCAS(info, cur, mine);
    if (prev == cur) return;
    cur = prev;
  }
}

// After the blocked Cholesky of node i (lower(A) = C, leading dimension lda):
// every diagonal entry must be a positive finite number.  All threads call it.
template <typename T>
__device__ __forceinline__ void check_factor(const Problem<T>& p, int b, int i, const T* A, int lda) {
  if (p.info == nullptr) return;
  bool bad = false;
  for (int r = threadIdx.x; r < p.n; r += blockDim.x) {
    const T d = A[r * lda + r];
    bad = bad || !(d > T(0)) || isinf(d);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) record_failure(p.info + b, i);
}

// One nested-dissection level (socu/block_tridiag_solver.py:869-914).
struct Level {
  int s;    // stride 2^l
  int d;    // nodes at this level, (N+s)/(2s)
  int oc;   // offset of this level's slots
  int on;   // offset of the next level's slots
  int op;   // offset of the previous level's slots (unused at level 0)
  int tc;   // sweeps on inverse-carrying factors: 1 = FP64 tensor-core (DMMA) products, 0 = SIMT row dots
  int tile; // output tile of the blocked Schur update (n > 64): 16 or 32
  int pre;  // sweeps: the factor blocks were complete before the previous kernel started, so they may be
            // loaded before the grid-dependency wait (programmatic dependent launch)
};

// Programmatic dependent launch (sm_90+).  A kernel launched with the
// programmatic-serialization attribute may start while its predecessor in the
// stream is still running; pdl_wait() returns once the predecessor grid has
// completed and its memory is visible, pdl_trigger() lets the successor start
// launching.  Both are no-ops for kernels launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// Asynchronous global -> shared copies (cp.async, element granular so that
// padded shared layouts are allowed).  Issue everything, then wait once.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

template <int BYTES>
__device__ __forceinline__ void cp_async_bytes(void* dst, const void* src) {
  if constexpr (BYTES == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(smem_addr(dst)), "l"(src), "n"(BYTES) : "memory");
}

template <typename T>
__device__ __forceinline__ void cp_async_elem(T* dst, const T* src) {
  cp_async_bytes<sizeof(T)>(dst, src);
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// widest copy (16, 8 or element bytes) that keeps every row chunk aligned
template <typename T>
__device__ __forceinline__ int copy_width(const T* dst, int ld, const T* src, int cols, long long src_ld) {
  const unsigned long long a = reinterpret_cast<unsigned long long>(src) |
                               (unsigned long long)smem_addr(dst) |
                               (unsigned long long)(cols * sizeof(T)) | (unsigned long long)(ld * sizeof(T)) |
                               (unsigned long long)(src_ld * (long long)sizeof(T));
  return (a & 15) == 0 ? 16 : ((a & 7) == 0 ? 8 : (int)sizeof(T));
}

template <typename T, int BYTES>
__device__ __forceinline__ void async_load_w(T* dst, int ld, const T* src, int rows, int cols, long long src_ld) {
  constexpr int V = BYTES / sizeof(T);
  const int cv = cols / V;
  const int total = rows * cv;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int r = e / cv, c = (e - r * cv) * V;
    cp_async_bytes<BYTES>(dst + r * ld + c, src + (long long)r * src_ld + c);
  }
}

// dst[r*ld + c] = src[r*src_ld + c]; vectorised when alignment allows
template <typename T>
__device__ __forceinline__ void async_load(T* dst, int ld, const T* src, int rows, int cols, long long src_ld) {
  const int w = copy_width(dst, ld, src, cols, src_ld);
  if (w == 16)
    async_load_w<T, 16>(dst, ld, src, rows, cols, src_ld);
  else if (w == 8)
    async_load_w<T, 8>(dst, ld, src, rows, cols, src_ld);
  else
    async_load_w<T, sizeof(T)>(dst, ld, src, rows, cols, src_ld);
}

// dst[c*ld + r] = src[r*src_ld + c]   (global rows become shared columns)
template <typename T>
__device__ __forceinline__ void async_load_t(T* dst, int ld, const T* src, int rows, int cols, long long src_ld) {
  const int total = rows * cols;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int r = e / cols, c = e - r * cols;
    cp_async_elem(dst + c * ld + r, src + (long long)r * src_ld + c);
  }
}

// even leading dimension (row starts 8/16-byte aligned) close to n
__host__ __device__ inline int even_ld(int n) { return n + ((n & 1) ? 1 : 2); }

template <typename T>
__device__ __forceinline__ void store_block(T* dst, long long dst_ld, const T* src, int ld, int rows, int cols) {
  const int total = rows * cols;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int r = e / cols, c = e - r * cols;
    dst[(long long)r * dst_ld + c] = src[r * ld + c];
  }
}

// dst[r*dst_ld + c] = src[c*ld + r]
template <typename T>
__device__ __forceinline__ void store_block_t(T* dst, long long dst_ld, const T* src, int ld, int rows, int cols) {
  const int total = rows * cols;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int r = e / cols, c = e - r * cols;
    dst[(long long)r * dst_ld + c] = src[c * ld + r];
  }
}

// ---------------------------------------------------------------------------
// Register-tiled CTA GEMM on shared-memory operands.
//   acc(r,c) = sum_{k<K} opA(r,k) opB(k,c),  0<=r<M, 0<=c<N
//   opA(r,k) = TA ? A[k*lda + r] : A[r*lda + k]
//   opB(k,c) = TB ? B[c*ldb + k] : B[k*ldb + c]
// then out(r, c, acc) for every valid entry (c <= r only if LOWER).
// Threads own TM x TN micro-tiles; consecutive threads take consecutive
// column tiles so row operands are broadcast inside a warp.  Out-of-range
// rows/columns are clamped for loading and masked on output, so the k-loop
// carries no branches.
// ---------------------------------------------------------------------------
template <typename T, int TM, int TN, bool TA, bool TB, bool LOWER = false, class Out>
__device__ __forceinline__ void smem_gemm(int M, int N, int K, const T* __restrict__ A, int lda,
                                          const T* __restrict__ B, int ldb, Out out) {
  const int tm = (M + TM - 1) / TM;
  const int tn = (N + TN - 1) / TN;
  for (int t = threadIdx.x; t < tm * tn; t += blockDim.x) {
    const int r0 = (t / tn) * TM;
    const int c0 = (t % tn) * TN;
    if (LOWER && c0 > r0 + TM - 1) continue;
    int ra[TM], cb[TN];
#pragma unroll
    for (int i = 0; i < TM; ++i) ra[i] = min(r0 + i, M - 1);
#pragma unroll
    for (int j = 0; j < TN; ++j) cb[j] = min(c0 + j, N - 1);
    T acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
      for (int j = 0; j < TN; ++j) acc[i][j] = T(0);
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
      T av[TM], bv[TN];
#pragma unroll
      for (int i = 0; i < TM; ++i) av[i] = TA ? A[k * lda + ra[i]] : A[ra[i] * lda + k];
#pragma unroll
      for (int j = 0; j < TN; ++j) bv[j] = TB ? B[cb[j] * ldb + k] : B[k * ldb + cb[j]];
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
// FP64 tensor-core (DMMA, mma.sync m8n8k4 f64) warp GEMM on shared operands
// of type T (float operands are widened to double in registers: exact
// products, FP64 sums).
//   acc(r,c) = sum_{k<K} opA(r,k) opB(k,c);  out(r, c, acc) per valid entry, acc a double.
// Warp tiles of 16 x 32 (2 x 4 mma tiles).  Fragment layouts (PTX ISA,
// mma.m8n8k4 .f64): A a0 = A[g][t], B b0 = B[t][g], C {c0,c1} = C[g][2t+{0,1}]
// with g = lane/4, t = lane%4.  Leading dimensions of 4 (mod 16) doubles make
// every fragment load conflict-free.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

__host__ __device__ inline int ld_dmma(int n) { return ((n + 15) / 16) * 16 + 4; }

template <typename T, bool TA, bool TB, bool LOWER = false, class Out>
__device__ __forceinline__ void warp_gemm_dmma(int M, int N, int K, const T* __restrict__ A, int lda,
                                               const T* __restrict__ B, int ldb, Out out) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int tm = (M + 15) / 16, tn = (N + 31) / 32;
  for (int tile = warp; tile < tm * tn; tile += nw) {
    const int r0 = (tile / tn) * 16, c0 = (tile % tn) * 32;
    if (LOWER && c0 > r0 + 15) continue;
    double acc[2][4][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    int ra[2], cb[4];
#pragma unroll
    for (int i = 0; i < 2; ++i) ra[i] = min(r0 + 8 * i + g, M - 1);
#pragma unroll
    for (int j = 0; j < 4; ++j) cb[j] = min(c0 + 8 * j + g, N - 1);
#pragma unroll 2
    for (int k0 = 0; k0 < K; k0 += 4) {
      const int k = k0 + t;
      const bool kv = k < K;
      const int kc = kv ? k : K - 1;
      double a[2], b[4];
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const double v = (double)(TA ? A[kc * lda + ra[i]] : A[ra[i] * lda + kc]);
        a[i] = kv ? v : 0.0;
      }
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double v = (double)(TB ? B[cb[j] * ldb + kc] : B[kc * ldb + cb[j]]);
        b[j] = kv ? v : 0.0;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int r = r0 + 8 * i + g, c = c0 + 8 * j + 2 * t + e;
          if (r < M && c < N && (!LOWER || c <= r)) out(r, c, acc[i][j][e]);
        }
  }
}

// Type-dispatching CTA GEMM: DMMA for double, 4x4 SIMT micro-tiles for float.
template <typename T, bool TA, bool TB, bool LOWER = false, class Out>
__device__ __forceinline__ void cta_gemm(int M, int N, int K, const T* __restrict__ A, int lda,
                                         const T* __restrict__ B, int ldb, Out out) {
  if constexpr (sizeof(T) == 8)
    warp_gemm_dmma<double, TA, TB, LOWER>(M, N, K, A, lda, B, ldb, out);
  else
    smem_gemm<T, 4, 4, TA, TB, LOWER>(M, N, K, A, lda, B, ldb, out);
}


// ---------------------------------------------------------------------------
// Trailing update of one 8-column step of cta_chol_solve, both parts in one
// tile loop (rows R0..n-1, P = A[R0.., K..K+kb) the solved panel):
//   A22[r][c] -= sum_k P[r][k] P[c][k]        (c <= r; only when factoring)
//   V[r][c]   -= sum_k P[r][k] V[K+k][c]      (c < nv)
// The accumulators start from the target values and the panel operand is
// negated, so a tile ends in a plain store.  FP64: DMMA warp tiles of 16 x 32
// (fragment layout of mma.m8n8k4 .f64: a0 = A[g][t], b0 = B[t][g],
// {c0, c1} = C[g][2t + {0, 1}], g = lane/4, t = lane%4).  FP32: 4 x 4 SIMT
// micro-tiles per thread.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void rank_update_f64(double* A, int lda, double* V, int ldv, int n, int K, int kb,
                                                int R0, int nv, bool factor) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int M = n - R0;
  const int tm = (M + 15) / 16;
  const int tnA = factor ? (M + 31) / 32 : 0, tnV = (nv + 31) / 32;
  const int nA = tm * tnA, total = nA + tm * tnV;
  const double* P = A + R0 * lda + K;
  for (int tile = warp; tile < total; tile += nw) {
    const bool isA = tile < nA;
    const int tt = isA ? tile : tile - nA;
    const int tn = isA ? tnA : tnV;
    const int r0 = (tt / tn) * 16, c0 = (tt % tn) * 32;
    if (isA && c0 > r0 + 15) continue;
    double* C = isA ? A + R0 * lda + R0 : V + R0 * ldv;
    const int ldc = isA ? lda : ldv;
    const int N = isA ? M : nv;
    double acc[2][4][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int r = r0 + 8 * i + g, c = c0 + 8 * j + 2 * t + e;
          acc[i][j][e] = (r < M && c < N) ? C[r * ldc + c] : 0.0;
        }
    int ra[2], cb[4];
#pragma unroll
    for (int i = 0; i < 2; ++i) ra[i] = min(r0 + 8 * i + g, M - 1);
#pragma unroll
    for (int j = 0; j < 4; ++j) cb[j] = min(c0 + 8 * j + g, N - 1);
#pragma unroll
    for (int k0 = 0; k0 < 8; k0 += 4) {
      const int k = k0 + t;
      const bool kv = k < kb;
      const int kc = kv ? k : 0;
      double a[2], b[4];
#pragma unroll
      for (int i = 0; i < 2; ++i) a[i] = kv ? -P[ra[i] * lda + kc] : 0.0;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const double v = isA ? P[cb[j] * lda + kc] : V[(K + kc) * ldv + cb[j]];
        b[j] = kv ? v : 0.0;
      }
#pragma unroll
      for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int r = r0 + 8 * i + g, c = c0 + 8 * j + 2 * t + e;
          if (r < M && c < N && (!isA || c <= r)) C[r * ldc + c] = acc[i][j][e];
        }
  }
}

template <typename T>
__device__ __forceinline__ void rank_update_simt(T* A, int lda, T* V, int ldv, int n, int K, int kb, int R0, int nv,
                                                 bool factor) {
  constexpr int BK = 8;
  const int M = n - R0;
  const int tm = (M + 3) / 4;
  const int tnA = factor ? (M + 3) / 4 : 0, tnV = (nv + 3) / 4;
  const int nA = tm * tnA, total = nA + tm * tnV;
  const T* P = A + R0 * lda + K;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const bool isA = idx < nA;
    const int tt = isA ? idx : idx - nA;
    const int tn = isA ? tnA : tnV;
    const int r0 = (tt / tn) * 4, c0 = (tt % tn) * 4;
    if (isA && c0 > r0 + 3) continue;
    T* C = isA ? A + R0 * lda + R0 : V + R0 * ldv;
    const int ldc = isA ? lda : ldv;
    const int N = isA ? M : nv;
    T acc[4][4];
    int ra[4], cb[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) ra[i] = min(r0 + i, M - 1);
#pragma unroll
    for (int j = 0; j < 4; ++j) cb[j] = min(c0 + j, N - 1);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = C[ra[i] * ldc + cb[j]];
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      if (k < kb) {
        T a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = P[ra[i] * lda + k];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = isA ? P[cb[j] * lda + k] : V[(K + k) * ldv + cb[j]];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(-a[i], b[j], acc[i][j]);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int r = r0 + i, c = c0 + j;
        if (r < M && c < N && (!isA || c <= r)) C[r * ldc + c] = acc[i][j];
      }
  }
}

// Float rank-kb update with the solved panel also held transposed in Pt
// (Pt[k * ldt + row], written by the item solves): the row operand of every
// tile and the column operand of the A22 tiles are 16-byte loads of
// consecutive rows, and with VEC_V (ldv a multiple of 4) the vector operand
// too.  Same tiles, values and order as rank_update_simt: identical results.
template <bool VEC_V>
__device__ __forceinline__ void rank_update_simt_pt(float* A, int lda, float* V, int ldv, int n, int K, int kb,
                                                    int R0, int nv, bool factor, const float* Pt, int ldt) {
  constexpr int BK = 8;
  const int M = n - R0;
  const int tm = (M + 3) / 4;
  const int tnA = factor ? (M + 3) / 4 : 0, tnV = (nv + 3) / 4;
  const int nA = tm * tnA, total = nA + tm * tnV;
  for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
    const bool isA = idx < nA;
    const int tt = isA ? idx : idx - nA;
    const int tn = isA ? tnA : tnV;
    const int r0 = (tt / tn) * 4, c0 = (tt % tn) * 4;
    if (isA && c0 > r0 + 3) continue;
    float* C = isA ? A + R0 * lda + R0 : V + R0 * ldv;
    const int ldc = isA ? lda : ldv;
    const int N = isA ? M : nv;
    float acc[4][4];
    int ra[4], cb[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) ra[i] = min(r0 + i, M - 1);
#pragma unroll
    for (int j = 0; j < 4; ++j) cb[j] = min(c0 + j, N - 1);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = C[ra[i] * ldc + cb[j]];
#pragma unroll
    for (int k = 0; k < BK; ++k) {
      if (k < kb) {
        const float4 a4 = *reinterpret_cast<const float4*>(Pt + k * ldt + R0 + r0);
        const float a[4] = {a4.x, a4.y, a4.z, a4.w};
        float b[4];
        if (isA) {
          const float4 b4 = *reinterpret_cast<const float4*>(Pt + k * ldt + R0 + c0);
          b[0] = b4.x; b[1] = b4.y; b[2] = b4.z; b[3] = b4.w;
        } else if (VEC_V) {
          const float4 b4 = *reinterpret_cast<const float4*>(V + (K + k) * ldv + c0);
          b[0] = b4.x; b[1] = b4.y; b[2] = b4.z; b[3] = b4.w;
        } else {
#pragma unroll
          for (int j = 0; j < 4; ++j) b[j] = V[(K + k) * ldv + cb[j]];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acc[i][j] = fma(-a[i], b[j], acc[i][j]);
      }
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int r = r0 + i, c = c0 + j;
        if (r < M && c < N && (!isA || c <= r)) C[r * ldc + c] = acc[i][j];
      }
  }
}

// ---------------------------------------------------------------------------
// CTA: blocked right-looking Cholesky of the n x n block in A fused with the
// solve C V = V for nv vectors (columns of V), by 8-column blocks.
//   1. every thread loads the diagonal block into registers and (when
//      FACTOR) factors it redundantly: no communication on the critical chain;
//   2. one thread per item solves against that block: each row of the panel
//      below it (A21 <- A21 C11^{-T}) and each vector segment
//      (V1 <- C11^{-1} V1) -- the same forward substitution;
//   3. trailing updates A22 -= P P^T (lower) and V2 -= P V1 with
//      P = the solved panel (tensor cores for double).
// FACTOR = false re-runs the solve with an already factored lower(A) = C.
// On exit lower(A) = C.  Two barriers per block.
// ---------------------------------------------------------------------------
// IDENTITY: V starts as the n x n identity (nv = n), so it ends as C^{-1}.
// Rows [K, K+kb) of column c are still zero for c >= K+kb, which leaves those
// columns out of the item solves and of the trailing update.
// Pt (float, optional, 8 x ldt with ldt >= n rounded up to 4 + 4, 16-byte
// aligned): transposed copy of each solved panel for rank_update_simt_pt.
template <typename T, bool FACTOR, bool IDENTITY = false>
__device__ void cta_chol_solve(T* A, int lda, int n, T* V, int ldv, int nv, float* Pt = nullptr, int ldt = 0) {
  // diagonal block width: the whole block lives in every thread's registers
  // and is factored redundantly by every thread (work grows as BK^3 x threads)
  constexpr int BK = 8;
  const int nv_all = nv;
  for (int K = 0; K < n; K += BK) {
    const int kb = min(BK, n - K);
    const int R0 = K + kb, rows = FACTOR ? n - R0 : 0;
    if (IDENTITY) nv = min(nv_all, R0);
    // 1. diagonal block in registers (identity-padded past kb), only in the
    //    threads that own an item (thread 0 always: it writes the block back)
    T c[BK][BK], rsv[BK];
    const bool act = threadIdx.x < max(rows + nv, 1);
    if (act) {
#pragma unroll
    for (int i = 0; i < BK; ++i)
#pragma unroll
      for (int j = 0; j <= i; ++j)
        c[i][j] = (i < kb) ? A[(K + i) * lda + K + j] : (i == j ? T(1) : T(0));
    if (FACTOR) {
#pragma unroll
      for (int j = 0; j < BK; ++j) {
        const T r = rsqrt_t(c[j][j]);
        rsv[j] = r;
        c[j][j] *= r;
#pragma unroll
        for (int i = j + 1; i < BK; ++i) c[i][j] *= r;
#pragma unroll
        for (int i = j + 1; i < BK; ++i)
#pragma unroll
          for (int l = j + 1; l <= i; ++l) c[i][l] = fma(-c[i][j], c[l][j], c[i][l]);
      }
    } else {
#pragma unroll
      for (int j = 0; j < BK; ++j) rsv[j] = T(1) / c[j][j];
    }
    // 2. forward substitution of every item against the diagonal block
    for (int it = threadIdx.x; it < rows + nv; it += blockDim.x) {
      T* base;
      int stride;
      if (it < rows) {
        base = A + (R0 + it) * lda + K;   // panel row: contiguous columns
        stride = 1;
      } else {
        base = V + K * ldv + (it - rows); // vector segment: rows of V
        stride = ldv;
      }
      T x[BK];
#pragma unroll
      for (int j = 0; j < BK; ++j) x[j] = j < kb ? base[j * stride] : T(0);
#pragma unroll
      for (int j = 0; j < BK; ++j) {
#pragma unroll
        for (int i = 0; i < j; ++i) x[j] = fma(-x[i], c[j][i], x[j]);
        x[j] *= rsv[j];
      }
#pragma unroll
      for (int j = 0; j < BK; ++j)
        if (j < kb) base[j * stride] = x[j];
      if constexpr (sizeof(T) == 4)
        if (Pt != nullptr && it < rows) {
#pragma unroll
          for (int j = 0; j < BK; ++j)
            if (j < kb) Pt[j * ldt + R0 + it] = x[j];
        }
    }
    }
    if constexpr (sizeof(T) == 4 && !FACTOR) {
      // solve-only pass: the panel is the stored factor's; copy it transposed
      if (Pt != nullptr)
        for (int e = threadIdx.x; e < (n - R0) * kb; e += blockDim.x) {
          const int r = e / kb, j = e - r * kb;
          Pt[j * ldt + R0 + r] = A[(R0 + r) * lda + K + j];
        }
    }
    __syncthreads();
    // 3. write the factored diagonal block (one thread, static register
    //    indices), then the trailing updates
    if (FACTOR && threadIdx.x == 0) {
#pragma unroll
      for (int i = 0; i < BK; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j)
          if (i < kb) A[(K + i) * lda + K + j] = c[i][j];
    }
    if (R0 < n) {
      if constexpr (sizeof(T) == 8) {
        rank_update_f64(A, lda, V, ldv, n, K, kb, R0, nv, FACTOR);
      } else {
        if (Pt != nullptr) {
          if ((ldv & 3) == 0 && (reinterpret_cast<uintptr_t>(V) & 15) == 0)
            rank_update_simt_pt<true>(A, lda, V, ldv, n, K, kb, R0, nv, FACTOR, Pt, ldt);
          else
            rank_update_simt_pt<false>(A, lda, V, ldv, n, K, kb, R0, nv, FACTOR, Pt, ldt);
        } else {
          rank_update_simt<T>(A, lda, V, ldv, n, K, kb, R0, nv, FACTOR);
        }
      }
    }
    __syncthreads();
  }
}

}  // namespace socu
