// Schur update and fill-in of one factor level for FLOAT blocks (n <= 128)
// on the tcgen05 tensor cores (tc_gemm.cuh: 3xTF32 split, FP32 accumulation
// in tensor memory).  Same tasks and results layout as update_full_body
// (nd_kernels.cuh): task u-1 < U updates target j = 2su-1 completely,
//     L_j -= F F^T + G^T G          (lower triangle; F = E[o_l+2u-2], G = E[o_l+2u-1])
// as one product D = A A^T with A = [F | G^T] (n x 2n), and task U + t-1
// forms the fill-in of node t,
//     X = E[o_{l+1}+t-1] -= F G     (F = E[o_l+2t], G = E[o_l+2t-1])
// as D = F (G^T)^T.  (socu: syrk K5/K6 and gemm K7,
// socu/block_tridiag_solver.py:282-377, socu/blas/syrk.py, socu/blas/gemm.py;
// the reference accumulates the two syrk contributions with atomics, here each
// output block has one writer.)
//
// The MMA is M = 128 rows (rows n..127 of A are zero), N = n rounded up to 16
// columns, K streamed in chunks of kTcKC columns through one shared buffer:
// stage (TF32 split, 8 rows x 4 columns per 32 threads: conflict-free) ->
// fence -> barrier -> one thread issues 3 kTcKC/8 MMAs and commits to an
// mbarrier -> everyone waits (bounded) -> next chunk.  The epilogue reads the
// accumulator from TMEM (warp w: rows 32 (w % 4).., column half w / 4) and
// subtracts it from the block in global memory.
#pragma once

#include "nd_kernels.cuh"
#include "tc_gemm.cuh"

namespace socu {

constexpr int kTcKC = 32;                                  // K columns per staged chunk
constexpr unsigned long long kTcWaitNs = 200000000ull;    // bound of one tensor-core wait (0.2 s)
constexpr int kTcMaxN = 128;

__host__ __device__ inline int tc_ncols(int n) { return ((n + 15) / 16) * 16; }
// shared memory: A hi/lo planes (128 x kTcKC) + B hi/lo planes (N x kTcKC)
__host__ __device__ inline long long smem_update_tc_bytes(int n) {
  return 2LL * 128 * kTcKC * 4 + 2LL * tc_ncols(n) * kTcKC * 4;
}
__host__ __device__ inline bool update_tc_ok(int n) { return n >= 1 && n <= kTcMaxN; }

using tc::g_tc_error;

// Stage columns [k0, k0 + KC) of a rows x K operand into hi/lo planes of a
// KC-column chunk.  val(r, k) gives the element (only called for r < rows,
// k < K); the rest is 0.  A warp writes 8 rows x 4 columns: conflict-free.
template <int KC, class Val>
__device__ __forceinline__ void tc_stage_kc(unsigned char* hi, unsigned char* lo, int rows_pad, int rows, int K,
                                            int k0, Val val) {
  constexpr int kq = KC / 4;                           // 4-column groups per chunk
  const int units = (rows_pad / 8) * kq;               // 8 x 4 units
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int u = warp; u < units; u += nw) {
    const int r = (u / kq) * 8 + (lane >> 2);
    const int kk = (u % kq) * 4 + (lane & 3);
    const int k = k0 + kk;
    const float v = (r < rows && k < K) ? val(r, k) : 0.0f;
    tc::put_split(hi, lo, r, kk, KC, v);
  }
}

template <class Val>
__device__ __forceinline__ void tc_stage(unsigned char* hi, unsigned char* lo, int rows_pad, int rows, int K,
                                         int k0, Val val) {
  tc_stage_kc<kTcKC>(hi, lo, rows_pad, rows, K, k0, val);
}

// The same staging in two halves, so that a chunk's global loads can be
// issued while the previous chunk's MMAs run: tc_load_kc reads this thread's
// elements (unit order of tc_stage_kc, at most MAXU per thread) into
// registers, tc_put_kc splits them into the planes.
template <int KC, int MAXU, class Val>
__device__ __forceinline__ void tc_load_kc(float (&v)[MAXU], int rows_pad, int rows, int K, int k0, Val val) {
  constexpr int kq = KC / 4;
  const int units = (rows_pad / 8) * kq;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < MAXU; ++j) {
    const int u = warp + j * nw;
    const int r = (u / kq) * 8 + (lane >> 2);
    const int k = k0 + (u % kq) * 4 + (lane & 3);
    v[j] = (u < units && r < rows && k < K) ? val(r, k) : 0.0f;
  }
}

template <int KC, int MAXU>
__device__ __forceinline__ void tc_put_kc(unsigned char* hi, unsigned char* lo, const float (&v)[MAXU],
                                          int rows_pad) {
  constexpr int kq = KC / 4;
  const int units = (rows_pad / 8) * kq;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < MAXU; ++j) {
    const int u = warp + j * nw;
    if (u < units) tc::put_split(hi, lo, (u / kq) * 8 + (lane >> 2), (u % kq) * 4 + (lane & 3), KC, v[j]);
  }
}
// per-thread elements of a 128 x kTcKC chunk at 256 threads
constexpr int kTcUnitsPerThread = 128 / 8 * (kTcKC / 4) / 8;

// One update task (see the file comment), all 256 threads of the CTA (the
// register staging holds kTcUnitsPerThread elements per thread at 256).  tmem: 128-column accumulator of this CTA; bar: its mbarrier,
// phase counter in *phase (the caller keeps it across tasks).
__device__ __forceinline__ void update_tc_body(const Problem<float>& p, const Level& lv, int b, int task,
                                               unsigned char* smem, uint32_t tmem, uint64_t* bar,
                                               unsigned* phase) {
  const int n = p.n, N = p.N, s = lv.s;
  const int U = N / (2 * s);
  const int nc = tc_ncols(n);
  unsigned char* a_hi = smem;
  unsigned char* a_lo = a_hi + 128 * kTcKC * 4;
  unsigned char* b_hi = a_lo + 128 * kTcKC * 4;
  unsigned char* b_lo = b_hi + nc * kTcKC * 4;
  const bool target = task < U;
  const float *F, *G;
  float* Out;
  int K;
  if (target) {
    const int u = task + 1, j = 2 * s * u - 1;
    F = p.Eb(b, lv.oc + 2 * (u - 1));
    G = j + s < N ? p.Eb(b, lv.oc + 2 * u - 1) : nullptr;
    Out = p.Lb(b, j);
    K = G ? 2 * n : n;
  } else {
    const int t = task - U + 1, i = s - 1 + 2 * s * t;
    if (i + s >= N) return;
    F = p.Eb(b, lv.oc + 2 * t);
    G = p.Eb(b, lv.oc + 2 * t - 1);
    Out = p.Eb(b, lv.on + t - 1);
    K = n;
  }
  bool ok;
  // A = [F | G^T] (target) or F (fill-in): A(r, k) = k < n ? F[r][k] : G[k-n][r];
  // fill-in: B(c, k) = G[k][c]; targets use B = A (its first nc rows).  The
  // next chunk's elements are loaded into registers while this chunk's MMAs run.
  // With 8 warps and 8 four-column groups per chunk, a thread's elements
  // (tc_put_kc's unit order) are one column k0 + kk of the chunk at rows
  // lane / 4 + 8 j: a strided run in F (rows) or G (columns).
  float ra[kTcUnitsPerThread], rb[kTcUnitsPerThread];
  const int kk = (threadIdx.x >> 5) * 4 + (threadIdx.x & 3), r0 = (threadIdx.x & 31) >> 2;
  auto load_chunk = [&](int k0) {
    const int k = k0 + kk;
    const float* a = nullptr;
    long long sa = 0;
    if (k < n) {
      a = F + (long long)r0 * n + k;
      sa = 8LL * n;
    } else if (k < K) {
      a = G + (long long)(k - n) * n + r0;
      sa = 8;
    }
#pragma unroll
    for (int j = 0; j < kTcUnitsPerThread; ++j) ra[j] = (a != nullptr && r0 + 8 * j < n) ? a[j * sa] : 0.0f;
    if (!target) {
      const float* g = k < K ? G + (long long)k * n + r0 : nullptr;
#pragma unroll
      for (int j = 0; j < kTcUnitsPerThread; ++j) rb[j] = (g != nullptr && r0 + 8 * j < n) ? g[8 * j] : 0.0f;
    }
  };
  load_chunk(0);
  for (int k0 = 0; k0 < K; k0 += kTcKC) {
    tc_put_kc<kTcKC, kTcUnitsPerThread>(a_hi, a_lo, ra, 128);
    if (!target) tc_put_kc<kTcKC, kTcUnitsPerThread>(b_hi, b_lo, rb, nc);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (threadIdx.x == 0) {
      const uint32_t ah = tc::saddr(a_hi), al = tc::saddr(a_lo);
      const uint32_t bh = target ? ah : tc::saddr(b_hi), bl = target ? al : tc::saddr(b_lo);
      tc::gemm_3xtf32(tmem, ah, al, bh, bl, nc, kTcKC, k0 > 0 ? 1u : 0u);
      tc::commit(bar);
    }
    if (k0 + kTcKC < K) load_chunk(k0 + kTcKC);
    // every thread waits for the chunk's MMAs before the buffer is restaged;
    // the vote keeps the CTA's control flow uniform if a wait runs out
    const bool done = tc::mbar_wait(bar, *phase & 1u, kTcWaitNs);
    ok = __syncthreads_and(done) != 0;
    tc::fence_after_sync();
    if (!ok) {
      // second bound for MMAs still in flight before the caller frees TMEM
      tc::mbar_wait(bar, *phase & 1u, kTcWaitNs);
      if (threadIdx.x == 0) atomicExch(&g_tc_error, 1);
      *phase += 1;
      return;
    }
    *phase += 1;
  }
  // epilogue: Out -= D (lower triangle for targets)
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3, halves = blockDim.x / 128, h = warp >> 2;
  const int r = 32 * q + lane;
  const int span = ((nc / 8 + halves - 1) / halves) * 8;
  const int c_begin = h * span, c_end = min(nc, c_begin + span);
  for (int c0 = c_begin; c0 < c_end; c0 += 8) {
    if (target && c0 > 32 * q + 31) break;   // warp-uniform: every column above this warp's rows
    if (32 * q >= n) break;
    float v[8];
    tc::tmem_ld8(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
    tc::tmem_wait_ld();
    if (r < n) {
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int c = c0 + i;
        if (c < n && (!target || c <= r)) Out[(long long)r * n + c] -= v[i];
      }
    }
  }
}

// One CTA per update task of one level (grid = B x update_blocks).
__global__ void __launch_bounds__(256, 3) k_update_tc(Problem<float> p, Level lv) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  const int per_b = update_blocks(p.N, lv);
  const int b = blockIdx.x / per_b;
  const int task = blockIdx.x - b * per_b;
  if (!p.active(b)) return;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tc::tmem_alloc(&tbase, 128);
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  pdl_wait();
  pdl_trigger();
  unsigned phase = 0;
  update_tc_body(p, lv, b, task, smem_raw, tbase, &bar, &phase);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tbase, 128);
}

// ---------------------------------------------------------------------------
// Level node of a FLOAT factor (n <= 128) with its products on the tcgen05
// tensor cores.  The factor part is the inverse-first node's (node_gemm_body:
// blocked Cholesky of L_i against the identity, C W = I, W = C^{-1}); the
// three products that follow -- F = R W^T (right slot), G = W Lf (left slot),
// y = W y (factor_and_solve) -- share the operand W and run as MMA groups of
//     D (n x NB) = W * Bm^T,   Bm rows: the n rows of R, the n columns of Lf,
//                              the m columns of y  (NB = nr + nl + m)
// in column groups of at most 256, so D's columns hold F^T, G and W y.
// socu: trsm_rltn / trsm_llnn (K3/K4) and the fused forward step,
// socu/block_tridiag_solver.py:219-279, :108-110, done here as products with
// the explicit inverse.  M = 64 rows for n <= 64 (row r of D in TMEM lane
// 32 (r / 16) + r % 16), else M = 128 (row r in lane r); rows n..M-1 of W are
// zero.  K is staged in chunks of 16 columns.  Shared memory: W, then one
// region that holds the factor's input block S1 and, once C has been written
// out, the A planes, then the B planes of one column group (52 KB at n = 64:
// four CTAs per SM, as for the SIMT node).
// ---------------------------------------------------------------------------
constexpr int kTcNodeMaxN = 128;
constexpr int kTcNodeGroup = 256;   // MMA columns per group (TMEM columns allocated)
constexpr int kTcNodeKC = 16;
__host__ __device__ inline int tc_node_M(int n) { return n <= 64 ? 64 : 128; }
__host__ __device__ inline uint32_t tmem_cols_for(int cols) {
  return cols <= 32 ? 32u : (cols <= 64 ? 64u : (cols <= 128 ? 128u : 256u));
}
__host__ __device__ inline long long round128(long long b) { return ((b + 127) / 128) * 128; }
__host__ __device__ inline long long smem_node_tc_w(int n) { return round128((long long)n * gemm_ld(n, 4) * 4); }
__host__ __device__ inline long long smem_node_tc_s1(int n) {
  const long long s1 = round128((long long)n * gemm_ld(n, 4) * 4), a = 2LL * tc_node_M(n) * kTcNodeKC * 4;
  return s1 > a ? s1 : a;
}
__host__ __device__ inline long long smem_node_tc_bytes(int n, int m) {
  const int nb = tc_ncols(2 * n + m), grp = nb < kTcNodeGroup ? nb : kTcNodeGroup;
  return smem_node_tc_w(n) + smem_node_tc_s1(n) + 2LL * grp * kTcNodeKC * 4;
}
__host__ __device__ inline bool node_tc_ok(int n, int m) { return n >= 1 && n <= kTcNodeMaxN && m >= 0; }

template <bool WITH_Y, bool INV, int KC>
__device__ __forceinline__ void node_tc_body(const Problem<float>& p, const Level& lv, int b, int t,
                                             unsigned char* smem, uint32_t tmem, uint64_t* bar, unsigned* phase) {
  const int n = p.n, s = lv.s, i = s - 1 + 2 * s * t;
  const bool right = i + s < p.N, left = t >= 1;
  const int ld = gemm_ld(n, 4);
  const int M = tc_node_M(n);
  float* W = reinterpret_cast<float*>(smem);
  unsigned char* region1 = smem + smem_node_tc_w(n);
  float* S1 = reinterpret_cast<float*>(region1);           // factor input / C ...
  unsigned char* a_hi = region1;                          // ... then the A planes
  unsigned char* a_lo = a_hi + M * KC * 4;
  unsigned char* b_hi = region1 + smem_node_tc_s1(n);
  const int nr = right ? n : 0, nl = left ? n : 0, ny = WITH_Y ? p.m : 0;
  const int NB = nr + nl + ny;
  float* Li = p.Lb(b, i);
  float* R = right ? p.Eb(b, lv.oc + 2 * t) : nullptr;
  float* Lf = left ? p.Eb(b, lv.oc + 2 * t - 1) : nullptr;
  float* yi = WITH_Y ? p.Xb(b, i) : nullptr;
  const int m = p.m;

  // factor: lower(S1) = C, W = C^{-1}
  async_load(S1, ld, Li, n, n, n);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e - r * n;
    W[r * ld + c] = r == c ? 1.0f : 0.0f;
  }
  cp_async_wait_all();
  __syncthreads();
  cta_chol_solve<float, true, true>(S1, ld, n, W, ld, n);
  check_factor(p, b, i, S1, ld);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e - r * n;
    Li[e] = c <= r ? S1[r * ld + c] : (INV ? W[c * ld + r] : 0.0f);
  }
  __syncthreads();   // S1's space becomes the A planes
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = warp & 3, parts = blockDim.x / 128, h = warp >> 2;
  // rows of D held by this warp's sub-partition: M = 64 -> 16 q .. 16 q + 15
  // (lanes 0-15), M = 128 -> 32 q .. 32 q + 31
  const int rows_q = M == 64 ? 16 : 32;
  const int r = rows_q * q + lane;
  const bool row_ok = lane < rows_q && r < n;
  for (int g0 = 0; g0 < NB; g0 += kTcNodeGroup) {
    const int NBg = min_i(kTcNodeGroup, NB - g0), NBgp = tc_ncols(NBg);
    unsigned char* b_lo = b_hi + NBgp * KC * 4;
    for (int k0 = 0; k0 < n; k0 += KC) {
      tc_stage_kc<KC>(a_hi, a_lo, M, n, n, k0, [&](int rr, int k) { return W[rr * ld + k]; });
      tc_stage_kc<KC>(b_hi, b_lo, NBgp, NBg, n, k0, [&](int cl, int k) {
        const int c = g0 + cl;
        if (c < nr) return R[(long long)c * n + k];
        if (c < nr + nl) return Lf[(long long)k * n + (c - nr)];
        return yi[(long long)k * m + (c - nr - nl)];
      });
      tc::fence_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      tc::fence_after_sync();
      if (threadIdx.x == 0) {
        tc::gemm_3xtf32(tmem, tc::saddr(a_hi), tc::saddr(a_lo), tc::saddr(b_hi), tc::saddr(b_lo), NBgp, KC,
                        k0 > 0 ? 1u : 0u, M);
        tc::commit(bar);
      }
      const bool done = tc::mbar_wait(bar, *phase & 1u, kTcWaitNs);
      const bool ok = __syncthreads_and(done) != 0;
      tc::fence_after_sync();
      if (!ok) {
        tc::mbar_wait(bar, *phase & 1u, kTcWaitNs);
        if (threadIdx.x == 0) atomicExch(&g_tc_error, 1);
        *phase += 1;
        return;
      }
      *phase += 1;
    }
    // epilogue of this group: columns split between the blockDim / 128 warps of a quadrant
    const int span = ((NBgp / 8 + parts - 1) / parts) * 8;
    const int c_begin = h * span, c_end = min_i(NBg, c_begin + span);
    if (rows_q * q < n) {
      for (int c0 = c_begin; c0 < c_end; c0 += 8) {
        float v[8];
        tc::tmem_ld8(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)c0, v);
        tc::tmem_wait_ld();
        if (row_ok) {
#pragma unroll
          for (int e = 0; e < 8; ++e) {
            const int c = g0 + c0 + e;
            if (c0 + e >= NBg) break;
            if (c < nr) R[(long long)c * n + r] = v[e];                    // F[c][r] = D[r][c]
            else if (c < nr + nl) Lf[(long long)r * n + (c - nr)] = v[e];  // G[r][c - nr]
            else yi[(long long)r * m + (c - nr - nl)] = v[e];
          }
        }
      }
    }
    // the next group overwrites the accumulator: every TMEM read of this one first
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
  }
}

template <bool WITH_Y, bool INV>
__global__ void __launch_bounds__(256, 1) k_node_tc(Problem<float> p, Level lv) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t bar;
  __shared__ uint32_t tbase;
  const int b = blockIdx.x / lv.d;
  const int t = blockIdx.x - b * lv.d;
  if (!p.active(b)) return;
  const int i = lv.s - 1 + 2 * lv.s * t;
  const int nb = (i + lv.s < p.N ? p.n : 0) + (t >= 1 ? p.n : 0) + (WITH_Y ? p.m : 0);
  const uint32_t ncols = tmem_cols_for(tc_ncols(nb < kTcNodeGroup ? nb : kTcNodeGroup));
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tc::tmem_alloc(&tbase, ncols);
  if (threadIdx.x == 0) tc::mbar_init(&bar, 1);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  pdl_wait();
  pdl_trigger();
  unsigned phase = 0;
  node_tc_body<WITH_Y, INV, kTcNodeKC>(p, lv, b, t, smem_raw, tbase, &bar, &phase);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tbase, ncols);
}

}  // namespace socu
