// Per-level kernels of the nested-dissection block-tridiagonal Cholesky.
//
// One factor level l (stride s) is two launches, all deterministic (no
// floating-point atomics, every output block has exactly one writer):
//   k_node    one CTA per level node i: C_i = chol(L_i) in place
//             (socu: potrf K2, block_tridiag_solver.py:197-216) fused with
//             C_i V = RHS, blocked by 8 columns (see cta_chol_solve).  The
//             vectors of node i are
//               rows of the right slot     -> F = E[o_l+i/s] C_i^{-T}   (K3 trsm_rltn, :219-248)
//               columns of the left slot   -> G = C_i^{-1} E[o_l+(i-s)/s] (K4 trsm_llnn, :251-279)
//               columns of y_i (factor_and_solve) -> y_i <- C_i^{-1} y_i (:108-110)
//   k_update  one CTA per 32x32 output tile:
//             target j = 2 s u - 1 (owner computes; the reference uses
//             atomics here, K5/K6 :282-342)
//                 L_j -= F_{j-s} F_{j-s}^T + G_{j+s}^T G_{j+s}
//             fill-in for nodes with both neighbours (K7, :345-377)
//                 E[o_{l+1} + t - 1] -= F_t G_t
// Substitution sweeps (K9-K16, :425-736), reading only lower(L_i):
//   k_fwd          levels ascending, one launch per level: each vector pulls
//                  the previous level's coupling updates
//                  y_j -= F_{j-s/2} y_{j-s/2} + G_{j+s/2}^T y_{j+s/2} and the
//                  level's nodes then solve y_i <- C_i^{-1} y_i
//   k_bwd          levels descending: x_i -= F_i^T x_{i+s} + G_i x_{i-s};
//                  x_i <- C_i^{-T} x_i
#pragma once

#include "nd_device.cuh"
#include "tma.cuh"

namespace socu {

constexpr int kTile = 32;     // output tile / streamed chunk width
constexpr int kMC = 32;       // RHS columns handled per pass in the sweeps

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
__host__ __device__ inline int min_i(int a, int b) { return a < b ? a : b; }

// shared-memory sizes (elements) ------------------------------------------------
__host__ __device__ inline int gemm_ld(int n, int es) { return es == 8 ? ((n + 15) / 16) * 16 + 4 : n + 1; }
// vectors solved per pass of k_node (items beyond the block size loop)
// (n > 64: 64 for float -- two CTAs per SM, measured faster than one pass of
// all vectors at one CTA per SM -- and 80 for double, the most that fit)
__host__ __device__ inline int node_chunk(int n, int es) { return n <= 64 ? 232 : (es == 4 ? 64 : 80); }
// float: vector rows on 16 bytes (4-wide operand loads in the rank updates),
// then the transposed panel Pt (8 x node_ldt(n)) of cta_chol_solve
__host__ __device__ inline int node_vld(int vc, int es) { return es == 8 ? gemm_ld(vc, es) : ((vc + 3) & ~3) + 4; }
__host__ __device__ inline int node_ldt(int n) { return ((n + 3) & ~3) + 4; }
__host__ __device__ inline long long node_v_off(int n, int es) {
  const long long a = (long long)n * gemm_ld(n, es);
  return es == 4 ? ((a + 3) & ~3LL) : a;
}
__host__ __device__ inline long long smem_node_elems(int n, int es) {
  const long long v = node_v_off(n, es) + (long long)n * node_vld(node_chunk(n, es), es);
  return es == 4 ? v + 8LL * node_ldt(n) : v;
}
__host__ __device__ inline int update_ld(int k, int es) { return gemm_ld(k, es); }
// blocked Schur update (n > 64) with tile x tile output tiles
__host__ __device__ inline long long smem_update_elems(int n, int es, int tile = kTile) {
  const long long a = 2LL * tile * update_ld(2 * n, es);
  const long long f = (long long)tile * update_ld(n, es) + (long long)n * update_ld(tile, es);
  return a > f ? a : f;
}
// streamed (non-resident) sweeps: Y, Z1, Z2 (n x sweep_ldy) and the chunk buffer
// Cc (n x sweep_ldc >= kTile x (n + 1) for the triangular panels), dv (kTile)
__host__ __device__ inline int sweep_ldy(int mc) { return mc + 4; }
constexpr int kSweepLdc = kTile + 4;   // 4 (mod 16) doubles: conflict-free DMMA fragments

// cp.async groups: close the group of copies issued so far / wait until at
// most one group is still in flight
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
// (two chunk buffers: the next chunk's copies overlap this chunk's product)
__host__ __device__ inline long long smem_sweep_elems(int n, int m) {
  const int mc = min_i(m, kMC);
  const long long cc = 2LL * n * kSweepLdc > (long long)kTile * (n + 1) ? 2LL * n * kSweepLdc
                                                                        : (long long)kTile * (n + 1);
  return 3LL * n * sweep_ldy(mc) + cc + kTile;
}

// ---------------------------------------------------------------------------
// k_node: 256 threads per level node i.
//   C_i = chol(L_i)  (potrf, K2)  fused with  C_i V = RHS for the node's
//   vectors: rows of the right slot (-> F), columns of the left slot (-> G)
//   and, with WITH_Y, the columns of y_i, in passes of node_chunk(n, es) vectors
//   (the first pass factors, later passes reuse the factor).
// ---------------------------------------------------------------------------
// INV: also solve C_i W = I and keep W = C_i^{-1} in the strict upper
// triangle of L_i (transposed: L_i[c][r] = W[r][c], r > c), for the sweeps
// that multiply by the inverse (see k_fwd / k_bwd with INV).
// Body of one node (instance b, level node t) with vc vectors per pass; the
// shared buffer holds n*gemm_ld(n) + n*gemm_ld(vc) elements.
template <typename T, bool WITH_Y, bool INV>
__device__ __forceinline__ void node_body(const Problem<T>& p, const Level& lv, int b, int t,
                                          unsigned char* smem_raw, int vc) {
  constexpr int es = sizeof(T);
  const int n = p.n, s = lv.s, i = s - 1 + 2 * s * t;
  const bool right = i + s < p.N, left = t >= 1;
  const int nr = right ? n : 0, nl = left ? n : 0, ny = WITH_Y ? p.m : 0, ni = INV ? n : 0;
  const int NV = nr + nl + ny + ni;
  const int lda = gemm_ld(n, es), ldv = node_vld(vc, es);
  T* A = reinterpret_cast<T*>(smem_raw);
  T* V = A + node_v_off(n, es);
  float* Pt = es == 4 ? reinterpret_cast<float*>(V + (long long)n * ldv) : nullptr;

  T* Li = p.Lb(b, i);
  T* R = right ? p.Eb(b, lv.oc + 2 * t) : nullptr;
  T* Lf = left ? p.Eb(b, lv.oc + 2 * t - 1) : nullptr;
  T* yi = WITH_Y ? p.Xb(b, i) : nullptr;

  // chunk [v0, v1) of the node's vectors: R rows, Lf columns, y columns,
  // then (INV) the columns of the identity
  auto chunk_io = [&](int v0, bool load) {
    const int v1 = min_i(NV, v0 + vc);
    const int rA = v0, rB = min_i(v1, nr);
    const int lS = max(v0, nr), lA = lS - nr, lB = min_i(v1, nr + nl) - nr;
    const int yS = max(v0, nr + nl), yA = yS - nr - nl, yB = min_i(v1, nr + nl + ny) - nr - nl;
    const int iS = max(v0, nr + nl + ny), iA = iS - nr - nl - ny, iB = v1 - nr - nl - ny;
    if (load) {
      if (rB > rA) async_load_t(V, ldv, R + (long long)rA * n, rB - rA, n, n);
      if (lB > lA) async_load(V + (lS - v0), ldv, Lf + lA, n, lB - lA, n);
      if (yB > yA) async_load(V + (yS - v0), ldv, yi + yA, n, yB - yA, p.m);
      if (INV && iB > iA)
        for (int e = threadIdx.x; e < n * (iB - iA); e += blockDim.x) {
          const int k = e / (iB - iA), j = e - k * (iB - iA);
          V[k * ldv + (iS - v0) + j] = k == iA + j ? T(1) : T(0);
        }
    } else {
      if (rB > rA) store_block_t(R + (long long)rA * n, n, V, ldv, rB - rA, n);
      if (lB > lA) store_block(Lf + lA, n, V + (lS - v0), ldv, n, lB - lA);
      if (yB > yA) store_block(yi + yA, p.m, V + (yS - v0), ldv, n, yB - yA);
      if (INV && iB > iA)   // W[r][c] (r > c) -> L_i[c][r]
        for (int e = threadIdx.x; e < n * (iB - iA); e += blockDim.x) {
          const int c = iA + e / n, r = e - (e / n) * n;
          if (r > c) Li[(long long)c * n + r] = V[r * ldv + (iS - v0) + (c - iA)];
        }
    }
  };

  async_load(A, lda, Li, n, n, n);
  if (NV > 0) chunk_io(0, true);
  cp_async_wait_all();
  __syncthreads();
  cta_chol_solve<T, true>(A, lda, n, V, ldv, min_i(NV, vc), Pt, node_ldt(n));
  check_factor(p, b, i, A, lda);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e - r * n;
    if (c <= r) Li[e] = A[r * lda + c];
    else if (!INV) Li[e] = T(0);
  }
  if (NV > 0) chunk_io(0, false);
  for (int v0 = vc; v0 < NV; v0 += vc) {
    __syncthreads();
    chunk_io(v0, true);
    cp_async_wait_all();
    __syncthreads();
    cta_chol_solve<T, false>(A, lda, n, V, ldv, min_i(NV - v0, vc), Pt, node_ldt(n));
    chunk_io(v0, false);
  }
}

// ---------------------------------------------------------------------------
// Float blocked Cholesky against the identity (cta_chol_solve<float, true,
// true>: lower(A) = C, V = C^{-1}) with the trailing matrices held in
// registers.  Each thread owns one fixed 4x4 tile for the whole
// factorisation -- a lower tile of A right of the first panel, or a strictly
// lower tile of V below the first rows (the only tiles a rank update ever
// touches) -- instead of loading and storing accumulators around each
// 8-column step's rank-8 update; a tile goes back to shared memory when it
// enters the next step's panel (A: its columns, V: its rows).  The item
// solves also write the solved panel transposed (Pt[k][row]) and the solved
// rows of V (Vt[k][col]), so both operands of the update are 16-byte loads.
// Same operations in the same order as cta_chol_solve: identical results.
// Returns false (nothing done) when the tiles outnumber the threads.
// ---------------------------------------------------------------------------
__host__ __device__ inline int reg_chain_ldt(int n) { return ((n + 3) / 4) * 4 + 4; }
// tiles the rank updates touch: A (row block >= column block >= 2), V (row block > column block, row block >= 2)
__host__ __device__ inline int reg_chain_tiles_a(int n) { const int b = (n + 3) / 4; return b < 3 ? 0 : (b - 2) * (b - 1) / 2; }
__host__ __device__ inline int reg_chain_tiles_v(int n) { const int b = (n + 3) / 4; return b < 3 ? 0 : (b - 1) * b / 2 - 1; }
__host__ __device__ inline bool reg_chain_ok(int n, int threads) {
  return n <= 64 && reg_chain_tiles_a(n) + reg_chain_tiles_v(n) <= threads;
}

// WT (optional, n x reg_chain_ldt(n), zero on entry): receives W^T, WT[c][r] = V[r][c],
// from the item solves (every final entry of V comes out of one).
__device__ bool cta_chol_inv_regs(float* A, int lda, int n, float* V, int ldv, float* Pt, float* Vt,
                                  float* WT = nullptr) {
  constexpr int BK = 8;
  const int na = reg_chain_tiles_a(n), total = na + reg_chain_tiles_v(n);
  if (total > (int)blockDim.x) return false;
  const int ldt = reg_chain_ldt(n);
  // this thread's tile
  const int id = threadIdx.x;
  const bool own = id < total, isA = id < na;
  int r0 = 0, c0 = 0;
  if (own) {
    if (isA) {
      int a = 0;
      while ((a + 1) * (a + 2) / 2 <= id) ++a;
      r0 = 4 * (2 + a);
      c0 = 4 * (2 + id - a * (a + 1) / 2);
    } else {
      const int v = id - na;
      int rb = 2;
      while ((rb + 1) * rb / 2 - 1 <= v) ++rb;   // tiles before row block rb + 1
      r0 = 4 * rb;
      c0 = 4 * (v - ((rb - 1) * rb / 2 - 1));
    }
  }
  float acc[4][4];
  {
    const float* src = isA ? A : V;
    const int ld = isA ? lda : ldv;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int r = r0 + i, c = c0 + j;
        acc[i][j] = (own && r < n && c < n) ? src[r * ld + c] : 0.0f;
      }
  }
  for (int K = 0; K < n; K += BK) {
    const int kb = min(BK, n - K);
    const int R0 = K + kb, rows = n - R0;
    const int nv = min(n, R0);
    // 1.-2. diagonal block in registers and item solves (as cta_chol_solve),
    //       the solved values also into Pt / Vt
    float c[BK][BK], rsv[BK];
    const bool act = threadIdx.x < max(rows + nv, 1);
    if (act) {
#pragma unroll
      for (int i = 0; i < BK; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) c[i][j] = (i < kb) ? A[(K + i) * lda + K + j] : (i == j ? 1.0f : 0.0f);
#pragma unroll
      for (int j = 0; j < BK; ++j) {
        const float r = rsqrt_t(c[j][j]);
        rsv[j] = r;
        c[j][j] *= r;
#pragma unroll
        for (int i = j + 1; i < BK; ++i) c[i][j] *= r;
#pragma unroll
        for (int i = j + 1; i < BK; ++i)
#pragma unroll
          for (int l = j + 1; l <= i; ++l) c[i][l] = fma(-c[i][j], c[l][j], c[i][l]);
      }
      for (int it = threadIdx.x; it < rows + nv; it += blockDim.x) {
        float* base;
        int stride;
        float* tb;
        if (it < rows) {
          base = A + (R0 + it) * lda + K;
          stride = 1;
          tb = Pt + R0 + it;
        } else {
          base = V + K * ldv + (it - rows);
          stride = ldv;
          tb = Vt + (it - rows);
        }
        float x[BK];
        if (kb == BK) {   // full step: straight-line loads, so they all issue before the substitution
#pragma unroll
          for (int j = 0; j < BK; ++j) x[j] = base[j * stride];
        } else {
#pragma unroll
          for (int j = 0; j < BK; ++j) x[j] = j < kb ? base[j * stride] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < BK; ++j) {
#pragma unroll
          for (int i = 0; i < j; ++i) x[j] = fma(-x[i], c[j][i], x[j]);
          x[j] *= rsv[j];
        }
        if (kb == BK) {
#pragma unroll
          for (int j = 0; j < BK; ++j) {
            base[j * stride] = x[j];
            tb[j * ldt] = x[j];
          }
        } else {
#pragma unroll
          for (int j = 0; j < BK; ++j)
            if (j < kb) {
              base[j * stride] = x[j];
              tb[j * ldt] = x[j];
            }
        }
        if (WT != nullptr && it >= rows) {   // rows K..K+kb of column it - rows: W^T row segment
          float* w = WT + (it - rows) * ldt + K;
          if (kb == BK) {
            reinterpret_cast<float4*>(w)[0] = make_float4(x[0], x[1], x[2], x[3]);
            reinterpret_cast<float4*>(w)[1] = make_float4(x[4], x[5], x[6], x[7]);
          } else {
#pragma unroll
            for (int j = 0; j < BK; ++j)
              if (j < kb) w[j] = x[j];
          }
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
#pragma unroll
      for (int i = 0; i < BK; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j)
          if (i < kb) A[(K + i) * lda + K + j] = c[i][j];
    }
    if (own && R0 < n) {
      // 3. rank-kb update: A tiles right of the panel (A22 -= P P^T), V tiles
      //    below it in the columns already reached (V2 -= P V1)
      const bool active = isA ? c0 >= R0 : (r0 >= R0 && c0 < R0);
      if (active) {   // R0 < n: a full 8-column step
        const float* bsrc = isA ? Pt : Vt;
        float4 a4[BK], b4[BK];
#pragma unroll
        for (int k = 0; k < BK; ++k) {
          a4[k] = *reinterpret_cast<const float4*>(Pt + k * ldt + r0);
          b4[k] = *reinterpret_cast<const float4*>(bsrc + k * ldt + c0);
        }
#pragma unroll
        for (int k = 0; k < BK; ++k) {
          const float av[4] = {a4[k].x, a4[k].y, a4[k].z, a4[k].w}, bv[4] = {b4[k].x, b4[k].y, b4[k].z, b4[k].w};
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) acc[i][j] = fma(-av[i], bv[j], acc[i][j]);
        }
      }
      // 4. a tile entering the next step's panel goes back to shared memory
      const int N1 = R0 + BK;
      const bool flush = isA ? (c0 >= R0 && c0 < N1) : (r0 >= R0 && r0 < N1);
      if (flush) {
        float* dst = isA ? A : V;
        const int ld = isA ? lda : ldv;
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int r = r0 + i, cc = c0 + j;
            if (r < n && cc < n && cc <= r) dst[r * ld + cc] = acc[i][j];
          }
      }
    }
    __syncthreads();
  }
  return true;
}

// Products of the inverse-first float node from W^T (WT[k][r] = W[r][k], W
// lower triangular):  F^T = W R^T (R row-major in S1: B(k, c) = R[c][k]),
// G = W Lf (S2), y = W y (Y), as one set of warp tasks of 8 rows x 64
// columns (lane: columns c and c + 32).  K stops at the tile's last row;
// the W^T rows are 16-byte broadcast loads, the B elements conflict-free
// (odd ld for the transposed R, consecutive columns otherwise).  Same
// products in the same order as the separate cta_gemm calls: identical
// results.  Heavy and light row tiles alternate between column groups.
template <class BVal, class Out>
__device__ __forceinline__ void wt_tile(int n, int r0, int cb, int ncols, const float* WT, int ldt, BVal bval,
                                        Out out) {
  const int lane = threadIdx.x & 31;
  const int kend = min_i(n, r0 + 8);
  const int c_a = cb + lane, c_b = cb + lane + 32;
  const bool va = c_a < ncols, vb = c_b < ncols;
  float acc[8][2];
#pragma unroll
  for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0f;
#pragma unroll 4
  for (int k = 0; k < kend; ++k) {
    const float4 w0 = *reinterpret_cast<const float4*>(WT + k * ldt + r0);
    const float4 w1 = *reinterpret_cast<const float4*>(WT + k * ldt + r0 + 4);
    const float wv[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
    const float b0 = va ? bval(k, c_a) : 0.0f, b1 = vb ? bval(k, c_b) : 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      acc[i][0] = fma(wv[i], b0, acc[i][0]);
      acc[i][1] = fma(wv[i], b1, acc[i][1]);
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    if (r0 + i >= n) break;
    if (va) out(r0 + i, c_a, acc[i][0]);
    if (vb) out(r0 + i, c_b, acc[i][1]);
  }
}

template <bool WITH_Y>
__device__ __forceinline__ void node_products_wt(int n, const float* WT, int ldt, const float* S1, const float* S2,
                                                 int ld, const float* Y, int ldy, int mc, float* R, float* Lf,
                                                 float* yi, int m, int c0y, bool right, bool left) {
  const int warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int rt = (n + 7) / 8, cg = (n + 63) / 64;
  const int gR = right ? cg : 0, gL = left ? cg : 0, gY = WITH_Y && mc > 0 ? 1 : 0;
  const int tasks = rt * (gR + gL + gY);
  for (int task = warp; task < tasks; task += nw) {
    const int g = task / rt, q = task - g * rt;
    const int r0 = 8 * ((g & 1) ? rt - 1 - q : q);
    if (g < gR) {
      wt_tile(n, r0, 64 * g, n, WT, ldt, [&](int k, int c) { return S1[c * ld + k]; },
              [&](int r, int c, float v) { R[(long long)c * n + r] = v; });   // F[c][r] = (F^T)[r][c]
    } else if (g < gR + gL) {
      wt_tile(n, r0, 64 * (g - gR), n, WT, ldt, [&](int k, int c) { return S2[k * ld + c]; },
              [&](int r, int c, float v) { Lf[(long long)r * n + c] = v; });
    } else {
      wt_tile(n, r0, 0, mc, WT, ldt, [&](int k, int c) { return Y[k * ldy + c]; },
              [&](int r, int c, float v) { yi[(long long)r * m + c0y + c] = v; });
    }
  }
}

// ---------------------------------------------------------------------------
// Inverse-first node (n <= kNodeGemmMaxN): factor L_i against the identity
// only, C W = I, so W = C^{-1} comes out of the blocked solve, then every
// other vector set is one dense GEMM with W (tensor cores for double):
//     F = R W^T      (rows of the right slot, R loaded row-major)
//     G = W Lf       (left slot)
//     y = W y        (factor_and_solve)
// R, Lf and the first y chunk are loaded together once the factor is done
// and the three GEMMs run back to back without barriers in between; results
// go from the accumulators straight to global memory.  Shared layout:
// S1 (n x ld: A/C, then R), W (n x ld), S2 (n x ld: Lf), Y (n x ldy).
// INV keeps W^T in the strict upper triangle of L_i.
// ---------------------------------------------------------------------------
constexpr int kNodeGemmMaxN = 64;
__host__ __device__ inline int node_gemm_ldy(int m) { return m > 0 ? even_ld(min_i(m, kMC)) : 0; }
// S1, W, S2 (n x ld), Y (n x ldy); float: then Pt, Vt (8 x reg_chain_ldt(n) each,
// on 16 bytes) of the register-resident chain, and with WT_PRODUCTS the
// W^T buffer (n x reg_chain_ldt(n))
// reg: the launch's CTAs are large enough for the register-resident chain
// (reg_chain_ok), which needs Pt / Vt; wt implies reg.
__host__ __device__ inline long long smem_node_gemm_elems(int n, int m, int es, bool wt = false, bool reg = true) {
  const long long base = 3LL * n * gemm_ld(n, es) + (long long)n * node_gemm_ldy(m);
  if (es != 4 || !(reg || wt)) return base;
  // WT_PRODUCTS also keeps a buffer for R, loaded during the chain
  return base + 4 + (16LL + (wt ? n : 0)) * reg_chain_ldt(n) + (wt ? (long long)n * gemm_ld(n, es) : 0);
}

// WT_PRODUCTS (float, with REG_CHAIN): the chain also writes W^T and the
// three products run as node_products_wt (levels of at most one wave of CTAs:
// the W^T buffer costs occupancy).
template <typename T, bool WITH_Y, bool INV, bool REG_CHAIN = true, bool WT_PRODUCTS = false>
__device__ __forceinline__ void node_gemm_body(const Problem<T>& p, const Level& lv, int b, int t,
                                               unsigned char* smem_raw) {
  constexpr int es = sizeof(T);
  const int n = p.n, s = lv.s, i = s - 1 + 2 * s * t;
  const bool right = i + s < p.N, left = t >= 1;
  const int ld = gemm_ld(n, es);
  const int ldy = node_gemm_ldy(WITH_Y ? p.m : 0);
  T* S1 = reinterpret_cast<T*>(smem_raw);
  T* W = S1 + n * ld;
  T* S2 = W + n * ld;
  T* Y = S2 + n * ld;
  T* Li = p.Lb(b, i);
  // float: operand rows of the register-resident chain, after Y on 16 bytes
  float* Pt = reinterpret_cast<float*>(smem_raw + ((((long long)(3 * n * ld + n * ldy)) * sizeof(T) + 15) & ~15LL));
  float* Vt = Pt + 8 * reg_chain_ldt(n);
  float* WT = Vt + 8 * reg_chain_ldt(n);
  float* Rb = WT + n * reg_chain_ldt(n);   // WT_PRODUCTS: R, loaded during the chain
  T* R = right ? p.Eb(b, lv.oc + 2 * t) : nullptr;
  T* Lf = left ? p.Eb(b, lv.oc + 2 * t - 1) : nullptr;
  T* yi = WITH_Y ? p.Xb(b, i) : nullptr;
  bool wt_ok = false;
  if constexpr (sizeof(T) == 4 && REG_CHAIN && WT_PRODUCTS) wt_ok = reg_chain_ok(n, blockDim.x) && (!WITH_Y || p.m <= kMC);

  async_load(S1, ld, Li, n, n, n);
  if (wt_ok) cp_async_commit();                // the chain waits for L_i only
  if (left) async_load(S2, ld, Lf, n, n, n);   // prefetch: S2 is untouched by the factor
  if constexpr (sizeof(T) == 4 && WT_PRODUCTS) {
    if (wt_ok) {
      if (right) async_load(Rb, ld, R, n, n, n);
      if (WITH_Y) async_load(Y, ldy, yi, n, p.m, p.m);
      cp_async_commit();
    }
  }
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e - r * n;
    W[r * ld + c] = r == c ? T(1) : T(0);
  }
  if constexpr (sizeof(T) == 4 && REG_CHAIN && WT_PRODUCTS) {
    if (wt_ok)
      for (int e = threadIdx.x; e < n * reg_chain_ldt(n); e += blockDim.x) WT[e] = 0.0f;
  }
  if (wt_ok)
    cp_async_wait_one();
  else
    cp_async_wait_all();
  __syncthreads();
  // lower(S1) = C, W = C^{-1} (zeros above)
  if constexpr (sizeof(T) == 4 && REG_CHAIN) {
    if (!cta_chol_inv_regs(S1, ld, n, W, ld, Pt, Vt, wt_ok ? WT : nullptr))
      cta_chol_solve<T, true, true>(S1, ld, n, W, ld, n);
  } else {
    cta_chol_solve<T, true, true>(S1, ld, n, W, ld, n);
  }
  check_factor(p, b, i, S1, ld);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e - r * n;
    if constexpr (sizeof(T) == 4 && WT_PRODUCTS)
      if (wt_ok) {
        Li[e] = c <= r ? S1[r * ld + c] : (INV ? WT[r * reg_chain_ldt(n) + c] : 0.0f);
        continue;
      }
    Li[e] = c <= r ? S1[r * ld + c] : (INV ? W[c * ld + r] : T(0));
  }
  const int mc0 = WITH_Y ? min_i(kMC, p.m) : 0;
  if constexpr (sizeof(T) == 4 && WT_PRODUCTS) {
    if (wt_ok) {   // R, Lf and y arrived during the chain
      cp_async_wait_all();
      __syncthreads();
      node_products_wt<WITH_Y>(n, WT, reg_chain_ldt(n), Rb, S2, ld, Y, ldy, mc0, R, Lf, yi, p.m, 0, right, left);
      return;
    }
  }
  __syncthreads();
  if (right) async_load(S1, ld, R, n, n, n);
  if (WITH_Y) async_load(Y, ldy, yi, n, mc0, p.m);
  cp_async_wait_all();
  __syncthreads();
  // F[r][c] = sum_k R[r][k] W[c][k]
  if (right)
    cta_gemm<T, false, true>(n, n, n, S1, ld, W, ld, [&](int r, int c, T v) { R[(long long)r * n + c] = v; });
  // G[r][c] = sum_k W[r][k] Lf[k][c]
  if (left)
    cta_gemm<T, false, false>(n, n, n, W, ld, S2, ld, [&](int r, int c, T v) { Lf[(long long)r * n + c] = v; });
  if (WITH_Y) {
    for (int c0 = 0; c0 < p.m; c0 += kMC) {
      const int mc = min_i(kMC, p.m - c0);
      if (c0 > 0) {
        __syncthreads();
        async_load(Y, ldy, yi + c0, n, mc, p.m);
        cp_async_wait_all();
        __syncthreads();
      }
      cta_gemm<T, false, false>(n, mc, n, W, ld, Y, ldy,
                                [&](int r, int c, T v) { yi[(long long)r * p.m + c0 + c] = v; });
    }
  }
}

// info reset before a factor: 0 for every batch entry
__global__ void k_info_reset(int* info, int B) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) info[b] = 0;
}

// node body used by the level kernels: inverse-first for small blocks
__host__ __device__ inline bool node_uses_gemm(int n) { return n <= kNodeGemmMaxN; }
__host__ __device__ inline bool inv_first_node(int n) { return node_uses_gemm(n); }
// dynamic shared memory (elements) of k_node; m_y = right-hand sides solved in the node (0 without y)
__host__ __device__ inline long long smem_node_launch_elems(int n, int m_y, int es, int threads = 256) {
  return node_uses_gemm(n) ? smem_node_gemm_elems(n, m_y, es, false, reg_chain_ok(n, threads))
                           : smem_node_elems(n, es);
}

template <typename T, bool WITH_Y, bool INV = false, bool WT_PRODUCTS = false>
__global__ void __launch_bounds__(256, sizeof(T) == 8 ? 1 : 2) k_node(Problem<T> p, Level lv) {
  const int b = blockIdx.x / lv.d;
  const int t = blockIdx.x - b * lv.d;
  pdl_wait();
  pdl_trigger();
  if (!p.active(b)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (node_uses_gemm(p.n))
    node_gemm_body<T, WITH_Y, INV, true, WT_PRODUCTS>(p, lv, b, t, smem_raw);
  else
    node_body<T, WITH_Y, INV>(p, lv, b, t, smem_raw, node_chunk(p.n, sizeof(T)));
}

// ---------------------------------------------------------------------------
// k_update
// ---------------------------------------------------------------------------
__device__ __forceinline__ void lower_tile_index(int lt, int& ta, int& tc) {
  int a = 0;
  while ((a + 1) * (a + 2) / 2 <= lt) ++a;
  ta = a;
  tc = lt - a * (a + 1) / 2;
}

// Number of output tiles of one update level per instance: U targets with
// nlt lower tiles each, then d-1 fill-in blocks with nt*nt tiles each.
__host__ __device__ inline int update_tiles(int n, int N, const Level& lv) {
  const int nt = ceil_div(n, lv.tile);
  return (N / (2 * lv.s)) * (nt * (nt + 1) / 2) + (lv.d - 1) * nt * nt;
}

// Body of one output tile `task` in [0, update_tiles) of instance b.
template <typename T>
__device__ __forceinline__ void update_body(const Problem<T>& p, const Level& lv, int b, int task,
                                            unsigned char* smem_raw) {
  constexpr int es = sizeof(T);
  const int n = p.n, N = p.N, s = lv.s;
  const int tile = lv.tile;
  const int nt = ceil_div(n, tile);
  const int nlt = nt * (nt + 1) / 2;
  const int U = N / (2 * s);
  T* Ab = reinterpret_cast<T*>(smem_raw);

  if (task < U * nlt) {
    const int u = task / nlt + 1;
    int ta, tc;
    lower_tile_index(task - (u - 1) * nlt, ta, tc);
    const int j = 2 * s * u - 1;
    const T* F = p.Eb(b, lv.oc + 2 * (u - 1));
    const bool hasG = j + s < N;
    const T* G = hasG ? p.Eb(b, lv.oc + 2 * u - 1) : nullptr;
    const int r0 = ta * tile, wa = min_i(tile, n - r0);
    const int c0 = tc * tile, wc = min_i(tile, n - c0);
    const bool diag = ta == tc;
    const int K = hasG ? 2 * n : n;
    const int lda = update_ld(K, es);       // rows of [F | G^T]
    T* Bb = Ab + tile * lda;
    T* Bop = diag ? Ab : Bb;
    // Ab[r][k] = F[r0+r][k], Ab[r][n+k] = G[k][r0+r]   (k < n)
    async_load(Ab, lda, F + (long long)r0 * n, wa, n, n);
    if (hasG) async_load_t(Ab + n, lda, G + r0, n, wa, n);
    if (!diag) {
      async_load(Bb, lda, F + (long long)c0 * n, wc, n, n);
      if (hasG) async_load_t(Bb + n, lda, G + c0, n, wc, n);
    }
    cp_async_wait_all();
    __syncthreads();
    T* Lj = p.Lb(b, j);
    auto out = [&](int r, int c, T v) { Lj[(long long)(r0 + r) * n + c0 + c] -= v; };
    if (diag)
      cta_gemm<T, false, true, true>(wa, wc, K, Ab, lda, Bop, lda, out);
    else
      cta_gemm<T, false, true, false>(wa, wc, K, Ab, lda, Bop, lda, out);
  } else {
    const int f = task - U * nlt;
    const int t = f / (nt * nt) + 1;
    const int tt = f - (t - 1) * nt * nt;
    const int ta = tt / nt, tc = tt - ta * nt;
    const int i = s - 1 + 2 * s * t;
    if (i + s >= N) return;
    const T* F = p.Eb(b, lv.oc + 2 * t);
    const T* G = p.Eb(b, lv.oc + 2 * t - 1);
    T* X = p.Eb(b, lv.on + t - 1);
    const int r0 = ta * tile, wa = min_i(tile, n - r0);
    const int c0 = tc * tile, wc = min_i(tile, n - c0);
    const int lda = update_ld(n, es), ldg = update_ld(tile, es);
    T* Bb = Ab + tile * lda;
    async_load(Ab, lda, F + (long long)r0 * n, wa, n, n);   // F rows
    async_load(Bb, ldg, G + c0, n, wc, n);                    // G columns, n x wc
    cp_async_wait_all();
    __syncthreads();
    cta_gemm<T, false, false>(wa, wc, n, Ab, lda, Bb, ldg,
                              [&](int r, int c, T v) { X[(long long)(r0 + r) * n + c0 + c] -= v; });
  }
}

// Whole-block update for n <= kNodeGemmMaxN: task u-1 < U updates target
// j = 2su-1 completely (all lower tiles, K = 2n), task U + t-1 forms the whole
// fill-in block of node t.  One CTA per block keeps every warp busy.
__host__ __device__ inline int update_blocks(int N, const Level& lv) { return N / (2 * lv.s) + lv.d - 1; }
// n <= 64 updates run on DMMA for both types; float rows padded to 4 (mod 32)
// words so the fragment loads hit distinct banks
__host__ __device__ inline int update_full_ld(int k, int es) { return es == 8 ? update_ld(k, es) : ((k + 3) & ~3) + 4; }
__host__ __device__ inline long long smem_update_full_elems(int n, int es) {
  const long long a = (long long)n * update_full_ld(2 * n, es);
  const long long f = 2LL * n * update_full_ld(n, es);
  return a > f ? a : f;
}

template <typename T>
__device__ __forceinline__ void update_full_body(const Problem<T>& p, const Level& lv, int b, int task,
                                                 unsigned char* smem_raw) {
  constexpr int es = sizeof(T);
  const int n = p.n, N = p.N, s = lv.s;
  const int U = N / (2 * s);
  T* Ab = reinterpret_cast<T*>(smem_raw);
  if (task < U) {
    const int u = task + 1;
    const int j = 2 * s * u - 1;
    const T* F = p.Eb(b, lv.oc + 2 * (u - 1));
    const bool hasG = j + s < N;
    const T* G = hasG ? p.Eb(b, lv.oc + 2 * u - 1) : nullptr;
    const int K = hasG ? 2 * n : n;
    const int lda = update_full_ld(2 * n, es);
    // Ab[r][k] = F[r][k], Ab[r][n+k] = G[k][r]
    async_load(Ab, lda, F, n, n, n);
    if (hasG) async_load_t(Ab + n, lda, G, n, n, n);
    cp_async_wait_all();
    __syncthreads();
    T* Lj = p.Lb(b, j);
    // DMMA for both types (float operands widened: one rounding per entry)
    warp_gemm_dmma<T, false, true, true>(n, n, K, Ab, lda, Ab, lda, [&](int r, int c, double v) {
      T* o = Lj + (long long)r * n + c;
      *o = (T)((double)*o - v);
    });
  } else {
    const int t = task - U + 1;
    const int i = s - 1 + 2 * s * t;
    if (i + s >= N) return;
    const T* F = p.Eb(b, lv.oc + 2 * t);
    const T* G = p.Eb(b, lv.oc + 2 * t - 1);
    T* X = p.Eb(b, lv.on + t - 1);
    const int ld = update_full_ld(n, es);
    T* Bb = Ab + n * ld;
    async_load(Ab, ld, F, n, n, n);
    async_load(Bb, ld, G, n, n, n);
    cp_async_wait_all();
    __syncthreads();
    warp_gemm_dmma<T, false, false>(n, n, n, Ab, ld, Bb, ld, [&](int r, int c, double v) {
      T* o = X + (long long)r * n + c;
      *o = (T)((double)*o - v);
    });
  }
}

// ---------------------------------------------------------------------------
// Whole-block update for 64 < n <= 128 (same tasks as update_full_body): one
// CTA of 256 threads per target / fill-in block, K streamed through shared
// memory in kBigKC-column chunks (target: A = [F | G^T], B = A; fill-in:
// A = F, B(c, k) = G[k][c]), and each warp keeping the accumulators of up to
// kBigTiles 16 x 32 DMMA tiles of the n x n output (lower tiles only for a
// target) in registers across the chunks; float operands are widened (exact
// products, FP64 sums, one rounding per entry).
// ---------------------------------------------------------------------------
constexpr int kBigMaxN = 128;
constexpr int kBigKC = 32;
constexpr int kBigLd = kBigKC + 4;   // 4 (mod 16) doubles: conflict-free fragments
constexpr int kBigTiles = 4;         // (128/16) x (128/32) = 32 tiles over 8 warps
// two chunk buffers (A and B each): the next chunk's copies overlap this chunk's products
__host__ __device__ inline long long smem_update_big_elems(int n) { return 4LL * n * kBigLd; }
__host__ __device__ inline bool update_uses_big(int n) { return n > kNodeGemmMaxN && n <= kBigMaxN; }

template <typename T>
__device__ __forceinline__ void update_big_body(const Problem<T>& p, const Level& lv, int b, int task,
                                                unsigned char* smem_raw) {
  const int n = p.n, N = p.N, s = lv.s;
  const int U = N / (2 * s);
  T* buf = reinterpret_cast<T*>(smem_raw);   // [2][A | B], each n x kBigLd
  const bool target = task < U;
  const T *F, *G;
  T* Out;
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
  // asynchronous copies of chunk c (columns [32c, 32c + 32) of A and B) into
  // buffer c & 1; columns past K are zero-filled with plain stores
  auto stage = [&](int c) {
    T* As = buf + (c & 1) * 2 * n * kBigLd;
    T* Bs = As + n * kBigLd;
    const int k0 = c * kBigKC, kw = min_i(kBigKC, K - k0);
    if (k0 + kw <= n) {
      // A(r, kk) = F[r][k0 + kk]: rows of F
      for (int e = threadIdx.x; e < n * kw; e += blockDim.x) {
        const int r = e / kw, kk = e - r * kw;
        cp_async_elem(As + r * kBigLd + kk, F + (long long)r * n + k0 + kk);
      }
    } else if (k0 >= n) {
      // A(r, kk) = G[k0 + kk - n][r]: rows of G, transposed
      for (int e = threadIdx.x; e < n * kw; e += blockDim.x) {
        const int kk = e / n, r = e - kk * n;
        cp_async_elem(As + r * kBigLd + kk, G + (long long)(k0 + kk - n) * n + r);
      }
    } else {
      for (int e = threadIdx.x; e < n * kw; e += blockDim.x) {
        const int r = e / kw, kk = e - r * kw, k = k0 + kk;
        cp_async_elem(As + r * kBigLd + kk, k < n ? F + (long long)r * n + k : G + (long long)(k - n) * n + r);
      }
    }
    if (!target)   // B(c, kk) = G[k0 + kk][c]
      for (int e = threadIdx.x; e < n * kw; e += blockDim.x) {
        const int kk = e / n, cc = e - kk * n;
        cp_async_elem(Bs + cc * kBigLd + kk, G + (long long)(k0 + kk) * n + cc);
      }
    if (kw < kBigKC)
      for (int e = threadIdx.x; e < n * (kBigKC - kw); e += blockDim.x) {
        const int r = e / (kBigKC - kw), kk = kw + e - r * (kBigKC - kw);
        As[r * kBigLd + kk] = T(0);
        if (!target) Bs[r * kBigLd + kk] = T(0);
      }
    cp_async_commit();
  };
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int tm = (n + 15) / 16, tn = (n + 31) / 32;
  // this warp's tiles: the warp-th, (warp + nw)-th, ... tile of the (lower) tile list
  int tr[kBigTiles], tc[kBigTiles];
  int nt = 0;
  {
    int idx = 0;
    for (int i = 0; i < tm; ++i)
      for (int j = 0; j < tn; ++j) {
        if (target && 32 * j > 16 * i + 15) continue;
        if (idx % nw == warp && nt < kBigTiles) {
          tr[nt] = i * 16;
          tc[nt] = j * 32;
          ++nt;
        }
        ++idx;
      }
  }
  double acc[kBigTiles][2][4][2];
#pragma unroll
  for (int q = 0; q < kBigTiles; ++q)
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[q][i][j][0] = acc[q][i][j][1] = 0.0;
  const int chunks = (K + kBigKC - 1) / kBigKC;
  stage(0);
  for (int c = 0; c < chunks; ++c) {
    if (c + 1 < chunks) stage(c + 1);
    else cp_async_commit();       // empty group: wait_group 1 then covers chunk c
    cp_async_wait_one();
    __syncthreads();
    const T* As = buf + (c & 1) * 2 * n * kBigLd;
    const T* Bsrc = target ? As : As + n * kBigLd;
#pragma unroll
    for (int q = 0; q < kBigTiles; ++q) {
      if (q >= nt) break;
      int ra[2], cb[4];
#pragma unroll
      for (int i = 0; i < 2; ++i) ra[i] = min_i(tr[q] + 8 * i + g, n - 1);
#pragma unroll
      for (int j = 0; j < 4; ++j) cb[j] = min_i(tc[q] + 8 * j + g, n - 1);
#pragma unroll 2
      for (int kq = 0; kq < kBigKC; kq += 4) {
        const int kk = kq + tq;
        double a[2], bb[4];
#pragma unroll
        for (int i = 0; i < 2; ++i) a[i] = (double)As[ra[i] * kBigLd + kk];
#pragma unroll
        for (int j = 0; j < 4; ++j) bb[j] = (double)Bsrc[cb[j] * kBigLd + kk];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma_8x8x4(acc[q][i][j][0], acc[q][i][j][1], a[i], bb[j]);
      }
    }
    __syncthreads();   // buffer c & 1 is restaged for chunk c + 2
  }
  // epilogue: Out -= D (lower triangle for a target)
#pragma unroll
  for (int q = 0; q < kBigTiles; ++q) {
    if (q >= nt) break;
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int r = tr[q] + 8 * i + g, c = tc[q] + 8 * j + 2 * tq + e;
          if (r < n && c < n && (!target || c <= r)) {
            T* o = Out + (long long)r * n + c;
            *o = (T)((double)*o - acc[q][i][j][e]);
          }
        }
  }
}

__host__ __device__ inline bool update_uses_full(int n) { return n <= kNodeGemmMaxN; }
__host__ __device__ inline int update_launch_tasks(int n, int N, const Level& lv) {
  return (update_uses_full(n) || update_uses_big(n)) ? update_blocks(N, lv) : update_tiles(n, N, lv);
}
__host__ __device__ inline long long smem_update_launch_elems(int n, int es, int tile = kTile) {
  if (update_uses_big(n)) return smem_update_big_elems(n);
  return update_uses_full(n) ? smem_update_full_elems(n, es) : smem_update_elems(n, es, tile);
}

template <typename T>
__global__ void __launch_bounds__(256) k_update(Problem<T> p, Level lv) {
  const int per_b = update_launch_tasks(p.n, p.N, lv);
  const int b = blockIdx.x / per_b;
  const int task = blockIdx.x - b * per_b;
  pdl_wait();
  pdl_trigger();
  if (!p.active(b)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  if (update_uses_full(p.n))
    update_full_body<T>(p, lv, b, task, smem_raw);
  else
    update_body<T>(p, lv, b, task, smem_raw);
}

// 64 < n <= 128: whole-block update (its own kernel: its register-held
// accumulators would lower the occupancy of the small-block update)
template <typename T>
__global__ void __launch_bounds__(256, 1) k_update_big(Problem<T> p, Level lv) {
  const int per_b = update_blocks(p.N, lv);
  const int b = blockIdx.x / per_b;
  const int task = blockIdx.x - b * per_b;
  pdl_wait();
  pdl_trigger();
  if (!p.active(b)) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  update_big_body<T>(p, lv, b, task, smem_raw);
}

// ---------------------------------------------------------------------------
// Sweeps.  Shared layout: Y, Z1, Z2 (n x (mc+1) each), Cc (n x (kTile+1)), dv (kTile)
// ---------------------------------------------------------------------------

// Y -= op(M1) Z1 + op(M2) Z2 with M1, M2 n x n global blocks (a null M skips
// its product), streamed through two Cc buffers in kTile chunks of the
// contraction index: the copies of chunk c + 1 are in flight while chunk c's
// product runs.  TRx: op(M)[r][k] = M[k][r].  Each chunk's product runs on the
// FP64 tensor cores (DMMA warp tiles of 16 x 32; float operands widened in
// registers, FP64 sums, one rounding per entry and chunk): with n > 64 and
// many right-hand sides these products, not the block loads, bound the sweep.
template <typename T, bool TR1, bool TR2>
__device__ void sweep_accumulate2(T* Y, const T* Z1, const T* __restrict__ M1, const T* Z2,
                                  const T* __restrict__ M2, int ldy, int mc, int n, T* Cc) {
  constexpr int ldc = kSweepLdc;
  const int per = (n + kTile - 1) / kTile;
  const int c1 = M1 ? per : 0, total = c1 + (M2 ? per : 0);
  if (total == 0) return;
  auto stage = [&](int c) {
    T* dst = Cc + (c & 1) * n * ldc;
    const bool first = c < c1;
    const T* M = first ? M1 : M2;
    const bool tr = first ? TR1 : TR2;
    const int k0 = (first ? c : c - c1) * kTile, kw = min_i(kTile, n - k0);
    if (tr)
      async_load_t(dst, ldc, M + (long long)k0 * n, kw, n, n);   // dst[r][kk] = M[k0+kk][r]
    else
      async_load(dst, ldc, M + k0, n, kw, n);                   // dst[r][kk] = M[r][k0+kk]
    cp_async_commit();
  };
  __syncthreads();
  stage(0);
  for (int c = 0; c < total; ++c) {
    if (c + 1 < total) stage(c + 1);
    else cp_async_commit();
    cp_async_wait_one();
    __syncthreads();
    const bool first = c < c1;
    const int k0 = (first ? c : c - c1) * kTile, kw = min_i(kTile, n - k0);
    const T* Z = first ? Z1 : Z2;
    warp_gemm_dmma<T, false, false>(n, mc, kw, Cc + (c & 1) * n * ldc, ldc, Z + k0 * ldy, ldy,
                                    [&](int r, int cc, double v) {
                                      T* o = Y + r * ldy + cc;
                                      *o = (T)((double)*o - v);
                                    });
    __syncthreads();
  }
}

// Y <- C^{-1} Y (lower C = lower(Lb)), blocked by kTile rows: a warp takes
// four columns at once (lane = row of the panel), so the panel elements are
// loaded once for four columns and the four substitution chains interleave.
constexpr int kSolveCols = 4;
template <typename T>
__device__ void sweep_lower_solve(T* Y, int ldy, int mc, const T* __restrict__ Lb, int n, T* Cc, T* dv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int ldc = n + 1;  // Cc holds >= kTile * (n + 1) elements
  for (int K = 0; K < n; K += kTile) {
    const int kb = min_i(kTile, n - K);
    __syncthreads();
    async_load(Cc, ldc, Lb + (long long)K * n, kb, K + kb, n);   // rows [K,K+kb), cols [0,K+kb)
    cp_async_wait_all();
    __syncthreads();
    if (threadIdx.x < kb) dv[threadIdx.x] = T(1) / Cc[threadIdx.x * ldc + K + threadIdx.x];
    __syncthreads();
    for (int cb = warp; cb < mc; cb += nw * kSolveCols) {
      int col[kSolveCols];
      bool cv[kSolveCols];
#pragma unroll
      for (int q = 0; q < kSolveCols; ++q) {
        col[q] = cb + q * nw;
        cv[q] = col[q] < mc;
        if (!cv[q]) col[q] = cb;
      }
      T v[kSolveCols];
#pragma unroll
      for (int q = 0; q < kSolveCols; ++q) v[q] = lane < kb ? Y[(K + lane) * ldy + col[q]] : T(0);
      if (lane < kb) {
        for (int k = 0; k < K; ++k) {
          const T cm = Cc[lane * ldc + k];
#pragma unroll
          for (int q = 0; q < kSolveCols; ++q) v[q] = fma(-cm, Y[k * ldy + col[q]], v[q]);
        }
      }
      for (int j = 0; j < kb; ++j) {
        const T cj = (lane > j && lane < kb) ? Cc[lane * ldc + K + j] : T(0);
#pragma unroll
        for (int q = 0; q < kSolveCols; ++q) {
          const T yj = __shfl_sync(kFull, v[q], j) * dv[j];
          v[q] = lane == j ? yj : fma(-cj, yj, v[q]);
        }
      }
      if (lane < kb) {
#pragma unroll
        for (int q = 0; q < kSolveCols; ++q)
          if (cv[q]) Y[(K + lane) * ldy + col[q]] = v[q];
      }
    }
  }
  __syncthreads();
}

// Y <- C^{-T} Y (lower C = lower(Lb)), blocks from the bottom, four columns per warp.
template <typename T>
__device__ void sweep_upper_solve(T* Y, int ldy, int mc, const T* __restrict__ Lb, int n, T* Cc, T* dv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  constexpr int ldc = kTile + 1;
  const int last = ((n - 1) / kTile) * kTile;
  for (int K = last; K >= 0; K -= kTile) {
    const int kb = min_i(kTile, n - K);
    __syncthreads();
    // column panel: rows [K, n), columns [K, K+kb): Cc[(k-K)][r] = C[k][K+r]
    async_load(Cc, ldc, Lb + (long long)K * n + K, n - K, kb, n);
    cp_async_wait_all();
    __syncthreads();
    if (threadIdx.x < kb) dv[threadIdx.x] = T(1) / Cc[threadIdx.x * ldc + threadIdx.x];
    __syncthreads();
    for (int cb = warp; cb < mc; cb += nw * kSolveCols) {
      int col[kSolveCols];
      bool cv[kSolveCols];
#pragma unroll
      for (int q = 0; q < kSolveCols; ++q) {
        col[q] = cb + q * nw;
        cv[q] = col[q] < mc;
        if (!cv[q]) col[q] = cb;
      }
      T v[kSolveCols];
#pragma unroll
      for (int q = 0; q < kSolveCols; ++q) v[q] = lane < kb ? Y[(K + lane) * ldy + col[q]] : T(0);
      if (lane < kb) {
        for (int k = K + kb; k < n; ++k) {
          const T cm = Cc[(k - K) * ldc + lane];
#pragma unroll
          for (int q = 0; q < kSolveCols; ++q) v[q] = fma(-cm, Y[k * ldy + col[q]], v[q]);
        }
      }
      for (int j = kb - 1; j >= 0; --j) {
        const T cj = lane < j ? Cc[j * ldc + lane] : T(0);
#pragma unroll
        for (int q = 0; q < kSolveCols; ++q) {
          const T xj = __shfl_sync(kFull, v[q], j) * dv[j];
          v[q] = lane == j ? xj : fma(-cj, xj, v[q]);
        }
      }
      if (lane < kb) {
#pragma unroll
        for (int q = 0; q < kSolveCols; ++q)
          if (cv[q]) Y[(K + lane) * ldy + col[q]] = v[q];
      }
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Resident sweep helpers: the whole factor block and both coupling blocks of
// a node sit in shared memory (one load round), Y/Z are n x mc column chunks.
// Leading dimensions are even so every load can be vectorised.
// ---------------------------------------------------------------------------
// vector leading dimension of the resident sweeps: rows start on 16 bytes and
// every 8-column pass can read 8 elements past its first column
__host__ __device__ inline int res_ldy(int mc) { return ((mc + 3) / 4) * 4 + 4; }
// block leading dimension of the resident sweeps: rows start on 16 bytes (one
// 16-byte copy per 4 floats / 2 doubles) and 4 threads x 8 rows of a warp hit
// distinct banks in the row-major reads
__host__ __device__ inline int res_ldm(int n) { return ((n + 3) & ~3) + 4; }
// elements of one resident-sweep region, rounded so the next region starts on
// 128 bytes (TMA destinations)
__host__ __device__ inline long long res_round(long long elems, int es) {
  const long long q = 128 / es;
  return ((elems + q - 1) / q) * q;
}
// three vector regions, three block regions, dv (n) and two mbarriers; the
// 4-byte rounding is the larger, so the count covers both element sizes
__host__ __device__ inline long long smem_sweep_res_elems(int n, int m) {
  const int mc = min_i(m, kMC);
  return 3LL * res_round((long long)n * res_ldy(mc), 4) + 3LL * res_round((long long)n * res_ldm(n), 4) + n + 8;
}

// TMA use of one resident-sweep CTA: block and vector loads by the validity of
// their maps and a 128-byte aligned shared base (the same in every thread);
// initialises the two mbarriers (all threads call).
struct ResTma {
  bool blocks, vecs;
};
__device__ __forceinline__ ResTma res_tma_begin(const SweepMaps* tm, unsigned char* raw, uint64_t* bar) {
  ResTma r{false, false};
  if (tm == nullptr || (smem_addr(raw) & 127u) != 0) return r;
  r.blocks = tm->blocks != 0;
  r.vecs = tm->vecs != 0;
  if (r.blocks || r.vecs) {
    if (threadIdx.x == 0) {
      tc::mbar_init(bar, 1);
      tc::mbar_init(bar + 1, 1);
    }
    __syncthreads();
  }
  return r;
}

// Wait for this chunk's TMA copies: the blocks (first chunk) and the vectors;
// false (in every thread) if a wait ran out.
__device__ __forceinline__ bool res_tma_wait(const ResTma& tu, bool blocks_pending, uint64_t* bar, int chunk) {
  const bool okb = (tu.blocks && blocks_pending) ? tma::wait(bar, 0) : true;
  const bool okv = tu.vecs ? tma::wait(bar + 1, (unsigned)chunk & 1u) : true;
  return okb && okv;
}

// CW consecutive elements from 16-byte-aligned shared memory (8-byte for CW = 2 floats)
template <typename T, int CW>
__device__ __forceinline__ void load_cols(const T* p, T (&v)[CW]) {
  if constexpr (CW == 1) {
    v[0] = p[0];
  } else if constexpr (sizeof(T) == 4 && CW == 2) {
    const float2 a = *reinterpret_cast<const float2*>(p);
    v[0] = a.x; v[1] = a.y;
  } else if constexpr (sizeof(T) == 4) {
#pragma unroll
    for (int h = 0; h < CW / 4; ++h) {
      const float4 a = *reinterpret_cast<const float4*>(p + 4 * h);
      v[4 * h] = a.x; v[4 * h + 1] = a.y; v[4 * h + 2] = a.z; v[4 * h + 3] = a.w;
    }
  } else {
#pragma unroll
    for (int h = 0; h < CW / 2; ++h) {
      const double2 a = *reinterpret_cast<const double2*>(p + 2 * h);
      v[2 * h] = a.x; v[2 * h + 1] = a.y;
    }
  }
}

// Resident block times resident vectors, n <= 64 rows, up to kMC columns:
//   MODE 0: Yout -= M Z            M(r,k) = M[r*ldm + k]
//   MODE 1: Yout -= M^T Z          M(r,k) = M[k*ldm + r]
//   MODE 2: Yout = W^T Z           W^T(r,k) = M[r*ldm + k] for k > r, diagonal dv[r]
//   MODE 3: Yout = W Z             W(r,k) = M[k*ldm + r] for k < r, diagonal dv[r]
// (modes 2/3 read the inverse W = C^{-1} that an inverse-carrying factor keeps
// in its strict upper triangle).  Four consecutive threads share a row and
// split its contraction; each holds CW output columns in registers (CW = 8,
// 4, 2 or 1 by the column count), reads Z rows with vector loads (rows are
// 16-byte aligned, ldy from res_ldy) and the four partial rows are combined
// with two shuffles.
template <typename T, int MODE, int CW>
__device__ __forceinline__ void res_rowdot(T* Yout, const T* Z, int ldy, int mc, const T* M, int ldm, const T* dv,
                                           int n) {
  const int q = threadIdx.x & 3;
  const int nr = ((n + 7) / 8) * 8;   // whole warps iterate together (shuffles)
  for (int c0 = 0; c0 < mc; c0 += CW) {
    for (int rb = threadIdx.x >> 2; rb < nr; rb += blockDim.x >> 2) {
      const int r = rb < n ? rb : n - 1;
      T acc[CW];
#pragma unroll
      for (int j = 0; j < CW; ++j) acc[j] = T(0);
      const int k0 = MODE == 2 ? r + 1 : 0, k1 = MODE == 3 ? r : n;
#pragma unroll 4
      for (int k = k0 + q; k < k1; k += 4) {
        const T mv = (MODE == 0 || MODE == 2) ? M[r * ldm + k] : M[k * ldm + r];
        T z[CW];
        load_cols<T, CW>(Z + k * ldy + c0, z);
#pragma unroll
        for (int j = 0; j < CW; ++j) acc[j] = fma(mv, z[j], acc[j]);
      }
#pragma unroll
      for (int j = 0; j < CW; ++j) {
        acc[j] += __shfl_xor_sync(kFull, acc[j], 1);
        acc[j] += __shfl_xor_sync(kFull, acc[j], 2);
      }
      if (rb < n) {
#pragma unroll
        for (int j = 0; j < CW; ++j) {
          if ((j & 3) != q || c0 + j >= mc) continue;
          if (MODE <= 1)
            Yout[r * ldy + c0 + j] -= acc[j];
          else
            Yout[r * ldy + c0 + j] = dv[r] * Z[r * ldy + c0 + j] + acc[j];
        }
      }
    }
  }
}

// Both coupling products of a sweep node in one pass:
//   Y -= A1 Z1 + A2 Z2,   A(r,k) = M[k*ldm + r] if transposed else M[r*ldm + k];
// a null M skips its product.  Same thread layout as res_rowdot.
template <typename T, int CW, bool TR1, bool TR2>
__device__ __forceinline__ void res_rowdot_pair(T* Y, const T* Z1, const T* M1, const T* Z2, const T* M2, int ldy,
                                                int mc, int ldm, int n) {
  const int q = threadIdx.x & 3;
  const int nr = ((n + 7) / 8) * 8;
  const bool h1 = M1 != nullptr, h2 = M2 != nullptr;
  for (int c0 = 0; c0 < mc; c0 += CW) {
    for (int rb = threadIdx.x >> 2; rb < nr; rb += blockDim.x >> 2) {
      const int r = rb < n ? rb : n - 1;
      T acc[CW];
#pragma unroll
      for (int j = 0; j < CW; ++j) acc[j] = T(0);
#pragma unroll 4
      for (int k = q; k < n; k += 4) {
        if (h1) {
          const T mv = TR1 ? M1[k * ldm + r] : M1[r * ldm + k];
          T z[CW];
          load_cols<T, CW>(Z1 + k * ldy + c0, z);
#pragma unroll
          for (int j = 0; j < CW; ++j) acc[j] = fma(mv, z[j], acc[j]);
        }
        if (h2) {
          const T mv = TR2 ? M2[k * ldm + r] : M2[r * ldm + k];
          T z[CW];
          load_cols<T, CW>(Z2 + k * ldy + c0, z);
#pragma unroll
          for (int j = 0; j < CW; ++j) acc[j] = fma(mv, z[j], acc[j]);
        }
      }
#pragma unroll
      for (int j = 0; j < CW; ++j) {
        acc[j] += __shfl_xor_sync(kFull, acc[j], 1);
        acc[j] += __shfl_xor_sync(kFull, acc[j], 2);
      }
      if (rb < n) {
#pragma unroll
        for (int j = 0; j < CW; ++j) {
          if ((j & 3) != q || c0 + j >= mc) continue;
          Y[r * ldy + c0 + j] -= acc[j];
        }
      }
    }
  }
}

template <typename T, bool TR1, bool TR2>
__device__ __forceinline__ void res_matvec_pair(T* Y, const T* Z1, const T* M1, const T* Z2, const T* M2, int ldy,
                                                int mc, int ldm, int n) {
  if (mc >= 8)
    res_rowdot_pair<T, 8, TR1, TR2>(Y, Z1, M1, Z2, M2, ldy, mc, ldm, n);
  else if (mc >= 4)
    res_rowdot_pair<T, 4, TR1, TR2>(Y, Z1, M1, Z2, M2, ldy, mc, ldm, n);
  else if (mc >= 2)
    res_rowdot_pair<T, 2, TR1, TR2>(Y, Z1, M1, Z2, M2, ldy, mc, ldm, n);
  else
    res_rowdot_pair<T, 1, TR1, TR2>(Y, Z1, M1, Z2, M2, ldy, mc, ldm, n);
}

template <typename T, int MODE>
__device__ __forceinline__ void res_matvec(T* Yout, const T* Z, int ldy, int mc, const T* M, int ldm, const T* dv,
                                           int n) {
  if (mc >= 8)
    res_rowdot<T, MODE, 8>(Yout, Z, ldy, mc, M, ldm, dv, n);
  else if (mc >= 4)
    res_rowdot<T, MODE, 4>(Yout, Z, ldy, mc, M, ldm, dv, n);
  else if (mc >= 2)
    res_rowdot<T, MODE, 2>(Yout, Z, ldy, mc, M, ldm, dv, n);
  else
    res_rowdot<T, MODE, 1>(Yout, Z, ldy, mc, M, ldm, dv, n);
}

// ---------------------------------------------------------------------------
// Products of the resident inverse sweeps on FP64 tensor cores (mma.m8n8k4
// .f64), for float and double blocks: operands are widened to double in
// registers, so products are exact and sums are FP64; the result is rounded
// to T once.  A(r,k) = TR ? M[k*ld + r] : M[r*ld + k].
//   MODE 0: Out -= A1 Z1 + A2 Z2     (a null A skips its product)
//   MODE 2: Out  = dv .* Z1 + A1 Z1, A1 strictly upper (k > r)
//   MODE 3: Out  = dv .* Z1 + A1 Z1, A1 strictly lower (k < r)
// Out never aliases Z1 or Z2.  Warp task = one 8 x 8 output tile, all k-steps,
// two accumulators per product (alternate k-steps).  Fragment layout: a0 =
// A[g][t], b0 = B[t][g], {c0, c1} = C[g][2t + {0, 1}] (g = lane / 4, t = lane % 4).
// ---------------------------------------------------------------------------
// Sweep products on inverse-carrying factors: FP64 sweeps always take the
// tensor-core products (faster at every level); FP32 sweeps only in launches
// wider than one wave of resident sweep CTAs, which are throughput-bound
// (measured at N=1024, n=64: bottom level 17.0 -> 15.7 us), while the
// dependent DMMA chain costs ~0.6 us per node on the 1-256-CTA levels and in
// the persistent ragged CTAs, where the SIMT products are faster.  The host
// decides per launch (Level::tc, from the launch width and the device's SM
// count, or from a tuned setting).
template <typename T>
__device__ __forceinline__ bool sweep_uses_dmma(const Level& lv) {
  return sizeof(T) == 8 || lv.tc != 0;
}

template <typename T, int MODE, bool TR>
__device__ __forceinline__ double dmma_a(const T* A, int ld, int n, int r, int k) {
  bool ok = r < n && k < n;
  if (MODE == 2) ok = ok && k > r;
  if (MODE == 3) ok = ok && k < r;
  const int rr = r < n ? r : 0, kk = k < n ? k : 0;
  const T v = TR ? A[kk * ld + rr] : A[rr * ld + kk];
  return ok ? (double)v : 0.0;
}

template <typename T, int MODE, bool TR1, bool TR2>
__device__ void dmma_product(T* Out, const T* Z1, const T* A1, int ld1, const T* Z2, const T* A2, int ld2, int ldy,
                             int mc, const T* dv, int n) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int rt = (n + 7) >> 3, ct = (mc + 7) >> 3, kt = (n + 3) >> 2;
  const bool h1 = A1 != nullptr, h2 = MODE == 0 && A2 != nullptr;
  for (int task = warp; task < rt * ct; task += nw) {
    const int r0 = (task / ct) * 8, c0 = (task % ct) * 8;
    const int ra = r0 + g, cb = c0 + g;
    const bool cv = cb < mc;
    const int cc = cv ? cb : 0;
    double acc[4][2] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
    int kb0 = 0, kb1 = kt;
    if (MODE == 2) kb0 = (r0 + 1) >> 2;                             // first k-step with some k > r
    if (MODE == 3) kb1 = min_i(kt, (r0 + 7 + 3) >> 2);              // past the last with some k < r
    for (int kb = kb0; kb < kb1; kb += 2) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {   // two k-steps, one accumulator each
        const int k = (kb + h) * 4 + t;
        const bool kv = kb + h < kb1 && k < n;
        const int kk = kv ? k : 0;
        if (h1) {
          const double a = kv ? dmma_a<T, MODE, TR1>(A1, ld1, n, ra, kk) : 0.0;
          const double b = (kv && cv) ? (double)Z1[kk * ldy + cc] : 0.0;
          dmma_8x8x4(acc[h][0], acc[h][1], a, b);
        }
        if (h2) {
          const double a = kv ? dmma_a<T, MODE, TR2>(A2, ld2, n, ra, kk) : 0.0;
          const double b = (kv && cv) ? (double)Z2[kk * ldy + cc] : 0.0;
          dmma_8x8x4(acc[2 + h][0], acc[2 + h][1], a, b);
        }
      }
    }
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int r = r0 + g, c = c0 + 2 * t + e;
      if (r < n && c < mc) {
        const double v = (acc[0][e] + acc[1][e]) + (acc[2][e] + acc[3][e]);
        T* out = Out + r * ldy + c;
        if (MODE == 0)
          *out = (T)((double)*out - v);
        else
          *out = (T)((double)dv[r] * (double)Z1[r * ldy + c] + v);
      }
    }
  }
}

// Y <- C^{-1} Y (UPPER: Y <- C^{-T} Y), C = lower(Cs) resident, dv[r] = 1/C[r][r].
// Right-looking by 8-row blocks: one thread per column solves the block
// against the 8x8 diagonal block held in registers, then every (row, column)
// of the remaining rows takes an 8-term update.
template <typename T, bool UPPER>
__device__ void res_tri_solve(T* Y, int ldy, int mc, const T* Cs, int ldc, const T* dv, int n) {
  constexpr int BK = 8;
  const int nblk = (n + BK - 1) / BK;
  for (int bi = 0; bi < nblk; ++bi) {
    const int K = UPPER ? (nblk - 1 - bi) * BK : bi * BK;
    const int kb = min_i(BK, n - K);
    for (int c = threadIdx.x; c < mc; c += blockDim.x) {
      T x[BK];
#pragma unroll
      for (int j = 0; j < BK; ++j) x[j] = j < kb ? Y[(K + j) * ldy + c] : T(0);
      if (!UPPER) {
#pragma unroll
        for (int j = 0; j < BK; ++j) {
          if (j < kb) {
#pragma unroll
            for (int i = 0; i < j; ++i) x[j] = fma(-Cs[(K + j) * ldc + K + i], x[i], x[j]);
            x[j] *= dv[K + j];
          }
        }
      } else {
#pragma unroll
        for (int j = BK - 1; j >= 0; --j) {
          if (j < kb) {
#pragma unroll
            for (int i = j + 1; i < BK; ++i)
              if (i < kb) x[j] = fma(-Cs[(K + i) * ldc + K + j], x[i], x[j]);
            x[j] *= dv[K + j];
          }
        }
      }
#pragma unroll
      for (int j = 0; j < BK; ++j)
        if (j < kb) Y[(K + j) * ldy + c] = x[j];
    }
    __syncthreads();
    // remaining rows: below the block (forward) or above it (backward)
    const int r0 = UPPER ? 0 : K + kb;
    const int nr = UPPER ? K : n - K - kb;
    for (int o = threadIdx.x; o < nr * mc; o += blockDim.x) {
      const int r = r0 + o / mc, c = o - (o / mc) * mc;
      T acc = T(0);
#pragma unroll
      for (int j = 0; j < BK; ++j)
        if (j < kb) acc = fma(UPPER ? Cs[(K + j) * ldc + r] : Cs[r * ldc + K + j], Y[(K + j) * ldy + c], acc);
      Y[r * ldy + c] -= acc;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// k_fwd (level l): pull the level-(l-1) coupling updates and solve.
//   l == 0: task t -> node i = 2t:  y_i <- C_i^{-1} y_i
//   l >= 1: task u-1, target j = s*u - 1 of the level-(l-1) updates:
//           y_j -= F y_{j-s/2} + G^T y_{j+s/2}   (slots o_{l-1}+2u-2, +2u-1)
//           and for odd u (j is a level-l node) y_j <- C_j^{-1} y_j.
// Every vector has one writer per launch (K launches per forward sweep).
// RES: factor and coupling blocks resident in shared memory.
// ---------------------------------------------------------------------------
// PULL_ONLY (fused factor_and_solve): apply the updates, never solve.
// INV (resident only): the factor carries its inverse (k_node<INV>), the
// triangular solve becomes a matvec.
// Tasks of one forward level per instance.
__host__ __device__ inline int fwd_tasks(int N, const Level& lv) { return lv.s == 1 ? lv.d : N / lv.s; }

template <typename T, bool RES, bool PULL_ONLY, bool INV>
__device__ __forceinline__ void fwd_body(const Problem<T>& p, const Level& lv, int b, int task,
                                         unsigned char* smem_raw, const SweepMaps* tm = nullptr) {
  const int s = lv.s, N = p.N, n = p.n;
  const int h = s / 2;
  int j, slot = 0;
  bool pull, solve;
  const T *F = nullptr, *G = nullptr;
  if (s == 1) {
    j = 2 * task;
    pull = false;
    solve = true;
  } else {
    const int u = task + 1;
    j = s * u - 1;
    pull = true;
    solve = !PULL_ONLY && (u & 1) != 0;
    slot = lv.op + 2 * u - 2;
    F = p.Eb(b, slot);
    if (j + h < N) G = p.Eb(b, slot + 1);
  }
  const int mcmax = min_i(p.m, kMC), ldy = RES ? res_ldy(mcmax) : sweep_ldy(mcmax);
  // RES: Y, Z1, Z2 (n x ldy), C, F, G (n x ldm), dv (n), two mbarriers, regions on
  // 128 bytes; else Y, Z1, Z2, Cc (smem_sweep_elems), dv
  const long long vy = RES ? res_round((long long)n * ldy, sizeof(T)) : (long long)n * ldy;
  T* Y = reinterpret_cast<T*>(smem_raw);
  T* Z1 = Y + vy;
  T* Z2 = Z1 + vy;
  T* Ms = Z2 + vy;
  const int ldm = res_ldm(n);
  const long long vm = res_round((long long)n * ldm, sizeof(T));
  T* Cs = Ms;
  T* Fs = Cs + vm;
  T* Gs = Fs + vm;
  T* dv = RES ? Gs + vm : Ms + (smem_sweep_elems(n, p.m) - 3LL * n * ldy - kTile);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + ((reinterpret_cast<unsigned char*>(dv + n) - smem_raw + 7) & ~7LL));
  T* yj = p.Xb(b, j);
  const T* Lj = p.Lb(b, j);
  const ResTma tu = RES ? res_tma_begin(tm, smem_raw, bar) : ResTma{false, false};
  const int nblk = RES ? (solve ? 1 : 0) + (F ? 1 : 0) + (G ? 1 : 0) : 0;
  if (!lv.pre) pdl_wait();
  if (RES) {
    if (tu.blocks) {
      if (threadIdx.x == 0 && nblk > 0) {
        tma::expect_tx(bar, (uint32_t)(nblk * n * ldm * sizeof(T)));
        if (solve) tma::load_4d(Cs, &tm->L, 0, 0, j, b, bar);
        if (F) tma::load_4d(Fs, &tm->E, 0, 0, slot, b, bar);
        if (G) tma::load_4d(Gs, &tm->E, 0, 0, slot + 1, b, bar);
      }
    } else {
      if (solve) async_load(Cs, ldm, Lj, n, n, n);
      if (F) async_load(Fs, ldm, F, n, n, n);
      if (G) async_load(Gs, ldm, G, n, n, n);
    }
  }
  if (lv.pre) pdl_wait();
  pdl_trigger();
  for (int c0 = 0, chunk = 0; c0 < p.m; c0 += kMC, ++chunk) {
    const int mc = min_i(kMC, p.m - c0);
    __syncthreads();
    if (tu.vecs) {
      if (threadIdx.x == 0) {
        tma::fence_proxy();
        tma::expect_tx(bar + 1, (uint32_t)((1 + (pull ? 1 : 0) + (G ? 1 : 0)) * n * ldy * sizeof(T)));
        tma::load_4d(Y, &tm->X, c0, 0, j, b, bar + 1);
        if (pull) tma::load_4d(Z1, &tm->X, c0, 0, j - h, b, bar + 1);
        if (G) tma::load_4d(Z2, &tm->X, c0, 0, j + h, b, bar + 1);
      }
    } else {
      async_load(Y, ldy, yj + c0, n, mc, p.m);
      if (pull) async_load(Z1, ldy, p.Xb(b, j - h) + c0, n, mc, p.m);
      if (G) async_load(Z2, ldy, p.Xb(b, j + h) + c0, n, mc, p.m);
    }
    cp_async_wait_all();
    if ((tu.blocks || tu.vecs) && !res_tma_wait(tu, nblk > 0 && chunk == 0, bar, chunk)) return;
    __syncthreads();
    if (RES) {
      if (c0 == 0 && solve)
        for (int r = threadIdx.x; r < n; r += blockDim.x) dv[r] = T(1) / Cs[r * ldm + r];
      // Y -= F y_{j-h} + G^T y_{j+h}
      const bool tc = INV && sweep_uses_dmma<T>(lv);
      if (pull) {
        if (tc)
          dmma_product<T, 0, false, true>(Y, Z1, Fs, ldm, G ? Z2 : nullptr, G ? Gs : nullptr, ldm, ldy, mc, nullptr, n);
        else
          res_matvec_pair<T, false, true>(Y, Z1, Fs, G ? Z2 : nullptr, G ? Gs : nullptr, ldy, mc, ldm, n);
      }
      __syncthreads();
      if (solve) {
        if (INV) {
          if (tc)
            dmma_product<T, 3, true, false>(Z2, Y, Cs, ldm, nullptr, nullptr, 0, ldy, mc, dv, n);   // y = W Y
          else
            res_matvec<T, 3>(Z2, Y, ldy, mc, Cs, ldm, dv, n);
          __syncthreads();
          store_block(yj + c0, p.m, Z2, ldy, n, mc);
          continue;
        }
        res_tri_solve<T, false>(Y, ldy, mc, Cs, ldm, dv, n);
      }
    } else {
      if (pull) sweep_accumulate2<T, false, true>(Y, Z1, F, Z2, G, ldy, mc, n, Ms);
      if (solve) sweep_lower_solve(Y, ldy, mc, Lj, n, Ms, dv);
    }
    store_block(yj + c0, p.m, Y, ldy, n, mc);
  }
}

template <typename T, bool RES, bool PULL_ONLY = false, bool INV = false>
__global__ void __launch_bounds__(256) k_fwd(Problem<T> p, Level lv, const __grid_constant__ SweepMaps tm) {
  const int per_b = fwd_tasks(p.N, lv);
  const int b = blockIdx.x / per_b;
  const int task = blockIdx.x - b * per_b;
  if (!p.active(b)) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  fwd_body<T, RES, PULL_ONLY, INV>(p, lv, b, task, smem_raw, &tm);
}

// ---------------------------------------------------------------------------
// k_bwd (level l, descending): x_i -= F_i^T x_{i+s} + G_i x_{i-s};  x_i <- C_i^{-T} x_i
// ---------------------------------------------------------------------------
template <typename T, bool RES, bool INV>
__device__ __forceinline__ void bwd_body(const Problem<T>& p, const Level& lv, int b, int t,
                                         unsigned char* smem_raw, const SweepMaps* tm = nullptr) {
  const int n = p.n, s = lv.s, N = p.N;
  const int i = s - 1 + 2 * s * t;
  const int mcmax = min_i(p.m, kMC), ldy = RES ? res_ldy(mcmax) : sweep_ldy(mcmax);
  // shared layout as in fwd_body
  const long long vy = RES ? res_round((long long)n * ldy, sizeof(T)) : (long long)n * ldy;
  T* Y = reinterpret_cast<T*>(smem_raw);
  T* Z1 = Y + vy;
  T* Z2 = Z1 + vy;
  T* Ms = Z2 + vy;
  const int ldm = res_ldm(n);
  const long long vm = res_round((long long)n * ldm, sizeof(T));
  T* Cs = Ms;
  T* Fs = Cs + vm;
  T* Gs = Fs + vm;
  T* dv = RES ? Gs + vm : Ms + (smem_sweep_elems(n, p.m) - 3LL * n * ldy - kTile);
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + ((reinterpret_cast<unsigned char*>(dv + n) - smem_raw + 7) & ~7LL));
  const bool right = i + s < N, left = i >= s;
  const int slot = lv.oc + 2 * t;
  const T* F = right ? p.Eb(b, slot) : nullptr;
  const T* G = left ? p.Eb(b, slot - 1) : nullptr;
  const T* Li = p.Lb(b, i);
  T* xi = p.Xb(b, i);
  const ResTma tu = RES ? res_tma_begin(tm, smem_raw, bar) : ResTma{false, false};
  if (!lv.pre) pdl_wait();
  if (RES) {
    if (tu.blocks) {
      if (threadIdx.x == 0) {
        tma::expect_tx(bar, (uint32_t)((1 + (right ? 1 : 0) + (left ? 1 : 0)) * n * ldm * sizeof(T)));
        tma::load_4d(Cs, &tm->L, 0, 0, i, b, bar);
        if (right) tma::load_4d(Fs, &tm->E, 0, 0, slot, b, bar);
        if (left) tma::load_4d(Gs, &tm->E, 0, 0, slot - 1, b, bar);
      }
    } else {
      async_load(Cs, ldm, Li, n, n, n);
      if (right) async_load(Fs, ldm, F, n, n, n);
      if (left) async_load(Gs, ldm, G, n, n, n);
    }
  }
  if (lv.pre) pdl_wait();
  pdl_trigger();
  for (int c0 = 0, chunk = 0; c0 < p.m; c0 += kMC, ++chunk) {
    const int mc = min_i(kMC, p.m - c0);
    __syncthreads();
    if (tu.vecs) {
      if (threadIdx.x == 0) {
        tma::fence_proxy();
        tma::expect_tx(bar + 1, (uint32_t)((1 + (right ? 1 : 0) + (left ? 1 : 0)) * n * ldy * sizeof(T)));
        tma::load_4d(Y, &tm->X, c0, 0, i, b, bar + 1);
        if (right) tma::load_4d(Z1, &tm->X, c0, 0, i + s, b, bar + 1);
        if (left) tma::load_4d(Z2, &tm->X, c0, 0, i - s, b, bar + 1);
      }
    } else {
      async_load(Y, ldy, xi + c0, n, mc, p.m);
      if (right) async_load(Z1, ldy, p.Xb(b, i + s) + c0, n, mc, p.m);
      if (left) async_load(Z2, ldy, p.Xb(b, i - s) + c0, n, mc, p.m);
    }
    cp_async_wait_all();
    if ((tu.blocks || tu.vecs) && !res_tma_wait(tu, chunk == 0, bar, chunk)) return;
    __syncthreads();
    if (RES) {
      if (c0 == 0)
        for (int r = threadIdx.x; r < n; r += blockDim.x) dv[r] = T(1) / Cs[r * ldm + r];
      // Y -= F^T x_{i+s} + G x_{i-s}
      const bool tc = INV && sweep_uses_dmma<T>(lv);
      if (right || left) {
        if (tc)
          dmma_product<T, 0, true, false>(Y, right ? Z1 : nullptr, right ? Fs : nullptr, ldm, left ? Z2 : nullptr,
                                          left ? Gs : nullptr, ldm, ldy, mc, nullptr, n);
        else
          res_matvec_pair<T, true, false>(Y, right ? Z1 : nullptr, right ? Fs : nullptr, left ? Z2 : nullptr,
                                          left ? Gs : nullptr, ldy, mc, ldm, n);
      }
      __syncthreads();
      if (INV) {
        if (tc)
          dmma_product<T, 2, false, false>(Z1, Y, Cs, ldm, nullptr, nullptr, 0, ldy, mc, dv, n);   // x = W^T Y
        else
          res_matvec<T, 2>(Z1, Y, ldy, mc, Cs, ldm, dv, n);
        __syncthreads();
        store_block(xi + c0, p.m, Z1, ldy, n, mc);
        continue;
      }
      res_tri_solve<T, true>(Y, ldy, mc, Cs, ldm, dv, n);
    } else {
      sweep_accumulate2<T, true, false>(Y, Z1, F, Z2, G, ldy, mc, n, Ms);
      sweep_upper_solve(Y, ldy, mc, Li, n, Ms, dv);
    }
    store_block(xi + c0, p.m, Y, ldy, n, mc);
  }
}

template <typename T, bool RES, bool INV = false>
__global__ void __launch_bounds__(256) k_bwd(Problem<T> p, Level lv, const __grid_constant__ SweepMaps tm) {
  const int b = blockIdx.x / lv.d;
  const int t = blockIdx.x - b * lv.d;
  if (!p.active(b)) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  bwd_body<T, RES, INV>(p, lv, b, t, smem_raw, &tm);
}

}  // namespace socu
