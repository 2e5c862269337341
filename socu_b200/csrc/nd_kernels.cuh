// Per-level kernels of the nested-dissection block-tridiagonal Cholesky.
//
// One factor level l (stride s) is three launches, all deterministic (no
// floating-point atomics, every output block has exactly one writer):
//   k_diag    one CTA per level node i: C_i = chol(L_i) and C_i^{-1}
//             (socu: potrf K2, block_tridiag_solver.py:197-216).  With a RHS it
//             also applies y_i <- C_i^{-1} y_i (fused forward step, :108-110).
//   k_couple  one CTA per (node, side, 32-row/col panel):
//             right  F = E[o_l + i/s] C_i^{-T}        (trsm_rltn K3, :219-248)
//             left   G = C_i^{-1} E[o_l + (i-s)/s]    (trsm_llnn K4, :251-279)
//             both as GEMMs against the stored inverse.
//   k_update  one CTA per 32x32 output tile:
//             target j = 2 s u - 1 (owner computes; the reference uses
//             atomics here, K5/K6 :282-342)
//                 L_j -= F_{j-s} F_{j-s}^T + G_{j+s}^T G_{j+s}
//             fill-in for nodes with both neighbours (K7, :345-377)
//                 E[o_{l+1} + t - 1] -= F_t G_t
// Substitution sweeps (K9-K16, :425-736):
//   k_fwd_node     y_i <- C_i^{-1} y_i           (levels ascending)
//   k_fwd_update   y_j -= F_{j-s} y_{j-s} + G_{j+s}^T y_{j+s}   (owner computes)
//   k_bwd          x_i -= F_i^T x_{i+s} + G_i x_{i-s};  x_i <- C_i^{-T} x_i
//                  (levels descending)
#pragma once

#include "nd_device.cuh"

namespace socu {

constexpr int kDiagBS = 16;   // diagonal block of the in-CTA blocked Cholesky
constexpr int kTile = 32;     // output tile / panel width
constexpr int kMC = 32;       // RHS columns handled per pass

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

// shared-memory sizes (elements) ------------------------------------------------
__host__ __device__ inline int diag_ld(int n) { return n + 1; }
__host__ __device__ inline long long smem_diag_elems(int n, int m) {
  const int mc = m < kMC ? m : kMC;
  return (long long)n * diag_ld(n) + n + (long long)n * kDiagBS + (long long)n * (mc > 0 ? mc : 0);
}
__host__ __device__ inline long long smem_couple_elems(int n) {
  return (long long)n * diag_ld(n) + (long long)n * (kTile + 1);
}
__host__ __device__ inline long long smem_update_elems(int n) {
  return 2LL * kTile * (n + 1) + 2LL * n * (kTile + 1);
}
__host__ __device__ inline long long smem_sweep_elems(int n, int m) {
  const int mc = m < kMC ? m : kMC;
  return 3LL * n * mc + (long long)n * (kTile + 1) + kTile;
}

// ---------------------------------------------------------------------------
// k_diag
// ---------------------------------------------------------------------------
template <typename T, bool WITH_Y>
__global__ void __launch_bounds__(256) k_diag(Problem<T> p, Level lv) {
  const int b = blockIdx.x / lv.d;
  const int t = blockIdx.x - b * lv.d;
  if (!p.active(b)) return;
  const int n = p.n, ld = diag_ld(n);
  const int i = lv.s - 1 + 2 * lv.s * t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* A = reinterpret_cast<T*>(smem_raw);
  T* dinv = A + n * ld;
  T* P = dinv + n;
  T* Y = P + n * kDiagBS;

  T* Li = p.Lb(b, i);
  load_block(A, ld, Li, n, n, n);
  __syncthreads();
  cta_chol_inv<T, kDiagBS>(A, ld, n, dinv, P);
  store_block(Li, n, A, ld, n, n);

  if (WITH_Y) {
    T* yi = p.Xb(b, i);
    for (int c0 = 0; c0 < p.m; c0 += kMC) {
      const int mc = min(kMC, p.m - c0);
      __syncthreads();
      load_block(Y, mc, yi + c0, n, mc, p.m);
      __syncthreads();
      // y_i <- W y_i with W = C^{-1}: W[r][k] = A[k*ld + r] (k<r), dinv[r] on the diagonal
      cta_gemm<T, 2, 2, false>(
          n, mc, n,
          [&](int r, int k) { return k < r ? A[k * ld + r] : (k == r ? dinv[r] : T(0)); },
          [&](int k, int c) { return Y[k * mc + c]; },
          [&](int r, int c, T v) { yi[(long long)r * p.m + c0 + c] = v; });
    }
  }
}

// ---------------------------------------------------------------------------
// k_couple
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_couple(Problem<T> p, Level lv) {
  const int n = p.n, ld = diag_ld(n);
  const int np = ceil_div(n, kTile);
  const int per_b = lv.d * 2 * np;
  const int b = blockIdx.x / per_b;
  int rem = blockIdx.x - b * per_b;
  const int t = rem / (2 * np);
  rem -= t * 2 * np;
  const int side = rem / np;        // 0 right, 1 left
  const int pnl = rem - side * np;
  if (!p.active(b)) return;
  const int i = lv.s - 1 + 2 * lv.s * t;
  if (side == 0 && i + lv.s >= p.N) return;
  if (side == 1 && t == 0) return;
  const int p0 = pnl * kTile, pw = min(kTile, n - p0);

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Wt = reinterpret_cast<T*>(smem_raw);   // n x ld, upper triangular = C^{-T}
  T* Pn = Wt + n * ld;                       // panel

  const T* Li = p.Lb(b, i);
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) {
    const int r = e / n, c = e - r * n;
    const T v = Li[e];
    Wt[r * ld + c] = r < c ? v : (r == c ? rcp_t(v) : T(0));
  }
  if (side == 0) {
    T* R = p.Eb(b, lv.oc + 2 * t);
    // rows [p0, p0+pw) of R, all n columns
    load_block(Pn, ld, R + (long long)p0 * n, pw, n, n);
    __syncthreads();
    // F[p0+r][c] = sum_{k<=c} R[p0+r][k] Wt[k][c]
    cta_gemm<T, 2, 2, false>(
        pw, n, n,
        [&](int r, int k) { return Pn[r * ld + k]; },
        [&](int k, int c) { return Wt[k * ld + c]; },
        [&](int r, int c, T v) { R[(long long)(p0 + r) * n + c] = v; });
  } else {
    T* Gs = p.Eb(b, lv.oc + 2 * t - 1);
    // columns [p0, p0+pw) of the slot, all n rows; stored as n x (kTile+1)
    load_block(Pn, kTile + 1, Gs + p0, n, pw, n);
    __syncthreads();
    // G[r][p0+c] = sum_{k<=r} Wt[k][r] Lf[k][p0+c]
    cta_gemm<T, 2, 2, false>(
        n, pw, n,
        [&](int r, int k) { return Wt[k * ld + r]; },
        [&](int k, int c) { return Pn[k * (kTile + 1) + c]; },
        [&](int r, int c, T v) { Gs[(long long)r * n + p0 + c] = v; });
  }
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

template <typename T>
__global__ void __launch_bounds__(256) k_update(Problem<T> p, Level lv) {
  const int n = p.n, N = p.N, s = lv.s;
  const int nt = ceil_div(n, kTile);
  const int nlt = nt * (nt + 1) / 2;
  const int U = N / (2 * s);
  const int nfill = lv.d - 1;
  const int per_b = U * nlt + nfill * nt * nt;
  const int b = blockIdx.x / per_b;
  const int task = blockIdx.x - b * per_b;
  if (!p.active(b)) return;

  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* S0 = reinterpret_cast<T*>(smem_raw);
  const int ldr = n + 1;               // row panels: kTile x (n+1)
  T* Fa = S0;
  T* Fc = Fa + kTile * ldr;
  T* Ga = Fc + kTile * ldr;            // column panels: n x (kTile+1)
  T* Gc = Ga + n * (kTile + 1);

  if (task < U * nlt) {
    const int u = task / nlt + 1;
    int ta, tc;
    lower_tile_index(task - (u - 1) * nlt, ta, tc);
    const int j = 2 * s * u - 1;
    const T* F = p.Eb(b, lv.oc + 2 * (u - 1));
    const bool hasG = j + s < N;
    const T* G = hasG ? p.Eb(b, lv.oc + 2 * u - 1) : nullptr;
    const int ra = ta * kTile, wa = min(kTile, n - ra);
    const int rc = tc * kTile, wc = min(kTile, n - rc);
    load_block(Fa, ldr, F + (long long)ra * n, wa, n, n);
    load_block(Fc, ldr, F + (long long)rc * n, wc, n, n);
    if (hasG) {
      load_block(Ga, kTile + 1, G + ra, n, wa, n);
      load_block(Gc, kTile + 1, G + rc, n, wc, n);
    }
    __syncthreads();
    T* Lj = p.Lb(b, j);
    const int K = hasG ? 2 * n : n;
    auto body = [&](int r, int c, T v) { Lj[(long long)(ra + r) * n + rc + c] -= v; };
    auto fa = [&](int r, int k) { return k < n ? Fa[r * ldr + k] : Ga[(k - n) * (kTile + 1) + r]; };
    auto fb = [&](int k, int c) { return k < n ? Fc[c * ldr + k] : Gc[(k - n) * (kTile + 1) + c]; };
    if (ta == tc)
      cta_gemm<T, 2, 2, true>(wa, wc, K, fa, fb, body);
    else
      cta_gemm<T, 2, 2, false>(wa, wc, K, fa, fb, body);
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
    const int ra = ta * kTile, wa = min(kTile, n - ra);
    const int rc = tc * kTile, wc = min(kTile, n - rc);
    load_block(Fa, ldr, F + (long long)ra * n, wa, n, n);
    load_block(Ga, kTile + 1, G + rc, n, wc, n);
    __syncthreads();
    cta_gemm<T, 2, 2, false>(
        wa, wc, n,
        [&](int r, int k) { return Fa[r * ldr + k]; },
        [&](int k, int c) { return Ga[k * (kTile + 1) + c]; },
        [&](int r, int c, T v) { X[(long long)(ra + r) * n + rc + c] -= v; });
  }
}

// ---------------------------------------------------------------------------
// Sweeps.  Shared layout: Y, Z1, Z2 (n x mc each), Cc (n x (kTile+1)), dv (kTile)
// ---------------------------------------------------------------------------

// Y -= op(M) Z with M an n x n global block, streamed through Cc in kTile
// chunks of the contraction index.  TRANS: out[r][c] = sum_k M[k][r] Z[k][c].
template <typename T, bool TRANS>
__device__ void sweep_accumulate(T* Y, const T* Z, int mc, const T* __restrict__ M, int n, T* Cc) {
  for (int k0 = 0; k0 < n; k0 += kTile) {
    const int kw = min(kTile, n - k0);
    __syncthreads();
    if (TRANS) {
      // rows [k0, k0+kw) of M, stored transposed: Cc[r * (kTile+1) + kk] = M[k0+kk][r]
      for (int e = threadIdx.x; e < kw * n; e += blockDim.x) {
        const int kk = e / n, r = e - kk * n;
        Cc[r * (kTile + 1) + kk] = M[(long long)(k0 + kk) * n + r];
      }
    } else {
      // columns [k0, k0+kw) of M: Cc[r * (kTile+1) + kk] = M[r][k0+kk]
      load_block(Cc, kTile + 1, M + k0, n, kw, n);
    }
    __syncthreads();
    cta_gemm<T, 2, 1, false>(
        n, mc, kw,
        [&](int r, int k) { return Cc[r * (kTile + 1) + k]; },
        [&](int k, int c) { return Z[(k0 + k) * mc + c]; },
        [&](int r, int c, T v) { Y[r * mc + c] -= v; });
  }
  __syncthreads();
}

// Y <- C^{-1} Y (lower C = lower(Lb)), blocked by kTile rows, warp per column.
template <typename T>
__device__ void sweep_lower_solve(T* Y, int mc, const T* __restrict__ Lb, int n, T* Cc, T* dv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int K = 0; K < n; K += kTile) {
    const int kb = min(kTile, n - K);
    __syncthreads();
    // rows [K, K+kb), columns [0, K+kb): Cc[r * (n+1) + c]; reuse Cc with row stride n+1
    // Cc holds n*(kTile+1) >= kb*(n+1) elements.
    const int ldc = n + 1;
    for (int e = threadIdx.x; e < kb * (K + kb); e += blockDim.x) {
      const int r = e / (K + kb), c = e - r * (K + kb);
      Cc[r * ldc + c] = Lb[(long long)(K + r) * n + c];
    }
    __syncthreads();
    if (threadIdx.x < kb) dv[threadIdx.x] = rcp_t(Cc[threadIdx.x * ldc + K + threadIdx.x]);
    __syncthreads();
    for (int c = warp; c < mc; c += nw) {
      T v = lane < kb ? Y[(K + lane) * mc + c] : T(0);
      if (lane < kb)
        for (int k = 0; k < K; ++k) v = fma(-Cc[lane * ldc + k], Y[k * mc + c], v);
      for (int j = 0; j < kb; ++j) {
        const T yj = __shfl_sync(0xffffffffu, v, j) * dv[j];
        if (lane == j) v = yj;
        else if (lane > j && lane < kb) v = fma(-Cc[lane * ldc + K + j], yj, v);
      }
      if (lane < kb) Y[(K + lane) * mc + c] = v;
    }
  }
  __syncthreads();
}

// Y <- C^{-T} Y (lower C = lower(Lb)), blocks from the bottom, warp per column.
template <typename T>
__device__ void sweep_upper_solve(T* Y, int mc, const T* __restrict__ Lb, int n, T* Cc, T* dv) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int last = ((n - 1) / kTile) * kTile;
  for (int K = last; K >= 0; K -= kTile) {
    const int kb = min(kTile, n - K);
    __syncthreads();
    // column panel: rows [K, n), columns [K, K+kb): Cc[(k-K) * (kTile+1) + r] = C[k][K+r]
    load_block(Cc, kTile + 1, Lb + (long long)K * n + K, n - K, kb, n);
    __syncthreads();
    if (threadIdx.x < kb) dv[threadIdx.x] = rcp_t(Cc[threadIdx.x * (kTile + 1) + threadIdx.x]);
    __syncthreads();
    for (int c = warp; c < mc; c += nw) {
      T v = lane < kb ? Y[(K + lane) * mc + c] : T(0);
      if (lane < kb)
        for (int k = K + kb; k < n; ++k) v = fma(-Cc[(k - K) * (kTile + 1) + lane], Y[k * mc + c], v);
      for (int j = kb - 1; j >= 0; --j) {
        const T xj = __shfl_sync(0xffffffffu, v, j) * dv[j];
        if (lane == j) v = xj;
        else if (lane < j) v = fma(-Cc[j * (kTile + 1) + lane], xj, v);
      }
      if (lane < kb) Y[(K + lane) * mc + c] = v;
    }
  }
  __syncthreads();
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwd_node(Problem<T> p, Level lv) {
  const int b = blockIdx.x / lv.d;
  const int t = blockIdx.x - b * lv.d;
  if (!p.active(b)) return;
  const int n = p.n, i = lv.s - 1 + 2 * lv.s * t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int mcmax = min(p.m, kMC);
  T* Y = reinterpret_cast<T*>(smem_raw);
  T* Cc = Y + 3 * n * mcmax;
  T* dv = Cc + n * (kTile + 1);
  T* yi = p.Xb(b, i);
  const T* Li = p.Lb(b, i);
  for (int c0 = 0; c0 < p.m; c0 += kMC) {
    const int mc = min(kMC, p.m - c0);
    __syncthreads();
    load_block(Y, mc, yi + c0, n, mc, p.m);
    sweep_lower_solve(Y, mc, Li, n, Cc, dv);
    store_block(yi + c0, p.m, Y, mc, n, mc);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwd_update(Problem<T> p, Level lv) {
  const int s = lv.s, N = p.N;
  const int U = N / (2 * s);
  const int b = blockIdx.x / U;
  const int u = blockIdx.x - b * U + 1;
  if (!p.active(b)) return;
  const int n = p.n, j = 2 * s * u - 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int mcmax = min(p.m, kMC);
  T* Y = reinterpret_cast<T*>(smem_raw);
  T* Z1 = Y + n * mcmax;
  T* Z2 = Z1 + n * mcmax;
  T* Cc = Z2 + n * mcmax;
  const T* F = p.Eb(b, lv.oc + 2 * (u - 1));
  const bool hasG = j + s < N;
  const T* G = hasG ? p.Eb(b, lv.oc + 2 * u - 1) : nullptr;
  T* yj = p.Xb(b, j);
  for (int c0 = 0; c0 < p.m; c0 += kMC) {
    const int mc = min(kMC, p.m - c0);
    __syncthreads();
    load_block(Y, mc, yj + c0, n, mc, p.m);
    load_block(Z1, mc, p.Xb(b, j - s) + c0, n, mc, p.m);
    if (hasG) load_block(Z2, mc, p.Xb(b, j + s) + c0, n, mc, p.m);
    sweep_accumulate<T, false>(Y, Z1, mc, F, n, Cc);   // Y -= F y_{j-s}
    if (hasG) sweep_accumulate<T, true>(Y, Z2, mc, G, n, Cc);  // Y -= G^T y_{j+s}
    store_block(yj + c0, p.m, Y, mc, n, mc);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_bwd(Problem<T> p, Level lv) {
  const int b = blockIdx.x / lv.d;
  const int t = blockIdx.x - b * lv.d;
  if (!p.active(b)) return;
  const int n = p.n, s = lv.s, N = p.N;
  const int i = s - 1 + 2 * s * t;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int mcmax = min(p.m, kMC);
  T* Y = reinterpret_cast<T*>(smem_raw);
  T* Z1 = Y + n * mcmax;
  T* Z2 = Z1 + n * mcmax;
  T* Cc = Z2 + n * mcmax;
  T* dv = Cc + n * (kTile + 1);
  const bool right = i + s < N, left = i >= s;
  const T* F = right ? p.Eb(b, lv.oc + 2 * t) : nullptr;
  const T* G = left ? p.Eb(b, lv.oc + 2 * t - 1) : nullptr;
  T* xi = p.Xb(b, i);
  for (int c0 = 0; c0 < p.m; c0 += kMC) {
    const int mc = min(kMC, p.m - c0);
    __syncthreads();
    load_block(Y, mc, xi + c0, n, mc, p.m);
    if (right) load_block(Z1, mc, p.Xb(b, i + s) + c0, n, mc, p.m);
    if (left) load_block(Z2, mc, p.Xb(b, i - s) + c0, n, mc, p.m);
    if (right) sweep_accumulate<T, true>(Y, Z1, mc, F, n, Cc);   // Y -= F^T x_{i+s}
    if (left) sweep_accumulate<T, false>(Y, Z2, mc, G, n, Cc);   // Y -= G x_{i-s}
    sweep_upper_solve(Y, mc, p.Lb(b, i), n, Cc, dv);
    store_block(xi + c0, p.m, Y, mc, n, mc);
  }
}

}  // namespace socu
