// Mixed-precision factorisation with FP64 iterative refinement.
//
// The FP64 problem (L, E, b) is left untouched.  A float copy of (L, E) is
// factored with the same nested-dissection kernels; then
//     x = 0, r = b
//     repeat: delta = solve32(r); x += delta; r = b - Psi x (FP64);
//             eta = ||r||_inf / (||Psi||_inf ||x||_inf + ||b||_inf)
//     until eta <= tol (per instance) or max_iter
// Converged instances drop out of every later kernel through the per-instance
// `active` flags, which the solver kernels take as their batch mask.
#pragma once

#include "nd_kernels.cuh"

namespace socu {

// Per-instance refinement state, in the caller's workspace.
struct RefineState {
  unsigned long long psi;   // ||Psi||_inf bits (non-negative doubles order like uint64)
  unsigned long long bnorm; // ||b||_inf bits
  unsigned long long rnorm; // ||r||_inf bits, accumulated per iteration
  unsigned long long xnorm; // ||x||_inf bits, accumulated per iteration
  unsigned done;            // residual CTAs of this round that have added their norms
  unsigned pad;
};

struct RefineArgs {
  const double* L;   // (B, N, n, n) original diagonal blocks (lower read)
  const double* E;   // (B, S, n, n) original off-diagonal storage (slots < N-1 read)
  const double* b;   // (B, N, n, m)
  double* x;         // (B, N, n, m) solution
  const uint8_t* mask;
  float* L32;
  float* E32;
  float* R32;        // (B, N, n, m) residual in / correction out
  uint8_t* active;
  RefineState* st;
  double* eta;       // (B,) last backward error
  int* iters;        // (B,) iterations performed
  int* any_active;   // 1 while some instance still iterates
  double* rout;      // plain residual output (k_residual<false>), else unused
  int B, N, n, m, S;
  double tol;
  int max_iter;
  int check_in_residual;   // 1: the residual's last CTA per instance also runs the convergence test
};

__device__ __forceinline__ void atomic_max_pos(unsigned long long* a, double v) {
  atomicMax(a, static_cast<unsigned long long>(__double_as_longlong(v)));
}

__device__ __forceinline__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(kFull, v, o));
  }
  return v;  // valid in thread 0
}

// Per-instance state reset (before k_ref_init accumulates into it).
__global__ void k_ref_reset(RefineArgs a) {
  pdl_wait();
  pdl_trigger();
  for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < a.B; bi += gridDim.x * blockDim.x) {
    const bool on = a.mask == nullptr || a.mask[bi] != 0;
    a.active[bi] = on ? 1 : 0;
    a.iters[bi] = 0;
    a.eta[bi] = on ? __longlong_as_double(0x7ff0000000000000LL) : 0.0;
    a.st[bi].psi = 0ull;
    a.st[bi].bnorm = 0ull;
    a.st[bi].rnorm = 0ull;
    a.st[bi].xnorm = 0ull;
    a.st[bi].done = 0u;
    if (on) atomicExch(a.any_active, 1);
  }
}

// One CTA per (instance, block index i < max(N, S)): float copies of L_i and
// slot i, R32 = b, x = 0, ||Psi||_inf and ||b||_inf contributions of block row i.
__device__ __forceinline__ void ref_init_body(const RefineArgs& a, int bi, int i) {
  __shared__ double red[32];
  const int n = a.n, m = a.m;
  const long long nn = (long long)n * n;
  if (i < a.N) {
    const double* Li = a.L + ((long long)bi * a.N + i) * nn;
    float* L32 = a.L32 + ((long long)bi * a.N + i) * nn;
    for (long long e = threadIdx.x; e < nn; e += blockDim.x) L32[e] = (float)Li[e];
  }
  if (i < a.S) {
    const long long off = ((long long)bi * a.S + i) * nn;
    float* E32 = a.E32 + off;
    if (i < a.N - 1) {
      for (long long e = threadIdx.x; e < nn; e += blockDim.x) E32[e] = (float)a.E[off + e];
    } else {
      for (long long e = threadIdx.x; e < nn; e += blockDim.x) E32[e] = 0.0f;
    }
  }
  if (i >= a.N) return;
  const long long vo = ((long long)bi * a.N + i) * n * m;
  double bmax = 0.0;
  for (int e = threadIdx.x; e < n * m; e += blockDim.x) {
    const double v = a.b[vo + e];
    a.R32[vo + e] = (float)v;
    a.x[vo + e] = 0.0;
    bmax = fmax(bmax, fabs(v));
  }
  // row sums of |Psi| over block row i: lower-symmetric D_i, E_{i-1} rows, E_i columns
  const double* Li = a.L + ((long long)bi * a.N + i) * nn;
  const double* Em = i > 0 ? a.E + ((long long)bi * a.S + i - 1) * nn : nullptr;
  const double* Ei = i < a.N - 1 ? a.E + ((long long)bi * a.S + i) * nn : nullptr;
  double rmax = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    double sum = 0.0;
    for (int c = 0; c < n; ++c) sum += fabs(c <= r ? Li[(long long)r * n + c] : Li[(long long)c * n + r]);
    if (Em)
      for (int c = 0; c < n; ++c) sum += fabs(Em[(long long)r * n + c]);
    if (Ei)
      for (int c = 0; c < n; ++c) sum += fabs(Ei[(long long)c * n + r]);
    rmax = fmax(rmax, sum);
  }
  const double bm = block_max(bmax, red);
  const double pm = block_max(rmax, red);
  if (threadIdx.x == 0) {
    atomic_max_pos(&a.st[bi].bnorm, bm);
    atomic_max_pos(&a.st[bi].psi, pm);
  }
}

__global__ void __launch_bounds__(256) k_ref_init(RefineArgs a) {
  pdl_wait();
  pdl_trigger();
  const int per = a.N > a.S ? a.N : a.S;
  const int bi = blockIdx.x / per;
  const int i = blockIdx.x - bi * per;
  if (a.mask != nullptr && a.mask[bi] == 0) return;
  ref_init_body(a, bi, i);
}


// r = b - Psi x for rows [r0, r0+32) of block row i (FP64 against the
// original blocks), R32 = float(r), ||r||_inf and ||x||_inf accumulated.
// Shared: Lr (32 x ldn) rows of L_i, Lc (n x 33) column panel of L_i,
// Er (32 x ldn) rows of E_{i-1}, Ec (n x 33) columns of E_i, X (3 x n x ldx).
constexpr int kResRows = 32;
constexpr int kResCols = 16;
__host__ __device__ inline long long smem_residual_elems(int n) {
  return 2LL * kResRows * (n + 1) + 2LL * n * (kResRows + 1) + 3LL * n * (kResCols + 1);
}

// REFINE: write R32 = float(r), accumulate norms, skip inactive instances.
// Otherwise write r (double) to a.rout for every instance.
// x += delta (R32) for active instances; grid-stride over the whole batch.
__global__ void __launch_bounds__(256) k_ref_update(RefineArgs a) {
  pdl_wait();
  pdl_trigger();
  const long long per = (long long)a.N * a.n * a.m;
  const long long total = (long long)a.B * per;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int bi = (int)(e / per);
    if (a.active[bi]) a.x[e] += (double)a.R32[e];
  }
}

// Convergence test of instance bi; clears the accumulators for the next
// round.  A non-finite eta (numerical breakdown of the float factor) stops the
// instance with iters = -(iterations done).
__device__ __forceinline__ void ref_check_instance(const RefineArgs& a, int bi) {
  RefineState& s = a.st[bi];
  // norms other CTAs added with atomics: read them the same way
  const double rn = __longlong_as_double((long long)atomicAdd(&s.rnorm, 0ull));
  const double xn = __longlong_as_double((long long)atomicAdd(&s.xnorm, 0ull));
  const double pn = __longlong_as_double((long long)s.psi);
  const double bn = __longlong_as_double((long long)s.bnorm);
  const double den = pn * xn + bn;
  const double eta = den > 0.0 ? rn / den : 0.0;
  const int it = a.iters[bi] + 1;
  a.iters[bi] = it;
  a.eta[bi] = eta;
  s.rnorm = 0ull;
  s.xnorm = 0ull;
  if (!(eta == eta) || isinf(eta)) {
    a.active[bi] = 0;
    a.iters[bi] = -it;
  } else if (eta <= a.tol || it >= a.max_iter) {
    a.active[bi] = 0;
  } else {
    atomicExch(a.any_active, 1);
  }
}

// check_in_residual: thread 0 of every residual CTA of an active instance,
// after its norms: the CTA that completes the instance's count runs the test
// (and rearms the count), so no separate test launch follows the residual.
__device__ __forceinline__ void residual_arrive(const RefineArgs& a, int bi, unsigned ctas) {
  if (!a.check_in_residual || threadIdx.x != 0) return;
  __threadfence();
  if (atomicAdd(&a.st[bi].done, 1u) + 1u == ctas) {
    __threadfence();
    ref_check_instance(a, bi);
    a.st[bi].done = 0u;
  }
}

template <bool REFINE>
__device__ __forceinline__ void residual_body(const RefineArgs& a, int bi, int i, int r0, unsigned char* smem_raw) {
  const int n = a.n, m = a.m, N = a.N;
  const int rw = min(kResRows, n - r0);
  const int ldn = n + 1, ldc = kResRows + 1, ldx = kResCols + 1;
  double* Lr = reinterpret_cast<double*>(smem_raw);
  double* Er = Lr + kResRows * ldn;
  double* Lc = Er + kResRows * ldn;
  double* Ec = Lc + n * ldc;
  double* X0 = Ec + n * ldc;   // x_{i-1}
  double* X1 = X0 + n * ldx;   // x_i
  double* X2 = X1 + n * ldx;   // x_{i+1}
  __shared__ double red[32];
  const long long nn = (long long)n * n;
  const double* Li = a.L + ((long long)bi * N + i) * nn;
  const bool hasm = i > 0, hasp = i < N - 1;
  const double* Em = hasm ? a.E + ((long long)bi * a.S + i - 1) * nn : nullptr;
  const double* Ei = hasp ? a.E + ((long long)bi * a.S + i) * nn : nullptr;
  async_load(Lr, ldn, Li + (long long)r0 * n, rw, n, n);
  async_load(Lc, ldc, Li + r0, n, rw, n);
  if (hasm) async_load(Er, ldn, Em + (long long)r0 * n, rw, n, n);
  if (hasp) async_load(Ec, ldc, Ei + r0, n, rw, n);
  const long long vi = ((long long)bi * N + i) * n * m;
  double rmax = 0.0, xmax = 0.0;
  for (int c0 = 0; c0 < m; c0 += kResCols) {
    const int mc = min(kResCols, m - c0);
    __syncthreads();
    async_load(X1, ldx, a.x + vi + c0, n, mc, m);
    if (hasm) async_load(X0, ldx, a.x + vi - (long long)n * m + c0, n, mc, m);
    if (hasp) async_load(X2, ldx, a.x + vi + (long long)n * m + c0, n, mc, m);
    cp_async_wait_all();
    __syncthreads();
    for (int o = threadIdx.x; o < rw * mc; o += blockDim.x) {
      const int rr = o / mc, c = o - rr * mc, r = r0 + rr;
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
      // D_i x_i with D symmetric from lower(L_i): k <= r from row r, k > r from column r
      for (int k = 0; k <= r; ++k) s0 = fma(Lr[rr * ldn + k], X1[k * ldx + c], s0);
      for (int k = r + 1; k < n; ++k) s0 = fma(Lc[k * ldc + rr], X1[k * ldx + c], s0);
      if (hasm)
        for (int k = 0; k < n; ++k) s1 = fma(Er[rr * ldn + k], X0[k * ldx + c], s1);
      if (hasp)
        for (int k = 0; k < n; ++k) s2 = fma(Ec[k * ldc + rr], X2[k * ldx + c], s2);
      const long long e = vi + (long long)r * m + c0 + c;
      const double res = a.b[e] - (s0 + s1 + s2);
      if (REFINE) {
        a.R32[e] = (float)res;
        const double xv = X1[r * ldx + c];
        // non-finite values poison the norms (fmax alone would drop a NaN)
        rmax = isfinite(res) ? fmax(rmax, fabs(res)) : __longlong_as_double(0x7ff0000000000000LL);
        xmax = isfinite(xv) ? fmax(xmax, fabs(xv)) : __longlong_as_double(0x7ff0000000000000LL);
      } else {
        a.rout[e] = res;
      }
    }
  }
  if (REFINE) {
    const double rm = block_max(rmax, red);
    const double xm = block_max(xmax, red);
    if (threadIdx.x == 0) {
      atomic_max_pos(&a.st[bi].rnorm, rm);
      atomic_max_pos(&a.st[bi].xnorm, xm);
    }
  }
}

template <bool REFINE>
__global__ void __launch_bounds__(256) k_residual(RefineArgs a) {
  pdl_wait();
  pdl_trigger();
  const int nrc = (a.n + kResRows - 1) / kResRows;
  const int per = a.N * nrc;
  const int bi = blockIdx.x / per;
  const int rem = blockIdx.x - bi * per;
  const int i = rem / nrc;
  if (REFINE && !a.active[bi]) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  residual_body<REFINE>(a, bi, i, (rem - i * nrc) * kResRows, smem_raw);
  if (REFINE) residual_arrive(a, bi, (unsigned)per);
}

// ---------------------------------------------------------------------------
// Block-row kernels for n <= kResRowMaxN: one CTA per block row i reads the
// three blocks of that row, L_i, E_{i-1} and E_i, with coalesced loads
// (missing neighbours as zeros), so every element of L and E is read from HBM
// once per row that needs it (and per 32 right-hand sides).
// ---------------------------------------------------------------------------
constexpr int kResRowMaxN = 128;
__host__ __device__ inline bool residual_uses_rows(int n) { return n <= kResRowMaxN; }

// r_i = b_i - (D_i x_i + E_{i-1} x_{i-1} + E_i^T x_{i+1}) for the whole block
// row, on FP64 tensor cores (mma.m8n8k4 .f64).  Per super-chunk of up to 32
// right-hand sides the CTA stages x_{i-1}, x_i, x_{i+1} in shared memory
// (stride 36: conflict-free B fragments; missing neighbours and columns as
// zeros); the matrix fragments are read straight from global memory, each
// element once per super-chunk, and multiplied into all (up to four) 8-column
// groups of the chunk.  Warp task = one 8-row output tile: 3 blocks x
// ceil(n/4) k-steps into independent accumulators (block x k parity x column
// group).  Fragment layout: a0 = A[g][t], b0 = B[t][g], {c0, c1} = C[g][2t +
// {0, 1}] (g = lane / 4, t = lane % 4).  D_i is symmetric from its lower
// triangle: above the diagonal the transposed element is read.  Any
// blockDim.x that is a multiple of 32 works.
// Shared: 3 x n x kResXld doubles (smem_residual_x_elems).
// GR = 8-column groups per super-chunk (1, 2 or 4, by the number of
// right-hand sides): the super-chunk is 8 GR columns wide, staged with stride
// 8 GR + 4 doubles (4 mod 16 for GR = 1 and 4; 20 for GR = 2).
__host__ __device__ inline int residual_groups(int m) { return m <= 8 ? 1 : (m <= 16 ? 2 : 4); }
__host__ __device__ inline long long smem_residual_x_elems(int n, int gr) { return 3LL * n * (8 * gr + 4); }
// shared memory the ragged kernel reserves for its residual / set-up phases
// (doubles): the one-group residual's x staging, which exceeds the set-up's 17 n
__host__ __device__ inline long long smem_residual_rows_elems(int n) { return smem_residual_x_elems(n, 1); }
template <bool REFINE, int GR>
__device__ __forceinline__ void residual_rows_body(const RefineArgs& a, int bi, int i, unsigned char* smem_raw) {
  constexpr int kResXC = 8 * GR, kResXld = kResXC + 4;
  __shared__ double red[32];
  double* const xs0 = reinterpret_cast<double*>(smem_raw);
  const int xstride = a.n * kResXld;   // x_{i-1}, x_i, x_{i+1} chunks back to back
  const int n = a.n, m = a.m, N = a.N;
  const long long nn = (long long)n * n;
  const double* D = a.L + ((long long)bi * N + i) * nn;
  const bool hasM = i > 0, hasP = i < N - 1;
  const double* Em = a.E + ((long long)bi * a.S + (hasM ? i - 1 : 0)) * nn;
  const double* Ep = a.E + ((long long)bi * a.S + (hasP ? i : 0)) * nn;
  const long long vi = ((long long)bi * N + i) * n * m;
  const double* x1 = a.x + vi;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int rts = (n + 7) >> 3;
  double rmax = 0.0, xmax = 0.0;
  for (int c0 = 0; c0 < m; c0 += kResXC) {
    const int mc = min(kResXC, m - c0);
    const int groups = (mc + 7) >> 3;
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * n * kResXC; e += blockDim.x) {
      const int j = e / (n * kResXC), rem = e - j * n * kResXC, k = rem / kResXC, c = rem - k * kResXC;
      const bool ok = c < mc && (j == 1 || (j == 0 ? hasM : hasP));
      xs0[j * xstride + k * kResXld + c] = ok ? x1[(long long)(j - 1) * n * m + (long long)k * m + c0 + c] : 0.0;
    }
    __syncthreads();
    for (int rt = warp; rt < rts; rt += nw) {
      const int r0 = rt * 8, ra = r0 + g;
      const bool rv = ra < n;
      const int rr = rv ? ra : 0;
      // accumulators per column group: block (D, E_{i-1}, E_i) x k-step parity
      // (KP = 2 independent chains per block when there is one group; several
      // groups already give the MMAs independent chains, and registers are short)
      constexpr int KP = GR >= 2 ? 1 : 2;
      double acc[GR][3 * KP][2];
#pragma unroll
      for (int q = 0; q < GR; ++q)
#pragma unroll
        for (int u = 0; u < 3 * KP; ++u) acc[q][u][0] = acc[q][u][1] = 0.0;
      // matrix fragments of one 8-column k-step (two m8n8k4 steps), loaded one
      // k-step ahead of their products so the global loads overlap the MMAs
      double fD[2], fM[2], fP[2];
      auto load_step = [&](int k0) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k = k0 + 4 * h + t;
          const bool kv = k < n;
          const int kk = kv ? k : 0;
          const bool av = rv && kv;
          const double dv = kk <= rr ? D[rr * n + kk] : D[kk * n + rr];
          fD[h] = av ? dv : 0.0;
          fM[h] = (av && hasM) ? Em[rr * n + kk] : 0.0;
          fP[h] = (av && hasP) ? Ep[kk * n + rr] : 0.0;
        }
      };
      load_step(0);
      for (int k0 = 0; k0 < n; k0 += 8) {
        const double cD[2] = {fD[0], fD[1]}, cM[2] = {fM[0], fM[1]}, cP[2] = {fP[0], fP[1]};
        if (k0 + 8 < n) load_step(k0 + 8);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int k = k0 + 4 * h + t;
          const bool kv = k < n;
          const int kk = kv ? k : 0;
#pragma unroll
          for (int q = 0; q < GR; ++q) {
            if (q >= groups) break;
            const int xo = kk * kResXld + 8 * q + g;
            const double b1 = kv ? xs0[xstride + xo] : 0.0;
            const double b0 = kv ? xs0[xo] : 0.0;
            const double b2 = kv ? xs0[2 * xstride + xo] : 0.0;
            const int u = KP == 2 ? h : 0;
            dmma_8x8x4(acc[q][u][0], acc[q][u][1], cD[h], b1);
            dmma_8x8x4(acc[q][KP + u][0], acc[q][KP + u][1], cM[h], b0);
            dmma_8x8x4(acc[q][2 * KP + u][0], acc[q][2 * KP + u][1], cP[h], b2);
          }
        }
      }
#pragma unroll
      for (int q = 0; q < GR; ++q) {
        if (q >= groups) break;
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int r = r0 + g, c = 8 * q + 2 * t + e;
          if (r < n && c < mc) {
            const long long o = vi + (long long)r * m + c0 + c;
            double y = 0.0;
#pragma unroll
            for (int u = 0; u < 3 * KP; ++u) y += acc[q][u][e];
            const double res = a.b[o] - y;
            if (REFINE) {
              a.R32[o] = (float)res;
              const double xv = xs0[xstride + r * kResXld + c];
              rmax = isfinite(res) ? fmax(rmax, fabs(res)) : __longlong_as_double(0x7ff0000000000000LL);
              xmax = isfinite(xv) ? fmax(xmax, fabs(xv)) : __longlong_as_double(0x7ff0000000000000LL);
            } else {
              a.rout[o] = res;
            }
          }
        }
      }
    }
  }
  if (REFINE) {
    const double rm = block_max(rmax, red);
    const double xm = block_max(xmax, red);
    if (threadIdx.x == 0) {
      atomic_max_pos(&a.st[bi].rnorm, rm);
      atomic_max_pos(&a.st[bi].xnorm, xm);
    }
  }
}

// (at most 256: warps loop over the 8-row tiles of larger blocks)
__host__ __device__ inline int residual_rows_threads(int n, int) {
  const int t = 32 * ((n + 7) / 8);
  return t < 256 ? t : 256;
}

template <bool REFINE, int GR>
__global__ void __launch_bounds__(256, GR == 4 ? 2 : 3) k_residual_rows(RefineArgs a) {
  pdl_wait();
  pdl_trigger();
  const int bi = blockIdx.x / a.N;
  const int i = blockIdx.x - bi * a.N;
  if (REFINE && !a.active[bi]) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  residual_rows_body<REFINE, GR>(a, bi, i, smem_raw);
  if (REFINE) residual_arrive(a, bi, (unsigned)a.N);
}

// Refinement set-up for block row i (if i < N) and storage slot i (if i < S):
// float copies of L_i and slot i, R32 = b_i, x_i = 0, ||b||_inf and the row
// sums of |Psi| over block row i.  One streaming pass, no staging: warp w
// takes rows w, w + nw, ... of L_i, E_{i-1} and E_i with coalesced loads
// (lane owns columns lane, lane + 32, ...), writes the float copies, reduces
// the row part of each row sum (lower(D) row, E_{i-1} row) with shuffles and
// keeps per-lane column partials for the transposed parts (strict lower(D)
// columns, E_i columns).  The warps' column partials are added in warp order
// in shared memory (smem_ref_init_elems doubles), so the sums are deterministic.
__host__ __device__ inline long long smem_ref_init_elems(int n) { return 2LL * 8 * n + n; }
__device__ __forceinline__ void ref_init_rows_body(const RefineArgs& a, int bi, int i, unsigned char* smem_raw) {
  __shared__ double red[32];
  const int n = a.n, m = a.m, N = a.N;
  const long long nn = (long long)n * n;
  if (i >= N) {   // storage tail: zero slots only
    if (i < a.S) {
      float* E32 = a.E32 + ((long long)bi * a.S + i) * nn;
      for (long long e = threadIdx.x; e < nn; e += blockDim.x) E32[e] = 0.0f;
    }
    return;
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* colp = reinterpret_cast<double*>(smem_raw);   // [warp][2][n] column partials
  double* rs = colp + 2 * 8 * n;                         // [n] row parts
  const bool hasM = i > 0, hasP = i < N - 1, hasS = i < a.S;
  const double* Lg = a.L + ((long long)bi * N + i) * nn;
  const double* Em = a.E + ((long long)bi * a.S + (hasM ? i - 1 : 0)) * nn;
  const double* Ep = a.E + ((long long)bi * a.S + (hasP ? i : 0)) * nn;
  float* L32 = a.L32 + ((long long)bi * N + i) * nn;
  float* E32 = a.E32 + ((long long)bi * a.S + (hasS ? i : 0)) * nn;
  const long long vo = ((long long)bi * N + i) * n * m;
  double bmax = 0.0;
  for (int e = threadIdx.x; e < n * m; e += blockDim.x) {
    const double v = a.b[vo + e];
    a.R32[vo + e] = (float)v;
    a.x[vo + e] = 0.0;
    bmax = fmax(bmax, fabs(v));
  }
  constexpr int H = kResRowMaxN / 32;   // columns per lane
  double cl[H], ce[H];
#pragma unroll
  for (int h = 0; h < H; ++h) cl[h] = ce[h] = 0.0;
  for (int r = warp; r < n; r += nw) {
    double vl[H], vm[H], vp[H];
#pragma unroll
    for (int h = 0; h < H; ++h) {
      const int c = lane + 32 * h;
      const bool ok = c < n;
      const int o = r * n + (ok ? c : 0);
      vl[h] = ok ? Lg[o] : 0.0;
      vm[h] = (ok && hasM) ? Em[o] : 0.0;
      vp[h] = (ok && hasP) ? Ep[o] : 0.0;
    }
    double part = 0.0;
#pragma unroll
    for (int h = 0; h < H; ++h) {
      const int c = lane + 32 * h;
      if (c < n) {
        L32[r * n + c] = (float)vl[h];
        if (hasS) E32[r * n + c] = (float)vp[h];
        part += (c <= r ? fabs(vl[h]) : 0.0) + fabs(vm[h]);
        cl[h] += c < r ? fabs(vl[h]) : 0.0;   // D(c, r) = L[r][c] for r > c: row c's transposed part
        ce[h] += fabs(vp[h]);                 // E_i^T couples row c to x_{i+1}: column sums of E_i
      }
    }
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(kFull, part, o);
    if (lane == 0) rs[r] = part;
  }
#pragma unroll
  for (int h = 0; h < H; ++h) {
    const int c = lane + 32 * h;
    if (c < n) {
      colp[(warp * 2 + 0) * n + c] = cl[h];
      colp[(warp * 2 + 1) * n + c] = ce[h];
    }
  }
  __syncthreads();
  double rmax = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    double sum = rs[r];
    for (int w = 0; w < nw; ++w) sum += colp[(w * 2 + 0) * n + r] + colp[(w * 2 + 1) * n + r];
    rmax = fmax(rmax, sum);
  }
  const double bm = block_max(bmax, red);
  const double pm = block_max(rmax, red);
  if (threadIdx.x == 0) {
    atomic_max_pos(&a.st[bi].bnorm, bm);
    atomic_max_pos(&a.st[bi].psi, pm);
  }
}

__global__ void __launch_bounds__(256) k_ref_init_rows(RefineArgs a) {
  pdl_wait();
  pdl_trigger();
  const int per = a.N > a.S ? a.N : a.S;
  const int bi = blockIdx.x / per;
  const int i = blockIdx.x - bi * per;
  if (a.mask != nullptr && a.mask[bi] == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  ref_init_rows_body(a, bi, i, smem_raw);
}

// ---------------------------------------------------------------------------
// FP64 fallback after refinement (graph-captured solve only).  Instances whose
// refinement did not reach tol -- it stalled, ran out of rounds, or the float
// factor broke down -- are solved again by the plain FP64 factor_and_solve on
// working copies of their original blocks, inside a conditional IF node that
// runs only when some instance needs it.
// ---------------------------------------------------------------------------
struct FallbackArgs {
  double* L64;     // (B, N, n, n) FP64 working copy of L
  double* E64;     // (B, S, n, n) FP64 working copy of E (slots >= N-1 zero)
  uint8_t* fb;     // per instance: solved again in FP64 (the FP64 solve's batch mask)
  int* any;        // 1 when some instance is in fb
  uint8_t* used;   // caller output (B,): 1 where x comes from the FP64 path
};

__global__ void k_fb_select(RefineArgs a, FallbackArgs f) {
  for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < a.B; bi += gridDim.x * blockDim.x) {
    const bool on = a.mask == nullptr || a.mask[bi] != 0;
    const bool fail = on && !(a.eta[bi] <= a.tol);
    f.fb[bi] = fail ? 1 : 0;
    f.used[bi] = fail ? 1 : 0;
    if (fail) atomicExch(f.any, 1);
  }
}

// IF-node condition: run the FP64 stage when some instance needs it.
__global__ void k_fb_decide(cudaGraphConditionalHandle h, int* any) {
  const int v = *any;
  *any = 0;
  cudaGraphSetConditional(h, v ? 1u : 0u);
}

// One CTA per (instance, block index i < max(N, S)) of the selected
// instances: FP64 copies of L_i and slot i (zero for slots >= N-1), x_i = b_i.
__global__ void __launch_bounds__(256) k_fb_copy(RefineArgs a, FallbackArgs f) {
  const int per = a.N > a.S ? a.N : a.S;
  const int bi = blockIdx.x / per;
  const int i = blockIdx.x - bi * per;
  if (!f.fb[bi]) return;
  const long long nn = (long long)a.n * a.n;
  if (i < a.N) {
    const long long o = ((long long)bi * a.N + i) * nn;
    for (long long e = threadIdx.x; e < nn; e += blockDim.x) f.L64[o + e] = a.L[o + e];
    const long long v = ((long long)bi * a.N + i) * a.n * a.m;
    for (long long e = threadIdx.x; e < (long long)a.n * a.m; e += blockDim.x) a.x[v + e] = a.b[v + e];
  }
  if (i < a.S) {
    const long long o = ((long long)bi * a.S + i) * nn;
    if (i < a.N - 1) {
      for (long long e = threadIdx.x; e < nn; e += blockDim.x) f.E64[o + e] = a.E[o + e];
    } else {
      for (long long e = threadIdx.x; e < nn; e += blockDim.x) f.E64[o + e] = 0.0;
    }
  }
}

// Backward error of the FP64 solution (norms accumulated by the residual
// kernel with fb as its instance mask).
__global__ void k_fb_eta(RefineArgs a, FallbackArgs f) {
  for (int bi = blockIdx.x * blockDim.x + threadIdx.x; bi < a.B; bi += gridDim.x * blockDim.x) {
    if (!f.fb[bi]) continue;
    RefineState& s = a.st[bi];
    const double rn = __longlong_as_double((long long)s.rnorm);
    const double xn = __longlong_as_double((long long)s.xnorm);
    const double pn = __longlong_as_double((long long)s.psi);
    const double bn = __longlong_as_double((long long)s.bnorm);
    const double den = pn * xn + bn;
    a.eta[bi] = den > 0.0 ? rn / den : 0.0;
    s.rnorm = 0ull;
    s.xnorm = 0ull;
  }
}

// Loop control for a graph WHILE node: keep iterating while some instance
// is still active, and clear the flag for the next round.
__global__ void k_ref_decide(cudaGraphConditionalHandle h, int* any_active) {
  const int v = *any_active;
  *any_active = 0;
  cudaGraphSetConditional(h, v ? 1u : 0u);
}

}  // namespace socu
