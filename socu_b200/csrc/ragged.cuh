// Ragged batches: many independent block-tridiagonal systems of different
// horizon N, block size n and right-hand-side count m, solved by ONE
// persistent launch that pulls (instance, phase, chunk) tasks from a device
// work queue.
//
// Every instance walks a fixed sequence of phases; a phase is a set of units
// (level nodes, update targets, sweep nodes, residual row panels), cut into
// chunks of `upc` units.  The units of one phase are independent; a phase may
// start only when the previous phase of the same instance has finished:
//
//   plain factor_and_solve (T = float or double), K separator levels:
//     NODE 0, UPD 0, NODE 1, UPD 1, ..., NODE K-1, BWD K-1, ..., BWD 0
//   mixed refinement (T = float factor of an FP64 problem):
//     INIT, then the plain phases on the float copy with y = b (the first
//     round fused into the factor), XUPD (x += delta), RES (FP64 residual and
//     eta); every further round is FWD 0..K-1, BWD K-1..0, XUPD, RES, until
//     eta <= tol, max_iter rounds, or a non-finite eta.
//
// NODE/UPD/FWD/BWD/RES run the same device bodies as the per-level kernels of
// the uniform batch (nd_kernels.cuh, refine.cuh), so each output block has one
// writer and the results do not depend on the task order.  UPD of the plain
// path also applies the fused forward pull of the next level (the uniform
// factor_and_solve launches it separately).
//
// Queue protocol (thread 0 of a CTA acts for the CTA):
//   pop:      k = atomicAdd(head, 1); wait until slot[k] holds a task, or all
//             instances are done (then exit); a wait that sees no queue
//             progress for timeout_ns (%globaltimer) records an error and exits.
//   complete: fence; if atomicSub(rem[inst], 1) == 1 the phase is over: fence,
//             set rem for the next phase, push its chunks 1..c-1 and keep
//             chunk 0 for this CTA (an instance's critical path never waits
//             in the queue).  The last phase increments `done`.
// Tasks never wait on one another, only on the queue, so the protocol cannot
// deadlock whether or not every CTA is resident.
#pragma once

#include "refine.cuh"

namespace socu {

struct RgInst {
  long long oL, oE, oX;   // element offsets of the instance in the packed L, E and x arrays
  int N, n, m, S;
  int K;                  // separator levels
  int upc;                // units per chunk
};

enum RgMode { kRgPlain = 0, kRgRefine = 1 };
enum RgKind { kRgNode = 0, kRgUpd, kRgBwd, kRgFwd, kRgInit, kRgXupd, kRgRes };

struct RgPhase {
  int kind, level, units, upc;
};

constexpr unsigned long long kRgValid = 1ull << 63;
constexpr unsigned long long kRgExit = ~0ull;
constexpr int kRgInstBits = 24, kRgPhaseBits = 16, kRgChunkBits = 23;

__host__ __device__ inline unsigned long long rg_encode(int inst, int ph, int chunk) {
  return kRgValid | ((unsigned long long)inst << (kRgPhaseBits + kRgChunkBits)) |
         ((unsigned long long)ph << kRgChunkBits) | (unsigned long long)chunk;
}
__host__ __device__ inline void rg_decode(unsigned long long t, int& inst, int& ph, int& chunk) {
  chunk = (int)(t & ((1ull << kRgChunkBits) - 1));
  ph = (int)((t >> kRgChunkBits) & ((1ull << kRgPhaseBits) - 1));
  inst = (int)((t >> (kRgPhaseBits + kRgChunkBits)) & ((1ull << kRgInstBits) - 1));
}

// Level l of the separator schedule of a horizon-N system
// (socu/block_tridiag_solver.py:869-914).
__host__ __device__ inline Level rg_level(int N, int l) {
  int s = 1, prev = 0, curr = 0, nxt = N - 1;
  for (int k = 0; k < l; ++k) {
    s *= 2;
    prev = curr;
    curr = nxt;
    nxt += N / s - 1;
  }
  Level lv;
  lv.s = s;
  lv.d = (N + s) / (2 * s);
  lv.oc = curr;
  lv.on = nxt;
  lv.op = prev;
  lv.tc = 0;       // persistent CTAs: SIMT sweep products (lower latency per node)
  lv.tile = 32;    // unused (n <= 64: whole-block updates)
  lv.pre = 0;      // no programmatic launches in the persistent kernel
  return lv;
}

// Phases of the plain path; the refinement path is unbounded (decided on the device).
__host__ __device__ inline int rg_plain_phases(int K) { return 3 * K - 1; }
// Phases of the refinement path with `rounds` refinement rounds.
__host__ __device__ inline int rg_refine_phases(int K, int rounds) { return 3 * K + 2 + (rounds - 1) * (2 * K + 2); }

__host__ __device__ inline RgPhase rg_phase(const RgInst& I, int mode, int ph) {
  const int K = I.K;
  RgPhase r;
  r.upc = I.upc;
  int f = ph;
  if (mode == kRgRefine) {
    if (ph == 0) {
      r.kind = kRgInit;
      r.level = 0;
      r.units = I.N > I.S ? I.N : I.S;
      r.upc = 2 * I.upc;
      return r;
    }
    f = ph - 1;
  }
  if (f < 2 * K - 1) {
    r.level = f >> 1;
    const Level lv = rg_level(I.N, r.level);
    if ((f & 1) == 0) {
      r.kind = kRgNode;
      r.units = lv.d;
    } else {
      r.kind = kRgUpd;
      r.units = I.N / (2 * lv.s);
    }
    return r;
  }
  f -= 2 * K - 1;
  if (mode == kRgPlain || f < K) {
    r.kind = kRgBwd;
    r.level = K - 1 - f;
    r.units = rg_level(I.N, r.level).d;
    return r;
  }
  // refinement: XUPD and RES of the first round, then whole rounds
  f -= K;
  const int q = f < 2 ? 2 * K + f : (f - 2) % (2 * K + 2);
  if (q < K) {
    r.kind = kRgFwd;
    r.level = q;
    r.units = fwd_tasks(I.N, rg_level(I.N, q));
  } else if (q < 2 * K) {
    r.kind = kRgBwd;
    r.level = 2 * K - 1 - q;
    r.units = rg_level(I.N, r.level).d;
  } else if (q == 2 * K) {
    r.kind = kRgXupd;
    r.level = 0;
    r.units = I.N;
    r.upc = 16;    // 16 blocks per chunk: a short elementwise pass
  } else {
    r.kind = kRgRes;
    r.level = 0;
    r.units = I.N;   // block rows (n <= 64: one CTA pass per row)
  }
  return r;
}

__host__ __device__ inline int rg_chunks(const RgPhase& P) { return (P.units + P.upc - 1) / P.upc; }

struct RgQueue {
  unsigned long long* slot;   // capacity entries; 0 = empty
  unsigned int* head;         // next slot to pop
  unsigned int* tail;         // next slot to push
  unsigned int* done;         // finished instances
  int* rem;                   // per instance: unfinished chunks of its current phase
  int* error;                 // 1: a queue wait gave up; 2: the queue overflowed
  const unsigned long long* init;   // first-phase chunks of every instance, in priority order
  unsigned int n_init;
  unsigned int capacity;
};

template <typename T>
struct RgArgs {
  const RgInst* inst;
  int count;
  T* L;   // packed diagonal blocks (factored in place; float copy when refining)
  T* E;   // packed off-diagonal storage
  T* X;   // packed right-hand sides / solutions (float correction when refining)
  // refinement only
  const double* L64;
  const double* E64;
  const double* b64;
  double* x64;
  RefineState* st;
  double* eta;
  int* iters;
  double tol;
  int max_iter;
  RgQueue q;
  int vc;                     // unused (node vectors per pass of the blocked-solve body)
  long long timeout_ns;       // bound of one queue wait
};

__device__ __forceinline__ unsigned long long rg_clock() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long rg_load_slot(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ unsigned int rg_load_u32(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Thread 0: next task for this CTA, or kRgExit.
template <typename T>
__device__ unsigned long long rg_pop(const RgArgs<T>& a) {
  const unsigned int k = atomicAdd(a.q.head, 1u);
  if (k >= a.q.capacity) {
    // more pops than slots: only possible once every task has been handed out
    if (rg_load_u32(a.q.done) < (unsigned)a.count) atomicExch(a.q.error, 2);
    return kRgExit;
  }
  // the bound runs from the last sign of progress (a push or a finished
  // instance), so only a queue that stopped moving gives up
  unsigned long long t0 = rg_clock();
  unsigned int seen_tail = rg_load_u32(a.q.tail), seen_done = rg_load_u32(a.q.done);
  unsigned int ns = 32;
  while (true) {
    const unsigned long long v = rg_load_slot(a.q.slot + k);
    if (v & kRgValid) {
      __threadfence();
      return v;
    }
    const unsigned int done = rg_load_u32(a.q.done), tail = rg_load_u32(a.q.tail);
    if (done >= (unsigned)a.count) return kRgExit;
    const unsigned long long now = rg_clock();
    if (done != seen_done || tail != seen_tail) {
      seen_done = done;
      seen_tail = tail;
      t0 = now;
    } else if ((long long)(now - t0) > a.timeout_ns) {
      atomicExch(a.q.error, 1);
      return kRgExit;
    }
    __nanosleep(ns);
    if (ns < 1024) ns *= 2;
  }
}

// Per-instance view of the packed arrays.
template <typename T>
__device__ __forceinline__ Problem<T> rg_problem(const RgArgs<T>& a, const RgInst& I, int m) {
  Problem<T> p;
  p.L = a.L + I.oL;
  p.E = a.E + I.oE;
  p.X = a.X + I.oX;
  p.mask = nullptr;
  p.info = nullptr;
  p.B = 1;
  p.N = I.N;
  p.n = I.n;
  p.m = m;
  p.S = I.S;
  p.sL = p.sE = p.sX = 0;
  return p;
}

template <typename T>
__device__ __forceinline__ RefineArgs rg_refine_args(const RgArgs<T>& a, const RgInst& I, int ii) {
  RefineArgs r;
  r.L = a.L64 + I.oL;
  r.E = a.E64 + I.oE;
  r.b = a.b64 + I.oX;
  r.x = a.x64 + I.oX;
  r.mask = nullptr;
  r.L32 = reinterpret_cast<float*>(a.L) + I.oL;
  r.E32 = reinterpret_cast<float*>(a.E) + I.oE;
  r.R32 = reinterpret_cast<float*>(a.X) + I.oX;
  r.active = nullptr;
  r.st = a.st + ii;
  r.eta = nullptr;
  r.iters = nullptr;
  r.any_active = nullptr;
  r.rout = nullptr;
  r.B = 1;
  r.N = I.N;
  r.n = I.n;
  r.m = I.m;
  r.S = I.S;
  r.tol = a.tol;
  r.max_iter = a.max_iter;
  r.check_in_residual = 0;
  return r;
}

// Execute one chunk (all threads of the CTA).
template <typename T, int MODE>
__device__ void rg_run(const RgArgs<T>& a, int ii, int ph, int chunk, unsigned char* smem) {
  const RgInst I = a.inst[ii];
  const RgPhase P = rg_phase(I, MODE, ph);
  const int u0 = chunk * P.upc;
  const int u1 = min_i(P.units, u0 + P.upc);
  const Level lv = rg_level(I.N, P.level);
  constexpr bool kPlain = MODE == kRgPlain;
  if (P.kind == kRgXupd) {
    if constexpr (!kPlain) {
      const long long per = (long long)I.n * I.m;
      const float* d = reinterpret_cast<const float*>(a.X) + I.oX + u0 * per;
      double* x = a.x64 + I.oX + u0 * per;
      const long long len = (long long)(u1 - u0) * per;
      for (long long e = threadIdx.x; e < len; e += blockDim.x) x[e] += (double)d[e];
    }
    return;
  }
  for (int u = u0; u < u1; ++u) {
    if (u > u0) __syncthreads();
    switch (P.kind) {
      case kRgNode: {
        const Problem<T> p = rg_problem(a, I, I.m);
        node_gemm_body<T, true, true, false>(p, lv, 0, u, smem);
        break;
      }
      case kRgUpd: {
        const Problem<T> p = rg_problem(a, I, I.m);
        const int U = I.N / (2 * lv.s);
        update_full_body<T>(p, lv, 0, u, smem);
        if (u + 1 <= lv.d - 1) {   // fill-in block of node t = u + 1
          __syncthreads();
          update_full_body<T>(p, lv, 0, U + u, smem);
        }
        // y_j -= F y_{j-s} + G^T y_{j+s} for target j = 2s(u+1) - 1
        __syncthreads();
        fwd_body<T, true, true, false>(p, rg_level(I.N, P.level + 1), 0, u, smem);
        break;
      }
      case kRgBwd: {
        const Problem<T> p = rg_problem(a, I, I.m);
        bwd_body<T, true, true>(p, lv, 0, u, smem);
        break;
      }
      case kRgFwd: {
        if constexpr (!kPlain) {
          const Problem<T> p = rg_problem(a, I, I.m);
          fwd_body<T, true, false, true>(p, lv, 0, u, smem);
        }
        break;
      }
      case kRgInit: {
        if constexpr (!kPlain) ref_init_rows_body(rg_refine_args(a, I, ii), 0, u, smem);
        break;
      }
      case kRgRes: {
        if constexpr (!kPlain) {
          residual_rows_body<true, 1>(rg_refine_args(a, I, ii), 0, u, smem);
        }
        break;
      }
      default:
        break;
    }
  }
}

// Thread 0, after the CTA finished chunk `chunk` of phase `ph` of instance ii:
// the continuation task (chunk 0 of the next phase) or 0.
template <typename T, int MODE>
__device__ unsigned long long rg_complete(const RgArgs<T>& a, int ii, int ph) {
  __threadfence();
  if (atomicSub(a.q.rem + ii, 1) != 1) return 0ull;
  __threadfence();
  const RgInst I = a.inst[ii];
  int nph = ph + 1;
  if (MODE == kRgRefine && rg_phase(I, MODE, ph).kind == kRgRes) {
    RefineState* s = a.st + ii;
    const double rn = __longlong_as_double((long long)atomicAdd(&s->rnorm, 0ull));
    const double xn = __longlong_as_double((long long)atomicAdd(&s->xnorm, 0ull));
    const double pn = __longlong_as_double((long long)atomicAdd(&s->psi, 0ull));
    const double bn = __longlong_as_double((long long)atomicAdd(&s->bnorm, 0ull));
    const double den = pn * xn + bn;
    const double eta = den > 0.0 ? rn / den : 0.0;
    const int it = a.iters[ii] + 1;
    a.eta[ii] = eta;
    atomicExch(&s->rnorm, 0ull);
    atomicExch(&s->xnorm, 0ull);
    if (!(eta == eta) || isinf(eta)) {
      a.iters[ii] = -it;
      nph = -1;
    } else {
      a.iters[ii] = it;
      if (eta <= a.tol || it >= a.max_iter) nph = -1;
    }
  }
  if (MODE == kRgPlain && nph >= rg_plain_phases(I.K)) nph = -1;
  RgPhase P{};
  if (nph >= 0) {
    P = rg_phase(I, MODE, nph);
    while (P.units <= 0) {   // no phase of a valid schedule is empty; stay safe regardless
      ++nph;
      if (MODE == kRgPlain && nph >= rg_plain_phases(I.K)) {
        nph = -1;
        break;
      }
      P = rg_phase(I, MODE, nph);
    }
  }
  if (nph < 0) {
    __threadfence();
    atomicAdd(a.q.done, 1u);
    return 0ull;
  }
  const int c = rg_chunks(P);
  atomicExch(a.q.rem + ii, c);
  __threadfence();
  if (c > 1) {
    const unsigned int base = atomicAdd(a.q.tail, (unsigned)(c - 1));
    for (int j = 1; j < c; ++j) {
      const unsigned int k = base + (unsigned)(j - 1);
      if (k < a.q.capacity) atomicExch(a.q.slot + k, rg_encode(ii, nph, j));
      else atomicExch(a.q.error, 2);
    }
  }
  return rg_encode(ii, nph, 0);
}

// Queue reset and first-phase chunks; per-instance refinement state.
template <typename T, int MODE>
__global__ void k_rg_start(RgArgs<T> a) {
  const int gid = blockIdx.x * blockDim.x + threadIdx.x, gs = gridDim.x * blockDim.x;
  for (unsigned int k = gid; k < a.q.n_init; k += gs) a.q.slot[k] = a.q.init[k];
  for (int i = gid; i < a.count; i += gs) {
    const RgInst I = a.inst[i];
    a.q.rem[i] = rg_chunks(rg_phase(I, MODE, 0));
    if (MODE == kRgRefine) {
      a.st[i].psi = 0ull;
      a.st[i].bnorm = 0ull;
      a.st[i].rnorm = 0ull;
      a.st[i].xnorm = 0ull;
      a.eta[i] = __longlong_as_double(0x7ff0000000000000LL);
      a.iters[i] = 0;
    }
  }
  if (gid == 0) {
    *a.q.head = 0u;
    *a.q.tail = a.q.n_init;
    *a.q.done = 0u;
    *a.q.error = 0;
  }
}

// The persistent solver: every CTA loops pop -> run -> complete.  128
// threads, 3 CTAs per SM at n = 48 (shared-memory bound); registers capped at
// 168 for FP64 (no spills: measured 66.9k -> 75.7k solves/s on the 4096-system
// batch) and at 128 for float (the float path measured faster there).
constexpr int kRgThreads = 128;
template <typename T, int MODE>
__global__ void __launch_bounds__(kRgThreads, sizeof(T) == 8 ? 3 : 4) k_ragged(RgArgs<T> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ unsigned long long s_task;
  unsigned long long task = 0ull;
  while (true) {
    if (task == 0ull) {
      if (threadIdx.x == 0) s_task = rg_pop(a);
      __syncthreads();
      task = s_task;
      __syncthreads();
      if (task == kRgExit) return;
    }
    int ii, ph, chunk;
    rg_decode(task, ii, ph, chunk);
    rg_run<T, MODE>(a, ii, ph, chunk, smem_raw);
    __syncthreads();
    if (threadIdx.x == 0) s_task = rg_complete<T, MODE>(a, ii, ph);
    __syncthreads();
    task = s_task;
    __syncthreads();
  }
}

}  // namespace socu
