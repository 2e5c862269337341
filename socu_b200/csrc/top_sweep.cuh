// Top levels of the substitution sweeps in one cluster-resident kernel.
//
// The upper levels of a sweep hold 1-16 nodes each.  Launched one level at a
// time, every level pays a kernel start, the load of its blocks (the factor
// block and up to two coupling blocks per node, 48 KB at n = 64 float) and
// the product chain, a few microseconds of latency for a few nodes of work.
// k_top walks all of those levels inside one thread-block cluster per system:
//
//   * forward levels fwd_lo .. K-1 (ascending), then backward levels
//     K-1 .. bwd_lo (descending) -- the same node arithmetic as k_fwd / k_bwd
//     (fwd_body / bwd_body, resident blocks), task t of a level on cluster
//     CTA t mod C;
//   * between two levels a cluster barrier (barrier.cluster arrive.release /
//     wait.acquire): every vector a level writes is visible to the next;
//   * the blocks a CTA needs are known up front (they do not depend on the
//     vectors), so the TMA copy of the next item's blocks runs into a second
//     shared buffer while the current item computes; vectors are read with
//     L2-only loads after the barrier (other CTAs of the cluster wrote them).
//
// Products are the ones the per-level kernels use, chosen by the same
// Level::tc, so the results are bit-identical to the per-level sweeps.
//
// Opt-in (SOCU_TOP_SWEEP=1): on B200 the per-level launches of a CUDA graph
// with programmatic dependent launch are faster.  Measured per level of a
// float sweep (N=1024, n=64, m=8, CTA 0 of k_top, %globaltimer): block wait
// 0.2 us (the prefetch works), vector reads from L2 1.1-1.7 us, products
// 2.6-3.5 us, cluster barrier 0.9-2.2 us -- about 6.5 us against ~5 us for a
// level launched on its own, whose launch and block loads overlap the kernel
// before it.
//
// The cluster barrier is the hardware barrier: every CTA of a cluster runs
// the same sequence of barriers (one per level but the last, whether or not
// it has a task there), so none can wait for a CTA that left.  TMA waits are
// bounded (tma::wait): after one runs out the CTA stops computing and
// copying, keeps taking part in the barriers and reports g_tc_error = 2.
// Copies are unicast loads of this GPU's own memory (no cluster multicast).
#pragma once

#include "nd_kernels.cuh"
#include "tma.cuh"

namespace socu {

constexpr int kTopMaxLevels = 12;

// Levels of one k_top launch.  fl[i]: forward level fwd_lo + i; bl[i]:
// backward level bwd_lo + i; the host fills them as it would for the
// per-level launches (tc, stride, slot offsets).
struct TopLevels {
  Level fl[kTopMaxLevels];
  Level bl[kTopMaxLevels];
  int fwd_lo, fwd_n;   // forward levels fwd_lo .. fwd_lo + fwd_n - 1 (fwd_n = 0: none)
  int bwd_lo, bwd_n;   // backward levels bwd_lo + bwd_n - 1 .. bwd_lo (bwd_n = 0: none)
  int pre;             // every block final before the kernel started: first copies before the dependency wait
  int stages;          // block buffers per CTA (1 or 2)
};

// shared memory of k_top in elements of T: stages x 3 block regions, three
// vector regions, dv (n) and the stage mbarriers (rounded as in smem_sweep_res_elems)
__host__ __device__ inline long long smem_top_elems(int n, int m, int stages) {
  const int mc = min_i(m, kMC);
  return 3LL * stages * res_round((long long)n * res_ldm(n), 4) + 3LL * res_round((long long)n * res_ldy(mc), 4) +
         n + 8;
}

__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

__device__ __forceinline__ unsigned cluster_ctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}

__device__ __forceinline__ unsigned cluster_nctarank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;\n" : "=r"(r));
  return r;
}

// rows x cols of a vector (row stride src_ld) into shared memory, through L2
// (ld.global.cg): the data may come from another CTA of the cluster
template <typename T>
__device__ __forceinline__ void load_vec_l2(T* dst, int ld, const T* src, int rows, int cols, long long src_ld) {
  const int total = rows * cols;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    const int r = e / cols, c = e - r * cols;
    dst[r * ld + c] = __ldcg(src + (long long)r * src_ld + c);
  }
}

// One item (a node task of one level) of a CTA: which blocks it reads.
struct TopItem {
  bool bwd;          // backward level (else forward)
  int s;             // stride of the level
  int j;             // node / target vector
  int cblk;          // factor block index (-1: none)
  int fslot, gslot;  // coupling slots (-1: none)
  bool pull, solve;  // forward: coupling updates, diagonal solve
  int zlo, zhi;      // vectors read besides j: forward j-h (pull), j+h (G); backward i+s (F), i-s (G); -1: none
};

__device__ __forceinline__ TopItem top_item(const TopLevels& tl, int N, bool bwd, int li, int t) {
  TopItem it;
  it.bwd = bwd;
  if (!bwd) {
    const Level& L = tl.fl[li];
    it.s = L.s;
    if (L.s == 1) {
      it.j = 2 * t;
      it.pull = false;
      it.solve = true;
      it.fslot = it.gslot = -1;
      it.zlo = it.zhi = -1;
    } else {
      const int u = t + 1, h = L.s / 2;
      it.j = L.s * u - 1;
      it.pull = true;
      it.solve = (u & 1) != 0;
      it.fslot = L.op + 2 * u - 2;
      it.gslot = it.j + h < N ? it.fslot + 1 : -1;
      it.zlo = it.j - h;
      it.zhi = it.gslot >= 0 ? it.j + h : -1;
    }
    it.cblk = it.solve ? it.j : -1;
  } else {
    const Level& L = tl.bl[li];
    const int s = L.s, i = s - 1 + 2 * s * t;
    it.s = s;
    it.j = i;
    it.pull = false;
    it.solve = true;
    it.cblk = i;
    const int slot = L.oc + 2 * t;
    it.fslot = i + s < N ? slot : -1;
    it.gslot = i >= s ? slot - 1 : -1;
    it.zlo = it.fslot >= 0 ? i + s : -1;   // right neighbour (with F)
    it.zhi = it.gslot >= 0 ? i - s : -1;   // left neighbour (with G)
  }
  return it;
}

// Walks a CTA's items in execution order: forward levels ascending, then
// backward levels descending, tasks rank, rank + C, ... of each level.
struct TopCursor {
  int ph, li, t;   // phase (0 forward, 1 backward, 2 done), level position in the phase, task
};

__device__ __forceinline__ int top_tasks(const TopLevels& tl, int N, int ph, int li) {
  return ph == 0 ? fwd_tasks(N, tl.fl[li]) : tl.bl[tl.bwd_n - 1 - li].d;
}

__device__ __forceinline__ void top_settle(const TopLevels& tl, int N, int rank, TopCursor& c) {
  while (c.ph < 2) {
    const int nl = c.ph == 0 ? tl.fwd_n : tl.bwd_n;
    if (c.li >= nl) {
      ++c.ph;
      c.li = 0;
      c.t = rank;
      continue;
    }
    if (c.t < top_tasks(tl, N, c.ph, c.li)) return;
    ++c.li;
    c.t = rank;
  }
}

__device__ __forceinline__ TopItem top_item_at(const TopLevels& tl, int N, const TopCursor& c) {
  return c.ph == 0 ? top_item(tl, N, false, c.li, c.t) : top_item(tl, N, true, tl.bwd_n - 1 - c.li, c.t);
}

// One thread: the TMA copies of an item's blocks into stage buffer Ms (C, F, G).
template <typename T>
__device__ __forceinline__ void top_issue(const TopItem& it, const SweepMaps& tm, int b, T* Ms, long long vm, int n,
                                          int ldm, uint64_t* bar) {
  const int nblk = (it.cblk >= 0 ? 1 : 0) + (it.fslot >= 0 ? 1 : 0) + (it.gslot >= 0 ? 1 : 0);
  tma::expect_tx(bar, (uint32_t)(nblk * n * ldm * sizeof(T)));
  if (it.cblk >= 0) tma::load_4d(Ms, &tm.L, 0, 0, it.cblk, b, bar);
  if (it.fslot >= 0) tma::load_4d(Ms + vm, &tm.E, 0, 0, it.fslot, b, bar);
  if (it.gslot >= 0) tma::load_4d(Ms + 2 * vm, &tm.E, 0, 0, it.gslot, b, bar);
}

template <typename T, bool INV>
__global__ void __launch_bounds__(256) k_top(Problem<T> p, const __grid_constant__ TopLevels tl,
                                             const __grid_constant__ SweepMaps tm) {
  const int C = (int)cluster_nctarank(), rank = (int)cluster_ctarank();
  const int b = blockIdx.x / C;
  if (!p.active(b)) return;   // the whole cluster (one instance) leaves together
  extern __shared__ __align__(128) unsigned char smem_raw[];
  const int n = p.n, N = p.N;
  const int mcmax = min_i(p.m, kMC), ldy = res_ldy(mcmax), ldm = res_ldm(n);
  const long long vm = res_round((long long)n * ldm, sizeof(T));
  const long long vy = res_round((long long)n * ldy, sizeof(T));
  const int stages = tl.stages;
  T* Mbase = reinterpret_cast<T*>(smem_raw);
  T* Y = Mbase + 3LL * stages * vm;
  T* Z1 = Y + vy;
  T* Z2 = Z1 + vy;
  T* dv = Z2 + vy;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw + ((reinterpret_cast<unsigned char*>(dv + n) - smem_raw + 7) & ~7LL));
  const bool use_tma = tm.blocks != 0 && (smem_addr(smem_raw) & 127u) == 0;
  if (use_tma) {
    if (threadIdx.x == 0)
      for (int k = 0; k < stages; ++k) tc::mbar_init(bar + k, 1);
    __syncthreads();
  }

  // loader cursor: the next item whose blocks are not yet requested
  TopCursor ld{tl.fwd_n > 0 ? 0 : 1, 0, rank};
  top_settle(tl, N, rank, ld);
  int issued = 0;
  auto issue_next = [&](int stage) {
    if (threadIdx.x == 0) {
      tma::fence_proxy();   // earlier reads of the stage before the async-proxy writes
      top_issue<T>(top_item_at(tl, N, ld), tm, b, Mbase + 3LL * stage * vm, vm, n, ldm, bar + stage);
    }
    ++issued;
    ld.t += C;
    top_settle(tl, N, rank, ld);
  };
  if (!tl.pre) pdl_wait();
  if (use_tma)
    for (int k = 0; k < stages && ld.ph < 2; ++k) issue_next(k);
  if (tl.pre) pdl_wait();
  pdl_trigger();

  bool ok = true;
  int consumed = 0;
  for (int ph = 0; ph < 2; ++ph) {
    const int nl = ph == 0 ? tl.fwd_n : tl.bwd_n;
    for (int li = 0; li < nl; ++li) {
      const int tasks = top_tasks(tl, N, ph, li);
      const Level& L = ph == 0 ? tl.fl[li] : tl.bl[tl.bwd_n - 1 - li];
      for (int t = rank; t < tasks; t += C) {
        const int stage = consumed % stages;
        const unsigned parity = (unsigned)(consumed / stages) & 1u;
        const TopItem it = ph == 0 ? top_item(tl, N, false, li, t) : top_item(tl, N, true, tl.bwd_n - 1 - li, t);
        T* Cs = Mbase + 3LL * stage * vm;
        T* Fs = Cs + vm;
        T* Gs = Fs + vm;
        if (ok) {
          if (use_tma) {
            ok = tma::wait(bar + stage, parity);
          } else {
            if (it.cblk >= 0) async_load(Cs, ldm, p.Lb(b, it.cblk), n, n, n);
            if (it.fslot >= 0) async_load(Fs, ldm, p.Eb(b, it.fslot), n, n, n);
            if (it.gslot >= 0) async_load(Gs, ldm, p.Eb(b, it.gslot), n, n, n);
            cp_async_wait_all();
            __syncthreads();
          }
        }
        if (ok) {
          const bool tc = INV && sweep_uses_dmma<T>(L);
          T* xj = p.Xb(b, it.j);
          for (int c0 = 0; c0 < p.m; c0 += kMC) {
            const int mc = min_i(kMC, p.m - c0);
            __syncthreads();
            load_vec_l2(Y, ldy, xj + c0, n, mc, p.m);
            if (it.zlo >= 0) load_vec_l2(Z1, ldy, p.Xb(b, it.zlo) + c0, n, mc, p.m);
            if (it.zhi >= 0) load_vec_l2(Z2, ldy, p.Xb(b, it.zhi) + c0, n, mc, p.m);
            __syncthreads();
            if (c0 == 0 && it.solve)
              for (int r = threadIdx.x; r < n; r += blockDim.x) dv[r] = T(1) / Cs[r * ldm + r];
            if (!it.bwd) {
              // Y -= F y_{j-h} + G^T y_{j+h}; then y_j <- C^{-1} Y on level nodes
              const bool hasG = it.gslot >= 0;
              if (it.pull) {
                if (tc)
                  dmma_product<T, 0, false, true>(Y, Z1, Fs, ldm, hasG ? Z2 : nullptr, hasG ? Gs : nullptr, ldm, ldy,
                                                  mc, nullptr, n);
                else
                  res_matvec_pair<T, false, true>(Y, Z1, Fs, hasG ? Z2 : nullptr, hasG ? Gs : nullptr, ldy, mc, ldm,
                                                  n);
              }
              __syncthreads();
              if (it.solve) {
                if (INV) {
                  if (tc)
                    dmma_product<T, 3, true, false>(Z2, Y, Cs, ldm, nullptr, nullptr, 0, ldy, mc, dv, n);
                  else
                    res_matvec<T, 3>(Z2, Y, ldy, mc, Cs, ldm, dv, n);
                  __syncthreads();
                  store_block(xj + c0, p.m, Z2, ldy, n, mc);
                  continue;
                }
                res_tri_solve<T, false>(Y, ldy, mc, Cs, ldm, dv, n);
              }
              store_block(xj + c0, p.m, Y, ldy, n, mc);
            } else {
              // Y -= F^T x_{i+s} + G x_{i-s}; then x_i <- C^{-T} Y
              const bool right = it.fslot >= 0, left = it.gslot >= 0;
              if (right || left) {
                if (tc)
                  dmma_product<T, 0, true, false>(Y, right ? Z1 : nullptr, right ? Fs : nullptr, ldm,
                                                  left ? Z2 : nullptr, left ? Gs : nullptr, ldm, ldy, mc, nullptr, n);
                else
                  res_matvec_pair<T, true, false>(Y, right ? Z1 : nullptr, right ? Fs : nullptr, left ? Z2 : nullptr,
                                                  left ? Gs : nullptr, ldy, mc, ldm, n);
              }
              __syncthreads();
              if (INV) {
                if (tc)
                  dmma_product<T, 2, false, false>(Z1, Y, Cs, ldm, nullptr, nullptr, 0, ldy, mc, dv, n);
                else
                  res_matvec<T, 2>(Z1, Y, ldy, mc, Cs, ldm, dv, n);
                __syncthreads();
                store_block(xj + c0, p.m, Z1, ldy, n, mc);
                continue;
              }
              res_tri_solve<T, true>(Y, ldy, mc, Cs, ldm, dv, n);
              store_block(xj + c0, p.m, Y, ldy, n, mc);
            }
          }
        }
        // the stage is free: request the blocks of the item `stages` ahead
        __syncthreads();
        if (use_tma && ok && ld.ph < 2) issue_next(stage);
        ++consumed;
      }
      const bool last = ph == 1 ? li == nl - 1 : (tl.bwd_n == 0 && li == nl - 1);
      if (!last) cluster_barrier();
    }
  }
  // after a wait ran out: let the copies still in flight land (bounded) before the CTA leaves
  if (!ok && threadIdx.x == 0)
    for (int k = consumed; k < issued; ++k) tc::mbar_wait(bar + k % stages, (unsigned)(k / stages) & 1u, kTmaWaitNs);
}

}  // namespace socu
