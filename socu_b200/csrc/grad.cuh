// Gradient of x = Psi^{-1} b with respect to the D and E blocks of Psi.
//
// With g = Psi^{-1} gx (gx = dloss/dx; Psi is symmetric), dloss/dPsi = -g x^T
// entrywise.  Psi reads only lower(D_i) (socu/blas/potrf.py:101-102), so
//   dD_i[r][c] = -sum_j (g_i[r][j] x_i[c][j] + g_i[c][j] x_i[r][j])   r > c
//   dD_i[r][r] = -sum_j  g_i[r][j] x_i[r][j]
//   dD_i[r][c] = 0                                                    r < c
// and E_i = Psi_{i+1,i} (its transpose is Psi_{i,i+1}):
//   dE_i[r][c] = -sum_j (g_{i+1}[r][j] x_i[c][j] + g_i[c][j] x_{i+1}[r][j])
// One CTA per (instance, block row i) writes dD_i and dE_i.
#pragma once

#include "nd_device.cuh"

namespace socu {

template <typename T>
struct GradArgs {
  const T* x;   // (B, N, n, m)
  const T* g;   // (B, N, n, m)
  T* dD;        // (B, N, n, n)
  T* dE;        // (B, SE, n, n), slots >= N-1 zeroed
  int B, N, n, m, SE;
};

__host__ __device__ inline long long smem_grad_elems(int n, int m) { return 4LL * n * (m + 1); }

template <typename T>
__global__ void __launch_bounds__(256) k_grad(GradArgs<T> a) {
  const int per = a.N > a.SE ? a.N : a.SE;
  const int b = blockIdx.x / per;
  const int i = blockIdx.x - b * per;
  const int n = a.n, m = a.m, ld = m + 1;
  const long long nn = (long long)n * n;
  if (i >= a.N) {   // storage slots beyond N-1 carry no entries of Psi
    T* dE = a.dE + ((long long)b * a.SE + i) * nn;
    for (long long e = threadIdx.x; e < nn; e += blockDim.x) dE[e] = T(0);
    return;
  }
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* Xi = reinterpret_cast<T*>(smem_raw);
  T* Gi = Xi + n * ld;
  T* Xn = Gi + n * ld;
  T* Gn = Xn + n * ld;
  const long long vo = ((long long)b * a.N + i) * n * m;
  const bool next = i + 1 < a.N;
  async_load(Xi, ld, a.x + vo, n, m, m);
  async_load(Gi, ld, a.g + vo, n, m, m);
  if (next) {
    async_load(Xn, ld, a.x + vo + (long long)n * m, n, m, m);
    async_load(Gn, ld, a.g + vo + (long long)n * m, n, m, m);
  }
  cp_async_wait_all();
  __syncthreads();
  T* dD = a.dD + ((long long)b * a.N + i) * nn;
  for (long long e = threadIdx.x; e < nn; e += blockDim.x) {
    const int r = (int)(e / n), c = (int)(e - (long long)r * n);
    T v = T(0);
    if (c < r) {
      for (int j = 0; j < m; ++j) v = fma(Gi[r * ld + j], Xi[c * ld + j], fma(Gi[c * ld + j], Xi[r * ld + j], v));
    } else if (c == r) {
      for (int j = 0; j < m; ++j) v = fma(Gi[r * ld + j], Xi[r * ld + j], v);
    }
    dD[e] = -v;
  }
  if (i < a.SE) {
    T* dE = a.dE + ((long long)b * a.SE + i) * nn;
    for (long long e = threadIdx.x; e < nn; e += blockDim.x) {
      const int r = (int)(e / n), c = (int)(e - (long long)r * n);
      T v = T(0);
      if (next)
        for (int j = 0; j < m; ++j) v = fma(Gn[r * ld + j], Xi[c * ld + j], fma(Gi[c * ld + j], Xn[r * ld + j], v));
      dE[e] = -v;
    }
  }
}

}  // namespace socu
