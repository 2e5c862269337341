// C ABI of socu_b200: argument validation, level scheduling, kernel enqueue,
// and launch objects with optional CUDA-graph capture.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "../../include/socu_b200.h"
#include "nd_kernels.cuh"

namespace socu {
namespace {

thread_local int g_last_cuda_error = 0;

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return SOCU_OK;
  g_last_cuda_error = static_cast<int>(e);
  return SOCU_ERR_CUDA;
}

std::vector<Level> schedule(int N) {
  // socu/block_tridiag_solver.py:869-914
  std::vector<Level> out;
  int s = 1, curr = 0, nxt = N - 1;
  const int K = static_cast<int>(socu_recursive_iterations(N));
  for (int l = 0; l < K; ++l) {
    Level lv;
    lv.s = s;
    lv.d = (N + s) / (2 * s);
    lv.oc = curr;
    lv.on = nxt;
    out.push_back(lv);
    s *= 2;
    curr = nxt;
    nxt += N / s - 1;
  }
  return out;
}

int threads_for(int n) { return n <= 16 ? 64 : (n <= 32 ? 128 : 256); }

int max_smem_optin() {
  static int cached = -1;
  if (cached < 0) {
    int dev = 0, v = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
      v = 227 * 1024;
    cached = v;
  }
  return cached;
}

// Opt in to large dynamic shared memory once per kernel and size (the
// attribute is per function and device; a small cache keeps repeated calls
// off the driver).
std::mutex g_prep_mu;
std::map<std::pair<const void*, int>, size_t> g_prepared;

template <typename K>
cudaError_t prepare(K kernel, size_t smem) {
  if (smem <= 48 * 1024) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
  std::lock_guard<std::mutex> g(g_prep_mu);
  auto it = g_prepared.find(key);
  if (it != g_prepared.end() && it->second >= smem) return cudaSuccess;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess) g_prepared[key] = smem;
  return e;
}

// The library links the CUDA runtime statically, so its notion of the
// current device is separate from the caller's: follow the device that owns
// the data.
cudaError_t ensure_device(const void* ptr) {
  if (ptr == nullptr) return cudaSuccess;
  cudaPointerAttributes attr;
  cudaError_t e = cudaPointerGetAttributes(&attr, ptr);
  if (e != cudaSuccess) return e;
  if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged) return cudaErrorInvalidValue;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != attr.device) e = cudaSetDevice(attr.device);
  return e;
}

struct Dims {
  int B, N, n, m, S;
};

bool grid_ok(long long blocks) { return blocks > 0 && blocks < (1LL << 31); }

template <typename T>
Problem<T> make_problem(void* L, void* E, void* x, const uint8_t* mask, const Dims& d) {
  Problem<T> p;
  p.L = static_cast<T*>(L);
  p.E = static_cast<T*>(E);
  p.X = static_cast<T*>(x);
  p.mask = mask;
  p.B = d.B;
  p.N = d.N;
  p.n = d.n;
  p.m = d.m;
  p.S = d.S;
  p.sL = (long long)d.N * d.n * d.n;
  p.sE = (long long)d.S * d.n * d.n;
  p.sX = (long long)d.N * d.n * d.m;
  return p;
}

// Enqueue (or count, when st == nullptr and count != nullptr) the kernels of one op.
template <typename T>
int enqueue(socu_op op, const Problem<T>& p, cudaStream_t st, long long* count) {
  const std::vector<Level> lv = schedule(p.N);
  const int K = static_cast<int>(lv.size());
  const int n = p.n, nth = threads_for(n);
  const bool withY = op == SOCU_OP_FACTOR_AND_SOLVE;
  const size_t sd = smem_diag_elems(n, withY ? p.m : 0) * sizeof(T);
  const size_t sc = smem_couple_elems(n) * sizeof(T);
  const size_t su = smem_update_elems(n) * sizeof(T);
  const size_t ss = smem_sweep_elems(n, p.m > 0 ? p.m : 1) * sizeof(T);
  const int nt = ceil_div(n, kTile), nlt = nt * (nt + 1) / 2;
  long long launches = 0;
  const bool run = count == nullptr;

  if (run) {
    cudaError_t e = cudaSuccess;
    if (op == SOCU_OP_FACTOR || op == SOCU_OP_FACTOR_AND_SOLVE) {
      e = withY ? prepare(k_diag<T, true>, sd) : prepare(k_diag<T, false>, sd);
      if (e == cudaSuccess) e = prepare(k_couple<T>, sc);
      if (e == cudaSuccess) e = prepare(k_update<T>, su);
    }
    if (e == cudaSuccess) e = prepare(k_fwd_node<T>, ss);
    if (e == cudaSuccess) e = prepare(k_fwd_update<T>, ss);
    if (e == cudaSuccess) e = prepare(k_bwd<T>, ss);
    if (e != cudaSuccess) return cuda_status(e);
  }

  auto go = [&](auto kernel, long long blocks, size_t smem, const Level& L) {
    if (blocks <= 0) return;
    ++launches;
    if (run) kernel<<<(unsigned)blocks, nth, smem, st>>>(p, L);
  };

  const bool factor = op == SOCU_OP_FACTOR || op == SOCU_OP_FACTOR_AND_SOLVE;
  if (factor) {
    for (int l = 0; l < K; ++l) {
      const Level& L = lv[l];
      if (withY)
        go(k_diag<T, true>, (long long)p.B * L.d, sd, L);
      else
        go(k_diag<T, false>, (long long)p.B * L.d, sd, L);
      if (l + 1 < K) {
        go(k_couple<T>, (long long)p.B * L.d * 2 * nt, sc, L);
        const int U = p.N / (2 * L.s);
        go(k_update<T>, (long long)p.B * (U * nlt + (L.d - 1) * nt * nt), su, L);
        if (withY) go(k_fwd_update<T>, (long long)p.B * U, ss, L);
      }
    }
  }
  if (op == SOCU_OP_FORWARD_SUBSTITUTION || op == SOCU_OP_SOLVE) {
    for (int l = 0; l < K; ++l) {
      const Level& L = lv[l];
      go(k_fwd_node<T>, (long long)p.B * L.d, ss, L);
      if (l + 1 < K) go(k_fwd_update<T>, (long long)p.B * (p.N / (2 * L.s)), ss, L);
    }
  }
  if (op == SOCU_OP_BACKWARD_SUBSTITUTION || op == SOCU_OP_SOLVE || op == SOCU_OP_FACTOR_AND_SOLVE) {
    for (int l = K - 1; l >= 0; --l) go(k_bwd<T>, (long long)p.B * lv[l].d, ss, lv[l]);
  }
  if (count) *count = launches;
  if (run) return cuda_status(cudaGetLastError());
  return SOCU_OK;
}

int validate(socu_op op, socu_dtype dtype, const void* L, const void* E, const void* x,
             int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, Dims* d) {
  if (dtype != SOCU_FLOAT32 && dtype != SOCU_FLOAT64) return SOCU_ERR_INVALID_ARGUMENT;
  if ((int)op < 0 || (int)op > 4) return SOCU_ERR_INVALID_ARGUMENT;
  if (batch < 0 || horizon <= 0 || n <= 0) return SOCU_ERR_INVALID_ARGUMENT;
  const bool needs_x = op != SOCU_OP_FACTOR;
  if (needs_x && n_rhs <= 0) return SOCU_ERR_INVALID_ARGUMENT;
  if (horizon > (1 << 30) || n > 4096 || batch > (1LL << 30) || (needs_x && n_rhs > (1 << 20)))
    return SOCU_ERR_UNSUPPORTED;
  const int64_t S = socu_off_diag_storage_len(horizon);
  if (batch > 0) {
    if (L == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
    if (S > 0 && E == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
    if (needs_x && x == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  }
  if ((int64_t)n > socu_max_block_size(dtype, needs_x ? n_rhs : 0)) return SOCU_ERR_UNSUPPORTED;
  d->B = (int)batch;
  d->N = (int)horizon;
  d->n = (int)n;
  d->m = needs_x ? (int)n_rhs : 0;
  d->S = (int)S;
  // grid sizes of the widest launches must fit
  const int nt = ceil_div(d->n, kTile);
  const long long widest = (long long)d->B * ((d->N + 1) / 2) * 2 * nt * nt + 1;
  if (!grid_ok(widest)) return SOCU_ERR_UNSUPPORTED;
  return SOCU_OK;
}

int dispatch(socu_op op, socu_dtype dtype, void* L, void* E, void* x, const uint8_t* mask,
             int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, cudaStream_t st,
             long long* count) {
  Dims d;
  const int v = validate(op, dtype, L, E, x, batch, horizon, n, n_rhs, &d);
  if (v != SOCU_OK) return v;
  if (d.B == 0) {
    if (count) *count = 0;
    return SOCU_OK;
  }
  if (count == nullptr) {
    const cudaError_t e = ensure_device(L);
    if (e != cudaSuccess) return cuda_status(e);
  }
  if (dtype == SOCU_FLOAT64)
    return enqueue<double>(op, make_problem<double>(L, E, x, mask, d), st, count);
  return enqueue<float>(op, make_problem<float>(L, E, x, mask, d), st, count);
}

}  // namespace
}  // namespace socu

using namespace socu;

struct socu_launch_s {
  socu_op op;
  socu_dtype dtype;
  void *L, *E, *x;
  const uint8_t* mask;
  int64_t batch, horizon, n, n_rhs;
  long long kernels;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};

extern "C" {

const char* socu_version(void) { return "socu_b200 0.1.0 (sm_100a)"; }

const char* socu_status_string(int status) {
  switch (status) {
    case SOCU_OK: return "ok";
    case SOCU_ERR_INVALID_ARGUMENT: return "invalid argument";
    case SOCU_ERR_CUDA: return "CUDA error";
    case SOCU_ERR_UNSUPPORTED: return "unsupported problem size";
    case SOCU_ERR_TIMEOUT: return "device wait timed out";
    default: return "unknown status";
  }
}

int socu_last_cuda_error(void) { return g_last_cuda_error; }

int64_t socu_recursive_iterations(int64_t horizon) {
  if (horizon <= 0) return -1;
  int64_t k = 0;
  while (horizon) {
    ++k;
    horizon >>= 1;
  }
  return k;
}

int64_t socu_off_diag_storage_len(int64_t horizon) {
  if (horizon <= 0) return -1;
  const int64_t K = socu_recursive_iterations(horizon);
  int64_t total = 0;
  for (int64_t l = 0; l < K; ++l) total += (horizon >> l) - 1;
  return total;
}

int64_t socu_max_block_size(socu_dtype dtype, int64_t n_rhs) {
  const size_t es = dtype == SOCU_FLOAT64 ? sizeof(double) : sizeof(float);
  const int m = n_rhs > 0 ? (int)(n_rhs < kMC ? n_rhs : kMC) : 0;
  const long long limit = max_smem_optin();
  int64_t best = 0;
  for (int n = 1; n <= 512; ++n) {
    long long need = smem_diag_elems(n, m);
    const long long c = smem_couple_elems(n), u = smem_update_elems(n), s = smem_sweep_elems(n, m > 0 ? m : 1);
    if (c > need) need = c;
    if (u > need) need = u;
    if (s > need) need = s;
    if (need * (long long)es <= limit) best = n;
  }
  return best;
}

int socu_cholesky_factor(socu_dtype dtype, void* L, void* E, const uint8_t* mask, int64_t batch,
                         int64_t horizon, int64_t n, void* stream) {
  return dispatch(SOCU_OP_FACTOR, dtype, L, E, nullptr, mask, batch, horizon, n, 0,
                  static_cast<cudaStream_t>(stream), nullptr);
}

int socu_cholesky_factor_and_solve(socu_dtype dtype, void* L, void* E, void* x, const uint8_t* mask,
                                   int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs,
                                   void* stream) {
  return dispatch(SOCU_OP_FACTOR_AND_SOLVE, dtype, L, E, x, mask, batch, horizon, n, n_rhs,
                  static_cast<cudaStream_t>(stream), nullptr);
}

int socu_cholesky_forward_substitution(socu_dtype dtype, const void* L, const void* E, void* x,
                                       const uint8_t* mask, int64_t batch, int64_t horizon,
                                       int64_t n, int64_t n_rhs, void* stream) {
  return dispatch(SOCU_OP_FORWARD_SUBSTITUTION, dtype, const_cast<void*>(L), const_cast<void*>(E), x,
                  mask, batch, horizon, n, n_rhs, static_cast<cudaStream_t>(stream), nullptr);
}

int socu_cholesky_backward_substitution(socu_dtype dtype, const void* L, const void* E, void* x,
                                        const uint8_t* mask, int64_t batch, int64_t horizon,
                                        int64_t n, int64_t n_rhs, void* stream) {
  return dispatch(SOCU_OP_BACKWARD_SUBSTITUTION, dtype, const_cast<void*>(L), const_cast<void*>(E), x,
                  mask, batch, horizon, n, n_rhs, static_cast<cudaStream_t>(stream), nullptr);
}

int socu_cholesky_solve(socu_dtype dtype, const void* L, const void* E, void* x, const uint8_t* mask,
                        int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, void* stream) {
  return dispatch(SOCU_OP_SOLVE, dtype, const_cast<void*>(L), const_cast<void*>(E), x, mask, batch,
                  horizon, n, n_rhs, static_cast<cudaStream_t>(stream), nullptr);
}

int socu_launch_create(socu_launch_t* out, socu_op op, socu_dtype dtype, void* L, void* E, void* x,
                       const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs,
                       int use_cuda_graph, void* stream) {
  if (out == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  long long kernels = 0;
  int st = dispatch(op, dtype, L, E, x, mask, batch, horizon, n, n_rhs, nullptr, &kernels);
  if (st != SOCU_OK) return st;
  socu_launch_s* h = new (std::nothrow) socu_launch_s();
  if (!h) return SOCU_ERR_UNSUPPORTED;
  h->op = op;
  h->dtype = dtype;
  h->L = L;
  h->E = E;
  h->x = x;
  h->mask = mask;
  h->batch = batch;
  h->horizon = horizon;
  h->n = n;
  h->n_rhs = n_rhs;
  h->kernels = kernels;
  h->graph = nullptr;
  h->exec = nullptr;
  if (use_cuda_graph && batch > 0) {
    const cudaError_t ed = ensure_device(L);
    if (ed != cudaSuccess) {
      delete h;
      return cuda_status(ed);
    }
    // Capture on a private stream (the legacy default stream cannot capture),
    // then instantiate eagerly so the first run is a single graph launch.
    cudaStream_t cap = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      st = dispatch(op, dtype, L, E, x, mask, batch, horizon, n, n_rhs, cap, nullptr);
      cudaGraph_t g = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(cap, &g);
      if (st == SOCU_OK && e2 != cudaSuccess) st = cuda_status(e2);
      h->graph = g;
      if (st == SOCU_OK) st = cuda_status(cudaGraphInstantiate(&h->exec, g, 0));
    } else {
      st = cuda_status(e);
    }
    if (cap) cudaStreamDestroy(cap);
    if (st != SOCU_OK) {
      if (h->exec) cudaGraphExecDestroy(h->exec);
      if (h->graph) cudaGraphDestroy(h->graph);
      delete h;
      return st;
    }
    (void)stream;
  }
  *out = h;
  return SOCU_OK;
}

int socu_launch_run(socu_launch_t h, void* stream) {
  if (h == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (h->exec) return cuda_status(cudaGraphLaunch(h->exec, st));
  return dispatch(h->op, h->dtype, h->L, h->E, h->x, h->mask, h->batch, h->horizon, h->n, h->n_rhs, st,
                  nullptr);
}

int64_t socu_launch_kernel_count(socu_launch_t h) { return h ? h->kernels : 0; }

int socu_launch_destroy(socu_launch_t h) {
  if (h == nullptr) return SOCU_OK;
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  delete h;
  return SOCU_OK;
}

}  // extern "C"
