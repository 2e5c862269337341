// C ABI of socu_b200: argument validation, level scheduling, kernel enqueue,
// and launch objects with optional CUDA-graph capture.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

#include "../../include/socu_b200.h"
#include "grad.cuh"
#include "ragged.cuh"
#include "tc_node.cuh"
#include "tc_update.cuh"
#include "top_sweep.cuh"

namespace socu {
namespace {

thread_local int g_last_cuda_error = 0;
thread_local int g_last_cuda_line = 0;   // source line of the call that reported it (diagnostics)

int cuda_status_line(cudaError_t e, int line) {
  if (e == cudaSuccess) return SOCU_OK;
  g_last_cuda_error = static_cast<int>(e);
  g_last_cuda_line = line;
  return SOCU_ERR_CUDA;
}
#define cuda_status(e) cuda_status_line((e), __LINE__)

// Level schedule of a horizon-N system (socu/block_tridiag_solver.py:869-914),
// written to a caller array of kMaxLevels entries (no heap: the no-allocation
// entry point shares this path).  Returns the number of levels K.
constexpr int kMaxLevels = 32;   // horizon <= 2^30
struct Schedule {
  Level lv[kMaxLevels];
  int K = 0;
  const Level& operator[](int l) const { return lv[l]; }
};

void schedule(int N, Schedule* out) {
  int s = 1, prev = 0, curr = 0, nxt = N - 1;
  const int K = static_cast<int>(socu_recursive_iterations(N));
  out->K = K;
  for (int l = 0; l < K; ++l) {
    Level& lv = out->lv[l];
    lv.s = s;
    lv.d = (N + s) / (2 * s);
    lv.oc = curr;
    lv.on = nxt;
    lv.op = prev;
    lv.tc = 0;
    lv.tile = kTile;
    lv.pre = 0;
    s *= 2;
    prev = curr;
    curr = nxt;
    nxt += N / s - 1;
  }
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

// Small fixed-capacity caches of per-kernel driver queries (static storage,
// no heap: every solve path, the no-allocation entry point included, uses
// them).  A full table just stops caching; lookups stay correct.
constexpr int kCacheSlots = 512;

// Opt in to large dynamic shared memory once per kernel, device and size (the
// attribute is per function and device).
struct PrepSlot {
  const void* fn;
  int dev;
  size_t smem;
};
std::mutex g_prep_mu;
PrepSlot g_prepared[kCacheSlots];
int g_n_prepared = 0;

template <typename K>
cudaError_t prepare(K kernel, size_t smem) {
  // the default limit (48 KB) covers dynamic plus static shared memory; keep a
  // margin for the kernels' static __shared__ words
  if (smem <= 40 * 1024) return cudaSuccess;
  int dev = 0;
  cudaGetDevice(&dev);
  const void* fn = reinterpret_cast<const void*>(kernel);
  std::lock_guard<std::mutex> g(g_prep_mu);
  int slot = -1;
  for (int i = 0; i < g_n_prepared; ++i)
    if (g_prepared[i].fn == fn && g_prepared[i].dev == dev) {
      if (g_prepared[i].smem >= smem) return cudaSuccess;
      slot = i;
      break;
    }
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  if (slot < 0 && g_n_prepared < kCacheSlots) slot = g_n_prepared++;
  if (slot >= 0) g_prepared[slot] = PrepSlot{fn, dev, smem};
  return e;
}

// Threads per CTA for a node launch: 128 instead of 256 when the narrower
// CTAs (twice as many resident per SM) finish the level in fewer waves, as on
// the wide bottom level of the float factor (measured: 80 -> 70 us for 512
// n = 64 nodes; the Schur-update launches lose more per CTA than the waves
// save and keep 256).  Occupancies are cached per kernel, device,
// shared-memory size and thread count.
struct OccSlot {
  const void* fn;
  int dev;
  size_t smem;
  int threads, blocks;
};
std::mutex g_occ_mu;
OccSlot g_occ[kCacheSlots];
int g_n_occ = 0;

template <typename K>
int occupancy(K kernel, int dev, int threads, size_t smem) {
  const void* fn = reinterpret_cast<const void*>(kernel);
  std::lock_guard<std::mutex> g(g_occ_mu);
  for (int i = 0; i < g_n_occ; ++i)
    if (g_occ[i].fn == fn && g_occ[i].dev == dev && g_occ[i].smem == smem && g_occ[i].threads == threads)
      return g_occ[i].blocks;
  int v = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, threads, smem) != cudaSuccess) {
    v = 0;
    (void)cudaGetLastError();   // the fallback path handles it; do not leave the error pending
  }
  if (g_n_occ < kCacheSlots) g_occ[g_n_occ++] = OccSlot{fn, dev, smem, threads, v};
  return v;
}

int sm_count() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 0;
  return sms;
}

template <typename K, class Smem>
int level_threads(K kernel, int nth, long long blocks, Smem smem) {
  if (nth != 256 || blocks <= 0) return nth;
  int dev = 0;
  const int sms = sm_count();
  if (sms <= 0 || cudaGetDevice(&dev) != cudaSuccess) return nth;
  const int o256 = occupancy(kernel, dev, 256, smem(256)), o128 = occupancy(kernel, dev, 128, smem(128));
  if (o256 <= 0 || o128 <= 0) return nth;
  const long long w256 = (blocks + (long long)sms * o256 - 1) / ((long long)sms * o256);
  const long long w128 = (blocks + (long long)sms * o128 - 1) / ((long long)sms * o128);
  return w128 < w256 ? 128 : 256;
}

// ---------------------------------------------------------------------------
// Launch settings.  Built-in heuristics, replaced field by field by a tuned
// entry for (dtype, n, n_rhs) -- or for (dtype, n, any n_rhs), stored with
// n_rhs = 0 -- installed with socu_tuning_set (the autotuner's cache), and by
// a per-launch override (the reference's block_dim / block_size arguments).
// A field of 0 means "not set".
// ---------------------------------------------------------------------------
struct TuneSlot {
  int dtype, n, m;
  socu_tuning t;
};
std::mutex g_tune_mu;
TuneSlot g_tune[kCacheSlots];
int g_n_tune = 0;

bool tuning_valid(const socu_tuning& t) {
  auto thr = [](int v) { return v == 0 || v == 64 || v == 128 || v == 256; };
  return thr(t.node_threads) && thr(t.update_threads) && thr(t.sweep_threads) && t.sweep_tensor_cores >= 0 &&
         t.sweep_tensor_cores <= 2 && (t.update_tile == 0 || t.update_tile == 16 || t.update_tile == 32) &&
         t.ragged_units >= 0 && t.ragged_units <= 64 && t.update_tensor_cores >= 0 && t.update_tensor_cores <= 2 &&
         t.node_tensor_cores >= 0 && t.node_tensor_cores <= 4;
}

void tuning_merge(socu_tuning* into, const socu_tuning& over) {
  if (over.node_threads) into->node_threads = over.node_threads;
  if (over.update_threads) into->update_threads = over.update_threads;
  if (over.sweep_threads) into->sweep_threads = over.sweep_threads;
  if (over.sweep_tensor_cores) into->sweep_tensor_cores = over.sweep_tensor_cores;
  if (over.update_tile) into->update_tile = over.update_tile;
  if (over.ragged_units) into->ragged_units = over.ragged_units;
  if (over.update_tensor_cores) into->update_tensor_cores = over.update_tensor_cores;
  if (over.node_tensor_cores) into->node_tensor_cores = over.node_tensor_cores;
}

// Tuned entry for (dtype, n, m), falling back to (dtype, n, any m); zeros if none.
socu_tuning tuning_lookup(int dtype, int n, int m) {
  socu_tuning out{};
  std::lock_guard<std::mutex> g(g_tune_mu);
  int wild = -1, exact = -1;
  for (int i = 0; i < g_n_tune; ++i) {
    if (g_tune[i].dtype != dtype || g_tune[i].n != n) continue;
    if (g_tune[i].m == m) exact = i;
    else if (g_tune[i].m == 0) wild = i;
  }
  if (wild >= 0) tuning_merge(&out, g_tune[wild].t);
  if (exact >= 0) tuning_merge(&out, g_tune[exact].t);
  return out;
}

// ---------------------------------------------------------------------------
// Profiling runs (socu_launch_profile): an event pair around every kernel
// launch of an eager run, summed per kernel kind afterwards.
// ---------------------------------------------------------------------------
struct Prof {
  std::vector<cudaEvent_t> start, stop;
  std::vector<int> kind;
  cudaError_t err = cudaSuccess;
  int err_kind = -1;    // kernel kind of the first failing launch
  int err_where = -1;   // 0: error pending before that launch, 1: raised by it, 2: event create / record,
                        // 3: a non-launch call of the op, 4: event synchronise / elapsed time
};
// kind and place of the last profiling failure in this thread (socu_profile_error)
thread_local int g_prof_err_kind = -1, g_prof_err_where = -1;
thread_local Prof* g_prof = nullptr;

void prof_mark(cudaStream_t s, bool begin, int kind) {
  if (g_prof == nullptr) return;
  cudaEvent_t e = nullptr;
  cudaError_t r = cudaEventCreate(&e);
  if (r == cudaSuccess) r = cudaEventRecord(e, s);
  if (r != cudaSuccess) {
    if (g_prof->err == cudaSuccess) {
      g_prof->err = r;
      g_prof->err_kind = kind;
      g_prof->err_where = 2;   // event create / record
    }
    if (e) cudaEventDestroy(e);
    return;
  }
  if (begin) {
    g_prof->start.push_back(e);
    g_prof->kind.push_back(kind);
  } else {
    g_prof->stop.push_back(e);
  }
}
inline void prof_begin(cudaStream_t s, int kind) {
  if (g_prof == nullptr) return;
  // a launch error must be charged to the launch that caused it
  const cudaError_t prev = cudaGetLastError();
  if (prev != cudaSuccess && g_prof->err == cudaSuccess) {
    g_prof->err = prev;
    g_prof->err_kind = kind;
    g_prof->err_where = 0;
  }
  prof_mark(s, true, kind);
}
inline void prof_end(cudaStream_t s) {
  if (g_prof == nullptr) return;
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess && g_prof->err == cudaSuccess) {
    g_prof->err = e;
    g_prof->err_kind = g_prof->kind.empty() ? -1 : g_prof->kind.back();
    g_prof->err_where = 1;
  }
  prof_mark(s, false, 0);
}

// Programmatic dependent launch of a kernel that follows another kernel of the
// same op on the same stream: it may start while its predecessor finishes and
// waits (griddepcontrol.wait in the kernel) before it reads the predecessor's
// results.  The first kernel of an op is launched plainly, so it is fully
// ordered after whatever the caller enqueued before.  SOCU_PDL=0 turns
// programmatic launches off.
bool pdl_enabled() {
  static const int on = [] {
    const char* v = std::getenv("SOCU_PDL");
    return (v != nullptr && v[0] == '0') ? 0 : 1;
  }();
  return on != 0;
}

template <typename... KArgs, typename... Args>
void launch(void (*kernel)(KArgs...), unsigned blocks, unsigned threads, size_t smem, cudaStream_t s, bool pdl,
            Args... args) {
  if (!pdl || !pdl_enabled()) {
    kernel<<<blocks, threads, smem, s>>>(args...);
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}

// As launch(), as clusters of `cluster` CTAs along x (blocks a multiple of it).
template <typename... KArgs, typename... Args>
void launch_cluster(void (*kernel)(KArgs...), unsigned blocks, unsigned threads, size_t smem, cudaStream_t s,
                    bool pdl, int cluster, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(blocks);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[2];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  int na = 1;
  if (pdl && pdl_enabled()) {
    attr[1].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[1].val.programmaticStreamSerializationAllowed = 1;
    na = 2;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Clusters of `cluster` CTAs (threads, smem each) that fit the device at once,
// cached per kernel, device and shape; 0 when the query fails (no device, or
// the size is not supported).
struct ClusterSlot {
  const void* fn;
  int dev, cluster, threads;
  size_t smem;
  int fits;
};
std::mutex g_cluster_mu;
ClusterSlot g_cluster[kCacheSlots];
int g_n_cluster = 0;

template <typename K>
int cluster_capacity(K kernel, int cluster, int threads, size_t smem) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  const void* fn = reinterpret_cast<const void*>(kernel);
  {
    std::lock_guard<std::mutex> g(g_cluster_mu);
    for (int i = 0; i < g_n_cluster; ++i)
      if (g_cluster[i].fn == fn && g_cluster[i].dev == dev && g_cluster[i].cluster == cluster &&
          g_cluster[i].threads == threads && g_cluster[i].smem == smem)
        return g_cluster[i].fits;
  }
  int fits = 0;
  cudaError_t e = prepare(kernel, smem);
  if (e == cudaSuccess && cluster > 8) e = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)cluster);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaOccupancyMaxActiveClusters(&fits, kernel, &cfg);
  }
  if (e != cudaSuccess) {
    fits = 0;
    (void)cudaGetLastError();   // a refused size only means "no cluster kernel"
  }
  std::lock_guard<std::mutex> g(g_cluster_mu);
  if (g_n_cluster < kCacheSlots) g_cluster[g_n_cluster++] = ClusterSlot{fn, dev, cluster, threads, smem, fits};
  return fits;
}

// SOCU_TOP_SWEEP=1 runs the top levels of the sweeps in the cluster-resident
// k_top instead of one launch per level.  Off by default: measured on B200,
// the per-level launches of a graph (programmatic dependent launch, blocks
// loaded before the dependency wait) are faster at every shape tried -- a
// float solve on an inverse-carrying factor at N=1024, n=64, m=8 takes 132 us
// with a launch per level vs 153 us with k_top, at N=20, n=16, m=1 29 vs 35 us
// (one k_top launch instead of ten): the cluster barrier and the L2 reads of
// the vectors after it cost more per level than a kernel boundary.
bool top_sweep_enabled() {
  static const int on = [] {
    const char* v = std::getenv("SOCU_TOP_SWEEP");
    return (v != nullptr && v[0] == '1') ? 1 : 0;
  }();
  return on != 0;
}

// ---------------------------------------------------------------------------
// TMA tensor maps of the resident sweeps.  cuTensorMapEncodeTiled is a
// driver-API call; it is resolved through the runtime's entry-point query, so
// the library does not link against libcuda.  SOCU_TMA=0 keeps the sweeps on
// per-thread cp.async copies.
// ---------------------------------------------------------------------------
using TmaEncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

TmaEncodeFn tma_encoder() {
  static const TmaEncodeFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &f, 12000, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess || f == nullptr) {
      (void)cudaGetLastError();
      return static_cast<TmaEncodeFn>(nullptr);
    }
    return reinterpret_cast<TmaEncodeFn>(f);
  }();
  return fn;
}

bool tma_enabled() {
  static const int on = [] {
    const char* v = std::getenv("SOCU_TMA");
    return (v != nullptr && v[0] == '0') ? 0 : 1;
  }();
  return on != 0;
}

// 4-D map {cols, rows, count, batch} of an array of row-major rows x cols
// tiles (batch entries batch_stride elements apart), box {box_cols, rows, 1, 1}.
// false when an alignment rule of the TMA unit is not met (the caller then
// copies with cp.async): base, row, tile and batch strides on 16 bytes, box
// rows of a multiple of 16 bytes, box extents <= 256.
bool encode_tiles(CUtensorMap* map, const void* base, int es, int cols, int rows, long long count, int batch,
                  long long batch_stride, int box_cols) {
  const TmaEncodeFn enc = tma_encoder();
  if (enc == nullptr || base == nullptr || cols < 1 || rows < 1 || count < 1 || batch < 1) return false;
  const unsigned long long row_b = (unsigned long long)cols * es, tile_b = row_b * (unsigned long long)rows;
  const unsigned long long batch_b =
      (unsigned long long)(batch > 1 ? batch_stride : count * rows * (long long)cols) * (unsigned long long)es;
  if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0 || (row_b & 15u) != 0 || (tile_b & 15u) != 0 ||
      (batch_b & 15u) != 0 || batch_b == 0)
    return false;
  if (box_cols < 1 || box_cols > 256 || rows > 256 || ((long long)box_cols * es) % 16 != 0) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)cols, (cuuint64_t)rows, (cuuint64_t)count, (cuuint64_t)batch};
  const cuuint64_t strides[3] = {row_b, tile_b, batch_b};
  const cuuint32_t box[4] = {(cuuint32_t)box_cols, (cuuint32_t)rows, 1u, 1u};
  const cuuint32_t estr[4] = {1u, 1u, 1u, 1u};
  return enc(map, es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4,
             const_cast<void*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Maps of one op's resident sweeps: factor / coupling blocks with the padded
// block row (res_ldm), vector chunks with the padded vector row (res_ldy).
template <typename T>
SweepMaps sweep_maps(const Problem<T>& p) {
  SweepMaps m;
  std::memset(&m, 0, sizeof m);
  // (the sweeps wait for their block copies in the first vector chunk)
  if (!tma_enabled() || p.m <= 0 || p.X == nullptr) return m;
  constexpr int es = sizeof(T);
  const int ldm = res_ldm(p.n);
  m.blocks = encode_tiles(&m.L, p.L, es, p.n, p.n, p.N, p.B, p.sL, ldm) &&
             (p.S == 0 || encode_tiles(&m.E, p.E, es, p.n, p.n, p.S, p.B, p.sE, ldm));
  m.vecs = p.X != nullptr && p.m > 0 &&
           encode_tiles(&m.X, p.X, es, p.m, p.n, p.N, p.B, p.sX, res_ldy(std::min(p.m, kMC)));
  return m;
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
  p.info = nullptr;
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

// Whether a factor may carry its diagonal inverses (k_node<INV>) for
// matvec-based sweeps: small blocks whose sweeps run resident.
template <typename T>
bool use_inverse(int n, int m) {
  return n <= 64 && (long long)smem_sweep_res_elems(n, m > 0 ? m : 1) * (long long)sizeof(T) <=
                        (long long)max_smem_optin();
}

// Second stream and two events for graph capture: inside factor_and_solve,
// each level's forward pull runs on a parallel branch beside the Schur update
// (both only depend on the level's node kernel).
struct Fork {
  cudaStream_t aux = nullptr;
  cudaEvent_t split = nullptr, join = nullptr;
  bool ok() const { return aux && split && join; }
  int create() {
    cudaError_t e = cudaStreamCreateWithFlags(&aux, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&split, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join, cudaEventDisableTiming);
    return cuda_status(e);
  }
  void destroy() {
    if (aux) cudaStreamDestroy(aux);
    if (split) cudaEventDestroy(split);
    if (join) cudaEventDestroy(join);
    aux = nullptr;
    split = join = nullptr;
  }
};

// Block-row FP64 residual (n <= 128): 1, 2 or 4 eight-column groups of
// right-hand sides per pass over the matrix blocks, by n_rhs.
template <bool REFINE>
cudaError_t launch_residual_rows(const RefineArgs& a, cudaStream_t st, bool pdl) {
  const int gr = residual_groups(a.m);
  const size_t smem = smem_residual_x_elems(a.n, gr) * sizeof(double);
  const unsigned blocks = (unsigned)((long long)a.B * a.N), threads = (unsigned)residual_rows_threads(a.n, a.m);
  cudaError_t e;
  if (gr == 1) {
    e = prepare(k_residual_rows<REFINE, 1>, smem);
    if (e == cudaSuccess) launch(k_residual_rows<REFINE, 1>, blocks, threads, smem, st, pdl, a);
  } else if (gr == 2) {
    e = prepare(k_residual_rows<REFINE, 2>, smem);
    if (e == cudaSuccess) launch(k_residual_rows<REFINE, 2>, blocks, threads, smem, st, pdl, a);
  } else {
    e = prepare(k_residual_rows<REFINE, 4>, smem);
    if (e == cudaSuccess) launch(k_residual_rows<REFINE, 4>, blocks, threads, smem, st, pdl, a);
  }
  return e;
}

// Enqueue (or count, when st == nullptr and count != nullptr) the kernels of one op.
// inv: the factor carries (FACTOR, FACTOR_AND_SOLVE) or has (SOLVE) its
// diagonal inverses; only for internal factors or within factor_and_solve.
// fork (graph capture only): run the forward pulls on a parallel branch.
// over: per-launch settings (block_dim / block_size), on top of the tuned table.
template <typename T>
int enqueue(socu_op op, const Problem<T>& p, cudaStream_t st, long long* count, bool inv = false,
            const Fork* fork = nullptr, const socu_tuning* over = nullptr) {
  const int n = p.n, nth = threads_for(n);
  socu_tuning cfg = tuning_lookup(sizeof(T) == 8 ? SOCU_FLOAT64 : SOCU_FLOAT32, n, p.m);
  if (over) tuning_merge(&cfg, *over);
  const int tile = cfg.update_tile ? cfg.update_tile : kTile;
  Schedule lv;
  schedule(p.N, &lv);
  const int K = lv.K;
  for (int l = 0; l < K; ++l) lv.lv[l].tile = tile;
  const bool withY = op == SOCU_OP_FACTOR_AND_SOLVE;
  // node shared memory by CTA size (the register-resident chain's buffers only where it runs)
  auto node_smem = [&](int threads) {
    return (size_t)smem_node_launch_elems(n, withY ? p.m : 0, sizeof(T), threads) * sizeof(T);
  };
  const size_t sd = node_smem(256);   // the largest
  const size_t su = smem_update_launch_elems(n, sizeof(T), tile) * sizeof(T);
  const int mm = p.m > 0 ? p.m : 1;
  const bool res = (long long)smem_sweep_res_elems(n, mm) * (long long)sizeof(T) <= (long long)max_smem_optin();
  const size_t ss = (res ? smem_sweep_res_elems(n, mm) : smem_sweep_elems(n, mm)) * sizeof(T);
  inv = inv && res && n <= 64;
  auto node_kernel = withY ? (inv ? k_node<T, true, true> : k_node<T, true, false>)
                           : (inv ? k_node<T, false, true> : k_node<T, false, false>);
  auto fwd_kernel = res ? (inv ? k_fwd<T, true, false, true> : k_fwd<T, true>) : k_fwd<T, false>;
  auto pull_kernel = res ? k_fwd<T, true, true> : k_fwd<T, false, true>;
  auto bwd_kernel = res ? (inv ? k_bwd<T, true, true> : k_bwd<T, true>) : k_bwd<T, false>;
  // Schur updates of float factors on the tcgen05 tensor cores (3xTF32), on
  // request: the FP64-pipe updates (exact products of the float operands,
  // FP64 sums) keep the float factor accurate enough for the reference's
  // float tolerances and for three refinement rounds instead of five
  const bool upd_tc = sizeof(T) == 4 && update_tc_ok(n) && cfg.update_tensor_cores == 1;
  const size_t su_tc = (size_t)smem_update_tc_bytes(n);
  // products of float level nodes on the tcgen05 tensor cores: on request
  // (node_tensor_cores = 1) at every level, or with node_tensor_cores = 3 only
  // on levels wide enough to be throughput-bound (at least 4 nodes per SM),
  // where the SIMT products cost more issue slots than the MMA round trips
  const bool node_tc_any = sizeof(T) == 4 && node_tc_ok(n, withY ? p.m : 0) &&
                           (cfg.node_tensor_cores == 1 || cfg.node_tensor_cores == 3) &&
                           (long long)smem_node_tc_bytes(n, withY ? p.m : 0) <= (long long)max_smem_optin();
  const bool node_tc_wide_only = cfg.node_tensor_cores == 3;
  const size_t sd_tc = (size_t)smem_node_tc_bytes(n, withY ? p.m : 0);
  auto node_tc_kernel = withY ? (inv ? k_node_tc<true, true> : k_node_tc<true, false>)
                              : (inv ? k_node_tc<false, true> : k_node_tc<false, false>);
  // float level nodes with 64 < n <= 128 resident in tensor memory, trailing
  // updates of the blocked factor on the tensor cores (node_tensor_cores = 4)
  const int m_node = withY ? p.m : 0;
  const bool node_tm = sizeof(T) == 4 && !inv && cfg.node_tensor_cores == 4 && node_tm_ok(n, m_node) &&
                       smem_node_tm_bytes(n, m_node) <= (long long)max_smem_optin();
  const size_t sd_tm = (size_t)smem_node_tm_bytes(n, m_node);
  auto node_tm_kernel = withY ? k_node_tm<true> : k_node_tm<false>;
  long long launches = 0;
  const bool run = count == nullptr;
  const int sms = run ? sm_count() : 0;
  const int upd_thr = cfg.update_threads ? cfg.update_threads : nth;
  const int swp_thr = cfg.sweep_threads ? cfg.sweep_threads : nth;

  if (run) {
    cudaError_t e = cudaSuccess;
    if (op == SOCU_OP_FACTOR || op == SOCU_OP_FACTOR_AND_SOLVE) {
      e = prepare(node_kernel, sd);
      if (e == cudaSuccess) e = update_uses_big(n) ? prepare(k_update_big<T>, su) : prepare(k_update<T>, su);
      if (e == cudaSuccess && upd_tc) e = prepare(k_update_tc, su_tc);
      if (e == cudaSuccess && node_tc_any) e = prepare(node_tc_kernel, sd_tc);
      if (e == cudaSuccess && node_tm) e = prepare(node_tm_kernel, sd_tm);
    }
    if (e == cudaSuccess) e = prepare(fwd_kernel, ss);
    if (e == cudaSuccess) e = prepare(pull_kernel, ss);
    if (e == cudaSuccess) e = prepare(bwd_kernel, ss);
    if (e != cudaSuccess) return cuda_status(e);
  }

  // sweep products on inverse-carrying float factors: tensor cores when the
  // launch is wider than the resident sweep CTAs (3 per SM), or as tuned
  // pre: the level's factor blocks were final before the previous kernel
  // started (any sweep over a stored factor, and every backward level of
  // factor_and_solve but the first), so they may be loaded before the wait
  auto sweep_level = [&](const Level& L, long long blocks, bool pre) {
    Level o = L;
    if (cfg.sweep_tensor_cores == 1) o.tc = 1;
    else if (cfg.sweep_tensor_cores == 2) o.tc = 0;
    else o.tc = sms > 0 && blocks > 3LL * sms;
    o.pre = pre ? 1 : 0;
    return o;
  };
  // programmatic launches inside the op's chain on its own stream (not the
  // first kernel, not the forked branch, not while profiling with events)
  bool first = true;
  auto go_on = [&](cudaStream_t s, auto kernel, int kind, long long blocks, size_t smem, const Level& L,
                   int threads, auto... extra) {
    if (blocks <= 0) return;
    ++launches;
    if (!run) return;
    const bool pdl = !first && s == st && g_prof == nullptr;
    first = false;
    prof_begin(s, kind);
    launch(kernel, (unsigned)blocks, (unsigned)threads, smem, s, pdl, p, L, extra...);
    prof_end(s);
  };
  // TMA maps of the resident sweeps (zeros: cp.async copies)
  SweepMaps maps;
  std::memset(&maps, 0, sizeof maps);
  if (run && res) maps = sweep_maps(p);
  auto node_threads = [&](long long blocks) {
    if (cfg.node_threads) return cfg.node_threads;
    return run ? level_threads(node_kernel, nth, blocks, node_smem) : nth;
  };
  const bool forked = run && fork != nullptr && fork->ok();

  // On request (SOCU_TOP_SWEEP=1), the top levels of the sweeps in one
  // cluster-resident kernel (k_top): the forward levels with at most `cluster`
  // tasks and the backward levels with at most `cluster` nodes, one cluster per
  // instance, when every instance's cluster fits the device at once (otherwise
  // the per-level launches parallelise better).  The decision needs the device;
  // without one (counting on a host without a GPU) every level keeps its own
  // launch.
  const bool want_fwd = op == SOCU_OP_FORWARD_SUBSTITUTION || op == SOCU_OP_SOLVE;
  const bool want_bwd =
      op == SOCU_OP_BACKWARD_SUBSTITUTION || op == SOCU_OP_SOLVE || op == SOCU_OP_FACTOR_AND_SOLVE;
  auto top_kernel = inv ? k_top<T, true> : k_top<T, false>;
  TopLevels top;
  std::memset(&top, 0, sizeof top);
  int top_cluster = 0;
  size_t top_smem = 0;
  const int top_thr = swp_thr;
  if (res && p.m > 0 && top_sweep_enabled() && (want_fwd || want_bwd)) {
    for (int stages = 2; stages >= 1 && top_smem == 0; --stages) {
      const size_t bytes = (size_t)smem_top_elems(n, p.m, stages) * sizeof(T);
      if (bytes <= (size_t)max_smem_optin()) {
        top_smem = bytes;
        top.stages = stages;
      }
    }
    for (int cl = 16; top_smem > 0 && cl >= 4 && top_cluster == 0; cl /= 2) {
      int flo = K, blo = K;
      if (want_fwd)
        while (flo > 0 && K - flo < kTopMaxLevels && fwd_tasks(p.N, lv[flo - 1]) <= cl) --flo;
      if (want_bwd)
        while (blo > 0 && K - blo < kTopMaxLevels && lv[blo - 1].d <= cl) --blo;
      if ((K - flo) + (K - blo) < 2) break;
      int widest = 1;
      for (int l = flo; l < K; ++l) widest = std::max(widest, fwd_tasks(p.N, lv[l]));
      for (int l = blo; l < K; ++l) widest = std::max(widest, lv[l].d);
      int c = 1;
      while (c < widest) c *= 2;
      if (cluster_capacity(top_kernel, c, top_thr, top_smem) < p.B) continue;
      top_cluster = c;
      top.fwd_lo = flo;
      top.fwd_n = K - flo;
      top.bwd_lo = blo;
      top.bwd_n = K - blo;
      top.pre = op != SOCU_OP_FACTOR_AND_SOLVE ? 1 : 0;
      for (int l = flo; l < K; ++l)
        top.fl[l - flo] = sweep_level(lv[l], (long long)p.B * fwd_tasks(p.N, lv[l]), true);
      for (int l = blo; l < K; ++l) top.bl[l - blo] = sweep_level(lv[l], (long long)p.B * lv[l].d, true);
    }
  }
  auto go_top = [&]() {
    ++launches;
    if (!run) return;
    const bool pdl = !first && g_prof == nullptr;
    first = false;
    prof_begin(st, top.bwd_n > 0 ? SOCU_KIND_BACKWARD : SOCU_KIND_FORWARD);
    launch_cluster(top_kernel, (unsigned)((long long)p.B * top_cluster), (unsigned)top_thr, top_smem, st, pdl,
                   top_cluster, p, top, maps);
    prof_end(st);
  };

  const bool factor = op == SOCU_OP_FACTOR || op == SOCU_OP_FACTOR_AND_SOLVE;
  if (factor && p.info != nullptr) {
    ++launches;
    if (run) {
      prof_begin(st, SOCU_KIND_NODE);
      k_info_reset<<<(p.B + 255) / 256 < 1024 ? (p.B + 255) / 256 : 1024, 256, 0, st>>>(p.info, p.B);
      prof_end(st);
      first = false;
    }
  }
  if (factor) {
    for (int l = 0; l < K; ++l) {
      const Level& L = lv[l];
      const long long node_blocks = (long long)p.B * L.d;
      if constexpr (sizeof(T) == 4) {
        const bool node_tc = node_tc_any && (!node_tc_wide_only || node_blocks >= 4LL * sms);
        // inverse-first nodes on levels that fit one wave of CTAs with the W^T
        // buffer: the chain also writes W^T and the products run from it
        auto node_wt_kernel = withY ? (inv ? k_node<float, true, true, true> : k_node<float, true, false, true>)
                                    : (inv ? k_node<float, false, true, true> : k_node<float, false, false, true>);
        const size_t sd_wt = (size_t)smem_node_gemm_elems(n, withY ? p.m : 0, 4, true) * 4;
        const int nthr = node_threads(node_blocks);
        bool node_wt = false;
        if (run && !node_tm && !node_tc && node_uses_gemm(n) && reg_chain_ok(n, nthr) &&
            sd_wt <= (size_t)max_smem_optin() && sms > 0 && prepare(node_wt_kernel, sd_wt) == cudaSuccess) {
          int dev = 0;
          cudaGetDevice(&dev);
          node_wt = (long long)occupancy(node_wt_kernel, dev, nthr, sd_wt) * sms >= node_blocks;
        }
        if (node_tm)
          go_on(st, node_tm_kernel, SOCU_KIND_NODE, node_blocks, sd_tm, L, 256);
        else if (node_tc)
          go_on(st, node_tc_kernel, SOCU_KIND_NODE, node_blocks, sd_tc, L, 256);
        else if (node_wt)
          go_on(st, node_wt_kernel, SOCU_KIND_NODE, node_blocks, sd_wt, L, nthr);
        else
          go_on(st, node_kernel, SOCU_KIND_NODE, node_blocks, node_smem(nthr), L, nthr);
      } else {
        {
          const int nthr = node_threads(node_blocks);
          go_on(st, node_kernel, SOCU_KIND_NODE, node_blocks, node_smem(nthr), L, nthr);
        }
      }
      if (l + 1 < K) {
        // fused forward: apply this level's updates to every target vector
        const long long pull_blocks = withY ? (long long)p.B * (p.N / lv[l + 1].s) : 0;
        const Level PL = sweep_level(lv[l + 1], pull_blocks, false);
        if (forked && pull_blocks > 0) {
          cudaEventRecord(fork->split, st);
          cudaStreamWaitEvent(fork->aux, fork->split, 0);
          go_on(fork->aux, pull_kernel, SOCU_KIND_PULL, pull_blocks, ss, PL, swp_thr, maps);
          cudaEventRecord(fork->join, fork->aux);
        }
        const long long upd_blocks = (long long)p.B * update_launch_tasks(n, p.N, L);
        bool tc_done = false;
        if constexpr (sizeof(T) == 4) {
          if (upd_tc) {
            go_on(st, k_update_tc, SOCU_KIND_UPDATE, (long long)p.B * update_blocks(p.N, L), su_tc, L, 256);
            tc_done = true;
          }
        }
        if (!tc_done) {
          if (update_uses_big(n))
            go_on(st, k_update_big<T>, SOCU_KIND_UPDATE, upd_blocks, su, L, 256);
          else
            go_on(st, k_update<T>, SOCU_KIND_UPDATE, upd_blocks, su, L, upd_thr);
        }
        if (forked && pull_blocks > 0) {
          cudaStreamWaitEvent(st, fork->join, 0);
          first = true;   // the next node waits for the forked branch in full
        } else
          go_on(st, pull_kernel, SOCU_KIND_PULL, pull_blocks, ss, PL, swp_thr, maps);
      }
    }
  }
  if (op == SOCU_OP_FORWARD_SUBSTITUTION || op == SOCU_OP_SOLVE) {
    for (int l = 0; l < (top_cluster ? top.fwd_lo : K); ++l) {
      const long long blocks = (long long)p.B * (l == 0 ? lv[l].d : p.N / lv[l].s);
      go_on(st, fwd_kernel, SOCU_KIND_FORWARD, blocks, ss, sweep_level(lv[l], blocks, true), swp_thr, maps);
    }
  }
  if (top_cluster) go_top();
  if (op == SOCU_OP_BACKWARD_SUBSTITUTION || op == SOCU_OP_SOLVE || op == SOCU_OP_FACTOR_AND_SOLVE) {
    for (int l = (top_cluster ? top.bwd_lo : K) - 1; l >= 0; --l) {
      const long long blocks = (long long)p.B * lv[l].d;
      go_on(st, bwd_kernel, SOCU_KIND_BACKWARD, blocks, ss,
            sweep_level(lv[l], blocks, op != SOCU_OP_FACTOR_AND_SOLVE || l != K - 1), swp_thr, maps);
    }
  }
  if (count) *count = launches;
  if (run) return cuda_status(cudaGetLastError());
  return SOCU_OK;
}

// The *_INV extension ops run the base op on a factor that carries W^T.
socu_op base_op(socu_op op, bool* inv) {
  *inv = (int)op >= (int)SOCU_OP_FACTOR_INV;
  switch (op) {
    case SOCU_OP_FACTOR_INV: return SOCU_OP_FACTOR;
    case SOCU_OP_FORWARD_INV: return SOCU_OP_FORWARD_SUBSTITUTION;
    case SOCU_OP_BACKWARD_INV: return SOCU_OP_BACKWARD_SUBSTITUTION;
    case SOCU_OP_SOLVE_INV: return SOCU_OP_SOLVE;
    default: return op;
  }
}

int validate(socu_op op, socu_dtype dtype, const void* L, const void* E, const void* x,
             int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, Dims* d) {
  if (dtype != SOCU_FLOAT32 && dtype != SOCU_FLOAT64) return SOCU_ERR_INVALID_ARGUMENT;
  if ((int)op < 0 || (int)op > 8) return SOCU_ERR_INVALID_ARGUMENT;
  bool inv_op = false;
  op = base_op(op, &inv_op);
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
  if (inv_op) {
    const int mm = needs_x ? (int)n_rhs : 1;
    const bool ok = dtype == SOCU_FLOAT64 ? use_inverse<double>((int)n, mm) : use_inverse<float>((int)n, mm);
    if (!ok) return SOCU_ERR_UNSUPPORTED;
  }
  d->B = (int)batch;
  d->N = (int)horizon;
  d->n = (int)n;
  d->m = needs_x ? (int)n_rhs : 0;
  d->S = (int)S;
  // grid sizes of the widest launches must fit (smallest update tile: 16)
  const int nt = ceil_div(d->n, 16);
  const long long per_node = 2LL * nt * nt + 1;
  const long long widest = (long long)d->B * ((d->N + 1) / 2) * per_node + 1;
  if (!grid_ok(widest)) return SOCU_ERR_UNSUPPORTED;
  return SOCU_OK;
}

int dispatch(socu_op op, socu_dtype dtype, void* L, void* E, void* x, const uint8_t* mask,
             int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, cudaStream_t st,
             long long* count, const Fork* fork = nullptr, const socu_tuning* over = nullptr,
             int32_t* info = nullptr) {
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
  // factor_and_solve keeps the diagonal inverses in the (unspecified) upper
  // triangles of L and uses them for its own backward sweep; the *_INV ops
  // keep or use them on request
  bool inv = false;
  op = base_op(op, &inv);
  inv = inv || op == SOCU_OP_FACTOR_AND_SOLVE;
  if (dtype == SOCU_FLOAT64) {
    Problem<double> p = make_problem<double>(L, E, x, mask, d);
    p.info = info;
    return enqueue<double>(op, p, st, count, inv, fork, over);
  }
  Problem<float> p = make_problem<float>(L, E, x, mask, d);
  p.info = info;
  return enqueue<float>(op, p, st, count, inv, fork, over);
}


// ---------------------------------------------------------------------------
// mixed precision + FP64 refinement
// ---------------------------------------------------------------------------
size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct RefineLayout {
  size_t l32, e32, r32, active, state, any, total;
};

RefineLayout refine_layout(int64_t B, int64_t N, int64_t n, int64_t m) {
  RefineLayout o;
  const int64_t S = socu_off_diag_storage_len(N);
  size_t off = 0;
  o.l32 = off; off += align256((size_t)B * N * n * n * sizeof(float));
  o.e32 = off; off += align256((size_t)B * (S > 0 ? S : 0) * n * n * sizeof(float));
  o.r32 = off; off += align256((size_t)B * N * n * m * sizeof(float));
  o.active = off; off += align256((size_t)B);
  o.state = off; off += align256((size_t)B * sizeof(RefineState));
  o.any = off; off += align256(sizeof(int));
  o.total = off;
  return o;
}

// Fallback workspace: the refinement workspace, then the FP64 working copies.
struct FallbackLayout {
  size_t l64, e64, fb, any, total;
};

FallbackLayout fallback_layout(int64_t B, int64_t N, int64_t n, int64_t m) {
  FallbackLayout o;
  const int64_t S = socu_off_diag_storage_len(N);
  size_t off = refine_layout(B, N, n, m).total;
  o.l64 = off; off += align256((size_t)B * N * n * n * sizeof(double));
  o.e64 = off; off += align256((size_t)B * (S > 0 ? S : 0) * n * n * sizeof(double));
  o.fb = off; off += align256((size_t)B);
  o.any = off; off += align256(sizeof(int));
  o.total = off;
  return o;
}

int refine_validate(const void* L, const void* E, const void* b, void* x, int64_t batch, int64_t horizon,
                    int64_t n, int64_t n_rhs, int max_iter, double tol, void* ws, size_t ws_bytes,
                    const double* eta, const int32_t* iters, Dims* d) {
  const int v = validate(SOCU_OP_SOLVE, SOCU_FLOAT32, L, E, x, batch, horizon, n, n_rhs, d);
  if (v != SOCU_OK) return v;
  if (max_iter < 1 || max_iter > 1000 || !(tol >= 0.0)) return SOCU_ERR_INVALID_ARGUMENT;
  if (batch > 0 && (b == nullptr || eta == nullptr || iters == nullptr)) return SOCU_ERR_INVALID_ARGUMENT;
  if ((long long)smem_residual_elems(d->n) * (long long)sizeof(double) > (long long)max_smem_optin())
    return SOCU_ERR_UNSUPPORTED;
  const RefineLayout lay = refine_layout(batch, horizon, n, n_rhs);
  if (batch > 0 && (ws == nullptr || ws_bytes < lay.total || (reinterpret_cast<uintptr_t>(ws) & 255) != 0))
    return SOCU_ERR_INVALID_ARGUMENT;
  return SOCU_OK;
}

RefineArgs refine_args(const double* L, const double* E, const double* b, double* x, const uint8_t* mask,
                       const Dims& d, int max_iter, double tol, void* ws, double* eta, int32_t* iters) {
  const RefineLayout lay = refine_layout(d.B, d.N, d.n, d.m);
  char* w = static_cast<char*>(ws);
  RefineArgs a;
  a.L = L; a.E = E; a.b = b; a.x = x; a.mask = mask;
  a.L32 = reinterpret_cast<float*>(w + lay.l32);
  a.E32 = reinterpret_cast<float*>(w + lay.e32);
  a.R32 = reinterpret_cast<float*>(w + lay.r32);
  a.active = reinterpret_cast<uint8_t*>(w + lay.active);
  a.st = reinterpret_cast<RefineState*>(w + lay.state);
  a.any_active = reinterpret_cast<int*>(w + lay.any);
  a.eta = eta; a.iters = iters; a.rout = nullptr;
  a.B = d.B; a.N = d.N; a.n = d.n; a.m = d.m; a.S = d.S;
  a.tol = tol; a.max_iter = max_iter;
  a.check_in_residual = 0;
  return a;
}

// One refinement round after a solve that left delta in R32: x += delta,
// FP64 residual (R32 = r, norms), convergence test.
// x += delta, then the residual, whose last CTA per instance also runs the
// convergence test (RefineArgs::check_in_residual)
int refine_finish_round(const RefineArgs& a, cudaStream_t st, long long* count) {
  if (count == nullptr) {
    const long long nvec = (long long)a.B * a.N * a.n * a.m;
    const int upd_blocks = (int)((nvec + 255) / 256 < 148 * 16 ? (nvec + 255) / 256 : 148 * 16);
    const int nrc = ceil_div(a.n, kResRows);
    // each kernel follows the previous one of the round on the same stream
    const bool pdl = g_prof == nullptr;
    prof_begin(st, SOCU_KIND_REFINE_UPDATE);
    launch(k_ref_update, (unsigned)upd_blocks, 256, 0, st, pdl, a);
    prof_end(st);
    RefineArgs ac = a;
    ac.check_in_residual = 1;
    prof_begin(st, SOCU_KIND_RESIDUAL);
    if (residual_uses_rows(a.n)) {
      const cudaError_t e = launch_residual_rows<true>(ac, st, pdl);
      if (e != cudaSuccess) return cuda_status(e);
    } else
      launch(k_residual<true>, (unsigned)((long long)a.B * a.N * nrc), 256, smem_residual_elems(a.n) * sizeof(double),
             st, pdl, ac);
    prof_end(st);
  } else {
    *count = 2;
  }
  return SOCU_OK;
}

// Mixed solve, part 1: state reset, float copies, norms, then the first
// round fused into the float factor: factor_and_solve on R32 = b gives
// delta = x_1, followed by x += delta, the FP64 residual and the test.
int refine_prologue(const RefineArgs& a, cudaStream_t st, long long* count, const Fork* fork = nullptr) {
  const bool run = count == nullptr;
  Dims d{a.B, a.N, a.n, a.m, a.S};
  Problem<float> pf = make_problem<float>(a.L32, a.E32, a.R32, a.active, d);
  const int chk_blocks = (a.B + 255) / 256;
  if (run) {
    const size_t sres = smem_residual_elems(a.n) * sizeof(double);
    const size_t sinit = smem_ref_init_elems(a.n) * sizeof(double);
    cudaError_t e = prepare(k_residual<true>, sres);
    if (e != cudaSuccess) return cuda_status(e);
    prof_begin(st, SOCU_KIND_REFINE_SETUP);
    k_ref_reset<<<chk_blocks, 256, 0, st>>>(a);
    prof_end(st);
    const unsigned init_blocks = (unsigned)((long long)a.B * (a.N > a.S ? a.N : a.S));
    prof_begin(st, SOCU_KIND_REFINE_SETUP);
    if (residual_uses_rows(a.n))
      k_ref_init_rows<<<init_blocks, 256, sinit, st>>>(a);
    else
      k_ref_init<<<init_blocks, 256, 0, st>>>(a);
    prof_end(st);
    e = cudaMemsetAsync(a.any_active, 0, sizeof(int), st);   // the first test decides
    if (e != cudaSuccess) return cuda_status(e);
  }
  long long c = 0, cr = 0;
  // the float factor of the mixed solve takes its Schur updates on the tcgen05
  // tensor cores for 64 < n <= 128 unless the tuned table says otherwise: the
  // 3xTF32 products cost accuracy the FP64 refinement wins back (measured at
  // N=16384, n=128, m=32: factor 27.0 -> 23.9 ms, still two rounds)
  socu_tuning mixed{};
  if (a.n > 64 && update_tc_ok(a.n) && tuning_lookup(SOCU_FLOAT32, a.n, a.m).update_tensor_cores == 0)
    mixed.update_tensor_cores = 1;
  int s = enqueue<float>(SOCU_OP_FACTOR_AND_SOLVE, pf, st, run ? nullptr : &c, use_inverse<float>(a.n, a.m), fork,
                         &mixed);
  if (s != SOCU_OK) return s;
  s = refine_finish_round(a, st, run ? nullptr : &cr);
  if (count) *count = 2 + c + cr;
  return s;
}

// Mixed solve, part 2: one further refinement round (float solve of R32,
// x update, FP64 residual, convergence test).
int refine_iteration(const RefineArgs& a, cudaStream_t st, long long* count) {
  const bool run = count == nullptr;
  Dims d{a.B, a.N, a.n, a.m, a.S};
  Problem<float> pf = make_problem<float>(a.L32, a.E32, a.R32, a.active, d);
  long long c = 0, cr = 0;
  int s = enqueue<float>(SOCU_OP_SOLVE, pf, st, run ? nullptr : &c, use_inverse<float>(a.n, a.m));
  if (s != SOCU_OK) return s;
  s = refine_finish_round(a, st, run ? nullptr : &cr);
  if (count) *count = c + cr;
  return s;
}

// Enqueue (or count) the full mixed solve with a fixed max_iter rounds
// (converged instances skip their work inside each round).
int refine_enqueue(const RefineArgs& a, cudaStream_t st, long long* count) {
  const bool run = count == nullptr;
  long long cp = 0, ci = 0;
  int s = refine_prologue(a, st, run ? nullptr : &cp);
  if (s != SOCU_OK) return s;
  for (int it = 1; it < a.max_iter; ++it) {
    s = refine_iteration(a, st, run ? nullptr : &ci);
    if (s != SOCU_OK) return s;
    if (!run) break;
  }
  if (count) *count = cp + ci * (a.max_iter - 1);
  if (run) return cuda_status(cudaGetLastError());
  return SOCU_OK;
}

// Capture the mixed solve into a graph whose refinement rounds sit in a
// conditional WHILE node: the loop stops as soon as every instance has
// converged (or hit max_iter), instead of launching max_iter rounds.
// FP64 fallback stage, appended after the loop: select, IF node (copy, FP64
// factor_and_solve, residual, eta).
int capture_fallback(const RefineArgs& a, const FallbackArgs& f, cudaStream_t cap, cudaStream_t body) {
  cudaStreamCaptureStatus cs;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  cudaGraph_t g = nullptr;
  cudaGraphConditionalHandle hnd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(cap, &cs, nullptr, &g, &deps, &nd);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hnd, g, 0, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) e = cudaMemsetAsync(f.any, 0, sizeof(int), cap);
  if (e != cudaSuccess) return cuda_status(e);
  const int chk_blocks = (a.B + 255) / 256;
  k_fb_select<<<chk_blocks, 256, 0, cap>>>(a, f);
  k_fb_decide<<<1, 1, 0, cap>>>(hnd, f.any);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(cap, &cs, nullptr, &g, &deps, &nd);
  cudaGraphNodeParams prm = {};
  prm.type = cudaGraphNodeTypeConditional;
  prm.conditional.handle = hnd;
  prm.conditional.type = cudaGraphCondTypeIf;
  prm.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, deps, nd, &prm);
  if (e == cudaSuccess) e = cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies);
  if (e == cudaSuccess)
    e = cudaStreamBeginCaptureToGraph(body, prm.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_status(e);
  const unsigned copy_blocks = (unsigned)((long long)a.B * (a.N > a.S ? a.N : a.S));
  k_fb_copy<<<copy_blocks, 256, 0, body>>>(a, f);
  const Dims d{a.B, a.N, a.n, a.m, a.S};
  int st = enqueue<double>(SOCU_OP_FACTOR_AND_SOLVE, make_problem<double>(f.L64, f.E64, a.x, f.fb, d), body, nullptr,
                           true);
  RefineArgs ra = a;
  ra.active = f.fb;
  if (st == SOCU_OK) {
    if (residual_uses_rows(a.n))
      launch_residual_rows<true>(ra, body, false);
    else
      k_residual<true><<<(unsigned)((long long)a.B * a.N * ceil_div(a.n, kResRows)), 256,
                         smem_residual_elems(a.n) * sizeof(double), body>>>(ra);
    k_fb_eta<<<chk_blocks, 256, 0, body>>>(a, f);
  }
  cudaGraph_t bg = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(body, &bg);
  if (st == SOCU_OK) st = cuda_status(e2 != cudaSuccess ? e2 : cudaGetLastError());
  return st;
}

int capture_refine_while(const RefineArgs& a, cudaGraph_t* out, const FallbackArgs* fallback = nullptr) {
  cudaStream_t cap = nullptr, body = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&body, cudaStreamNonBlocking);
  int st = cuda_status(e);
  bool capturing = false;
  if (st == SOCU_OK) {
    e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    st = cuda_status(e);
    capturing = st == SOCU_OK;
  }
  Fork fork;
  if (st == SOCU_OK) st = fork.create();
  if (st == SOCU_OK) st = refine_prologue(a, cap, nullptr, &fork);
  cudaGraph_t g = nullptr;
  cudaGraphConditionalHandle hnd = 0;
  cudaGraphNode_t node = nullptr;
  cudaGraph_t bodyg = nullptr;
  if (st == SOCU_OK) {
    // the handle is created first so that the test after the fused first
    // round (upstream of the loop) can set it: a solve that converged after
    // one round never enters the loop
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    e = cudaStreamGetCaptureInfo(cap, &cs, nullptr, &g, &deps, &nd);
    if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&hnd, g, 0, cudaGraphCondAssignDefault);
    if (e == cudaSuccess) {
      k_ref_decide<<<1, 1, 0, cap>>>(hnd, a.any_active);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamGetCaptureInfo(cap, &cs, nullptr, &g, &deps, &nd);
    cudaGraphNodeParams prm = {};
    prm.type = cudaGraphNodeTypeConditional;
    prm.conditional.handle = hnd;
    prm.conditional.type = cudaGraphCondTypeWhile;
    prm.conditional.size = 1;
    if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, deps, nd, &prm);
    if (e == cudaSuccess) {
      bodyg = prm.conditional.phGraph_out[0];
      e = cudaStreamUpdateCaptureDependencies(cap, &node, 1, cudaStreamSetCaptureDependencies);
    }
    st = cuda_status(e);
  }
  if (st == SOCU_OK) {
    e = cudaStreamBeginCaptureToGraph(body, bodyg, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    st = cuda_status(e);
    if (st == SOCU_OK) {
      st = refine_iteration(a, body, nullptr);
      if (st == SOCU_OK) k_ref_decide<<<1, 1, 0, body>>>(hnd, a.any_active);
      cudaGraph_t bg = nullptr;
      const cudaError_t e2 = cudaStreamEndCapture(body, &bg);
      if (st == SOCU_OK) st = cuda_status(e2 != cudaSuccess ? e2 : cudaGetLastError());
    }
  }
  if (st == SOCU_OK && fallback != nullptr) st = capture_fallback(a, *fallback, cap, body);
  cudaGraph_t fin = nullptr;
  if (capturing) {
    const cudaError_t e3 = cudaStreamEndCapture(cap, &fin);
    if (st == SOCU_OK && e3 != cudaSuccess) st = cuda_status(e3);
  }
  if (cap) cudaStreamDestroy(cap);
  if (body) cudaStreamDestroy(body);
  fork.destroy();
  if (st != SOCU_OK) {
    if (fin) cudaGraphDestroy(fin);
    return st;
  }
  *out = fin;
  return SOCU_OK;
}
}  // namespace
}  // namespace socu

using namespace socu;

// A ragged batch: per-instance descriptors, the device work queue and (for
// the mixed path) the float workspace, all allocated once at creation.
struct socu_ragged_s {
  int dtype = SOCU_FLOAT64;
  bool refine = false;
  int max_iter = 0;
  int count = 0;
  int device = 0;
  std::vector<RgInst> inst;
  long long tot[3] = {0, 0, 0};   // elements of the packed L, E, x arrays
  RgInst* d_inst = nullptr;
  unsigned long long* d_slot = nullptr;
  unsigned long long* d_init = nullptr;
  unsigned int* d_ctr = nullptr;  // head, tail, done
  int* d_rem = nullptr;
  int* d_err = nullptr;
  unsigned int n_init = 0, capacity = 0;
  std::vector<unsigned long long> init;   // host copy of the queue's initial contents
  long long timeout_ns = 0;
  float* d_w32 = nullptr;         // refinement: L32 | E32 | R32
  size_t w_off[3] = {0, 0, 0};
  RefineState* d_state = nullptr;
  int vc = 0, grid = 0;
  size_t smem = 0;
};

struct socu_launch_s {
  socu_op op;
  socu_dtype dtype;
  void *L, *E, *x;
  const uint8_t* mask;
  int64_t batch, horizon, n, n_rhs;
  long long kernels;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  bool refine = false;
  RefineArgs ra{};
  long long round_kernels = 0;   // graph WHILE loop: kernels per refinement round
  socu_ragged_s* rg = nullptr;   // ragged batch (b, tol, eta, iters below for its mixed path)
  const double* b = nullptr;
  double tol = 0.0;
  double* eta = nullptr;
  int32_t* iters = nullptr;
  socu_tuning over{};               // per-launch settings (block_dim / block_size)
  int32_t* info = nullptr;          // per-instance factor status (factor ops), may be null
};

namespace {
// ---------------------------------------------------------------------------
// ragged batches
// ---------------------------------------------------------------------------
constexpr int kRgMaxBlock = 64;                 // resident sweeps with diagonal inverses
constexpr long long kRgTimeoutNs = 4000000000LL;   // bound of one queue wait (4 s)

int rg_upc(int n) { return n <= 8 ? 8 : (n <= 16 ? 4 : (n <= 32 ? 2 : 1)); }

// Per-instance descriptors and packed offsets, in instance order.
int rg_layout(const int64_t* horizon, const int64_t* n, const int64_t* n_rhs, int64_t count,
              std::vector<RgInst>* out, long long tot[3], int dtype = SOCU_FLOAT64) {
  if (count < 0) return SOCU_ERR_INVALID_ARGUMENT;
  if (count >= (1LL << kRgInstBits)) return SOCU_ERR_UNSUPPORTED;
  if (count > 0 && (horizon == nullptr || n == nullptr || n_rhs == nullptr)) return SOCU_ERR_INVALID_ARGUMENT;
  long long oL = 0, oE = 0, oX = 0;
  if (out) out->clear();
  for (int64_t i = 0; i < count; ++i) {
    if (horizon[i] <= 0 || n[i] <= 0 || n_rhs[i] <= 0) return SOCU_ERR_INVALID_ARGUMENT;
    if (n[i] > kRgMaxBlock || horizon[i] > (1 << 22) || n_rhs[i] > (1 << 20)) return SOCU_ERR_UNSUPPORTED;
    RgInst I;
    I.N = (int)horizon[i];
    I.n = (int)n[i];
    I.m = (int)n_rhs[i];
    I.S = (int)socu_off_diag_storage_len(horizon[i]);
    I.K = (int)socu_recursive_iterations(horizon[i]);
    const int tu = tuning_lookup(dtype, I.n, I.m).ragged_units;
    I.upc = tu > 0 ? tu : rg_upc(I.n);
    I.oL = oL;
    I.oE = oE;
    I.oX = oX;
    oL += (long long)I.N * I.n * I.n;
    oE += (long long)I.S * I.n * I.n;
    oX += (long long)I.N * I.n * I.m;
    if (out) out->push_back(I);
  }
  tot[0] = oL;
  tot[1] = oE;
  tot[2] = oX;
  return SOCU_OK;
}

void rg_free(socu_ragged_s* r) {
  cudaFree(r->d_inst);
  cudaFree(r->d_slot);
  cudaFree(r->d_init);
  cudaFree(r->d_ctr);
  cudaFree(r->d_rem);
  cudaFree(r->d_err);
  cudaFree(r->d_w32);
  cudaFree(r->d_state);
}

template <typename T, int MODE>
int rg_prepare_kernel(socu_ragged_s* r) {
  auto kern = k_ragged<T, MODE>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)r->smem);
  int per_sm = 0, sms = 0;
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kRgThreads, r->smem);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, r->device);
  if (e != cudaSuccess) return cuda_status(e);
  if (per_sm < 1) return SOCU_ERR_UNSUPPORTED;
  r->grid = per_sm * sms;
  return SOCU_OK;
}

int rg_create(socu_ragged_s* r, const int64_t* horizon, const int64_t* n, const int64_t* n_rhs, int64_t count) {
  int st = rg_layout(horizon, n, n_rhs, count, &r->inst, r->tot, r->refine ? SOCU_FLOAT32 : r->dtype);
  if (st != SOCU_OK) return st;
  r->count = (int)count;
  if (count == 0) return SOCU_OK;
  const int mode = r->refine ? kRgRefine : kRgPlain;
  const int es = r->refine ? 4 : (r->dtype == SOCU_FLOAT64 ? 8 : 4);
  // queue capacity: every chunk of every phase (max_iter rounds when refining)
  long long cap = 0;
  int maxn = 1, maxm = 1, maxnv = 1;
  for (const RgInst& I : r->inst) {
    const int phases = r->refine ? rg_refine_phases(I.K, r->max_iter) : rg_plain_phases(I.K);
    if (phases >= (1 << kRgPhaseBits)) return SOCU_ERR_UNSUPPORTED;
    for (int ph = 0; ph < phases; ++ph) cap += rg_chunks(rg_phase(I, mode, ph));
    maxn = std::max(maxn, I.n);
    maxm = std::max(maxm, I.m);
    maxnv = std::max(maxnv, 3 * I.n + I.m);
  }
  // first-phase chunks, largest instances first
  std::vector<int> order(r->inst.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
    const RgInst &A = r->inst[a], &B = r->inst[b];
    return (double)A.N * A.n * A.n * A.n > (double)B.N * B.n * B.n * B.n;
  });
  std::vector<unsigned long long>& init = r->init;
  init.clear();
  for (int i : order) {
    const int c = rg_chunks(rg_phase(r->inst[i], mode, 0));
    for (int j = 0; j < c; ++j) init.push_back(rg_encode(i, 0, j));
  }
  // shared memory: the largest body at the largest block size (n <= 64: the
  // inverse-first node body)
  r->vc = maxnv;
  size_t smem = (size_t)smem_node_gemm_elems(maxn, maxm, es, false, false) * es;   // ragged nodes: shared-memory chain (measured faster there)
  smem = std::max(smem, (size_t)smem_update_full_elems(maxn, es) * es);
  smem = std::max(smem, (size_t)smem_sweep_res_elems(maxn, maxm) * es);
  if (r->refine) smem = std::max(smem, (size_t)smem_residual_rows_elems(maxn) * sizeof(double));
  if ((long long)smem > (long long)max_smem_optin()) return SOCU_ERR_UNSUPPORTED;
  r->smem = smem;
  cudaError_t e = cudaGetDevice(&r->device);
  if (e != cudaSuccess) return cuda_status(e);
  if (r->refine) st = rg_prepare_kernel<float, kRgRefine>(r);
  else if (r->dtype == SOCU_FLOAT64) st = rg_prepare_kernel<double, kRgPlain>(r);
  else st = rg_prepare_kernel<float, kRgPlain>(r);
  if (st != SOCU_OK) return st;
  cap += r->grid + 64;
  if (cap >= (1LL << 31)) return SOCU_ERR_UNSUPPORTED;
  r->capacity = (unsigned)cap;
  r->n_init = (unsigned)init.size();
  e = cudaMalloc(&r->d_inst, sizeof(RgInst) * r->inst.size());
  if (e == cudaSuccess) e = cudaMalloc(&r->d_slot, sizeof(unsigned long long) * r->capacity);
  if (e == cudaSuccess) e = cudaMalloc(&r->d_init, sizeof(unsigned long long) * init.size());
  if (e == cudaSuccess) e = cudaMalloc(&r->d_ctr, 4 * sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMalloc(&r->d_rem, sizeof(int) * r->inst.size());
  if (e == cudaSuccess) e = cudaMalloc(&r->d_err, sizeof(int));
  if (e == cudaSuccess)
    e = cudaMemcpy(r->d_inst, r->inst.data(), sizeof(RgInst) * r->inst.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(r->d_init, init.data(), sizeof(unsigned long long) * init.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(r->d_err, 0, sizeof(int));
  if (e == cudaSuccess && r->refine) {
    r->w_off[0] = 0;
    r->w_off[1] = align256((size_t)r->tot[0] * sizeof(float));
    r->w_off[2] = r->w_off[1] + align256((size_t)r->tot[1] * sizeof(float));
    const size_t bytes = r->w_off[2] + align256((size_t)r->tot[2] * sizeof(float));
    e = cudaMalloc(&r->d_w32, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&r->d_state, sizeof(RefineState) * r->inst.size());
  }
  if (e != cudaSuccess) return cuda_status(e);
  return SOCU_OK;
}

template <typename T, int MODE>
int rg_launch(socu_ragged_s* r, RgArgs<T> a, cudaStream_t st) {
  a.inst = r->d_inst;
  a.count = r->count;
  a.q.slot = r->d_slot;
  a.q.head = r->d_ctr;
  a.q.tail = r->d_ctr + 1;
  a.q.done = r->d_ctr + 2;
  a.q.rem = r->d_rem;
  a.q.error = r->d_err;
  a.q.init = r->d_init;
  a.q.n_init = r->n_init;
  a.q.capacity = r->capacity;
  a.vc = r->vc;
  a.timeout_ns = r->timeout_ns > 0 ? r->timeout_ns : kRgTimeoutNs;
  cudaError_t e = cudaMemsetAsync(r->d_slot + r->n_init, 0,
                                  sizeof(unsigned long long) * (r->capacity - r->n_init), st);
  if (e != cudaSuccess) return cuda_status(e);
  const long long work = std::max<long long>(r->n_init, r->count);
  const int sb = (int)std::min<long long>((work + 255) / 256, 1024);
  prof_begin(st, SOCU_KIND_RAGGED);
  k_rg_start<T, MODE><<<sb, 256, 0, st>>>(a);
  k_ragged<T, MODE><<<r->grid, kRgThreads, r->smem, st>>>(a);
  prof_end(st);
  return cuda_status(cudaGetLastError());
}

int rg_device(const socu_ragged_s* r) {
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != r->device) return cuda_status(cudaSetDevice(r->device));
  return SOCU_OK;
}

int rg_factor_and_solve(socu_ragged_s* r, void* L, void* E, void* x, cudaStream_t st) {
  if (r->refine) return SOCU_ERR_INVALID_ARGUMENT;
  if (r->count == 0) return SOCU_OK;
  if (L == nullptr || x == nullptr || (r->tot[1] > 0 && E == nullptr)) return SOCU_ERR_INVALID_ARGUMENT;
  int s = rg_device(r);
  if (s != SOCU_OK) return s;
  if (r->dtype == SOCU_FLOAT64) {
    RgArgs<double> a{};
    a.L = static_cast<double*>(L);
    a.E = static_cast<double*>(E);
    a.X = static_cast<double*>(x);
    return rg_launch<double, kRgPlain>(r, a, st);
  }
  RgArgs<float> a{};
  a.L = static_cast<float*>(L);
  a.E = static_cast<float*>(E);
  a.X = static_cast<float*>(x);
  return rg_launch<float, kRgPlain>(r, a, st);
}

int rg_refine_solve(socu_ragged_s* r, const double* L, const double* E, const double* b, double* x, double tol,
                    double* eta, int32_t* iters, cudaStream_t st) {
  if (!r->refine || !(tol >= 0.0)) return SOCU_ERR_INVALID_ARGUMENT;
  if (r->count == 0) return SOCU_OK;
  if (L == nullptr || b == nullptr || x == nullptr || eta == nullptr || iters == nullptr ||
      (r->tot[1] > 0 && E == nullptr))
    return SOCU_ERR_INVALID_ARGUMENT;
  int s = rg_device(r);
  if (s != SOCU_OK) return s;
  char* w = reinterpret_cast<char*>(r->d_w32);
  RgArgs<float> a{};
  a.L = reinterpret_cast<float*>(w + r->w_off[0]);
  a.E = reinterpret_cast<float*>(w + r->w_off[1]);
  a.X = reinterpret_cast<float*>(w + r->w_off[2]);
  a.L64 = L;
  a.E64 = E;
  a.b64 = b;
  a.x64 = x;
  a.st = r->d_state;
  a.eta = eta;
  a.iters = iters;
  a.tol = tol;
  a.max_iter = r->max_iter;
  return rg_launch<float, kRgRefine>(r, a, st);
}

// enqueue one run of a launch object on `st` (fork: graph capture only)
int launch_enqueue(socu_launch_s* h, cudaStream_t st, const Fork* fork = nullptr) {
  if (h->rg) {
    if (h->rg->refine)
      return rg_refine_solve(h->rg, static_cast<const double*>(h->L), static_cast<const double*>(h->E), h->b,
                             static_cast<double*>(h->x), h->tol, h->eta, h->iters, st);
    return rg_factor_and_solve(h->rg, h->L, h->E, h->x, st);
  }
  if (h->refine) {
    if (h->batch == 0) return SOCU_OK;
    const cudaError_t e = ensure_device(h->L);
    if (e != cudaSuccess) return cuda_status(e);
    return refine_enqueue(h->ra, st, nullptr);
  }
  return dispatch(h->op, h->dtype, h->L, h->E, h->x, h->mask, h->batch, h->horizon, h->n, h->n_rhs, st, nullptr,
                  fork, &h->over, h->info);
}

// Capture one run into a CUDA graph on a private stream (the legacy default
// stream cannot capture) and instantiate it eagerly.
int capture(socu_launch_s* h) {
  if (h->rg) {
    const int sd = rg_device(h->rg);
    if (sd != SOCU_OK) return sd;
  } else {
    const cudaError_t ed = ensure_device(h->L);
    if (ed != cudaSuccess) return cuda_status(ed);
  }
  cudaStream_t cap = nullptr;
  cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
  int st = SOCU_OK;
  Fork fork;
  if (e == cudaSuccess && fork.create() != SOCU_OK) e = static_cast<cudaError_t>(g_last_cuda_error);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = launch_enqueue(h, cap, &fork);
    cudaGraph_t g = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(cap, &g);
    if (st == SOCU_OK && e2 != cudaSuccess) st = cuda_status(e2);
    h->graph = g;
    if (st == SOCU_OK) st = cuda_status(cudaGraphInstantiate(&h->exec, g, 0));
  } else {
    st = cuda_status(e);
  }
  if (cap) cudaStreamDestroy(cap);
  fork.destroy();
  if (st != SOCU_OK) {
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->exec = nullptr;
    h->graph = nullptr;
  }
  return st;
}
}  // namespace


// ---------------------------------------------------------------------------
// Refined solve without any allocation.
//
// Some callers cannot allocate device memory while they solve: an XLA/JAX
// custom call receives its buffers from XLA's allocator and must not call
// cudaMalloc inside the handler; a real-time MPC loop forbids allocation
// after start-up because cudaMalloc/cudaFree can block for an unbounded time
// and synchronise the device; and cudaMalloc is not allowed while a stream
// is being captured into a CUDA graph.  For them the float factor, the
// correction vector and the per-instance refinement state live in the fixed
// array below instead of a caller workspace.  The host side uses only stack
// and static storage.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;   // == SOCU_NOALLOC_SCRATCH_BYTES
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device (with that device current) and cached.
int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_status(e);
  if (dev < 0 || dev >= kMaxDevices) return SOCU_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e);
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return SOCU_OK;
}

}  // namespace

extern "C" {

const char* socu_version(void) { return "socu_b200 0.1.0 (sm_100a)"; }

const char* socu_status_string(int status) {
  switch (status) {
    case SOCU_OK: return "ok";
    case SOCU_ERR_INVALID_ARGUMENT: return "invalid argument";
    case SOCU_ERR_CUDA: return "CUDA error";
    case SOCU_ERR_UNSUPPORTED: return "unsupported problem size";
    case SOCU_ERR_TIMEOUT: return "device wait timed out";
    case SOCU_ERR_SCRATCH_TOO_SMALL:
      return "problem needs more scratch than the fixed no-allocation array holds (SOCU_NOALLOC_SCRATCH_BYTES)";
    default: return "unknown status";
  }
}

int socu_last_cuda_error(void) { return g_last_cuda_error; }

int socu_last_cuda_error_line(void) { return g_last_cuda_line; }

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
    long long need = smem_node_elems(n, (int)es);
    const long long u = smem_update_elems(n, (int)es), s = smem_sweep_elems(n, m > 0 ? m : 1);
    if (u > need) need = u;
    if (s > need) need = s;
    if (need * (long long)es <= limit && n <= 128) best = n;
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

int socu_cholesky_run(socu_op op, socu_dtype dtype, void* L, void* E, void* x, const uint8_t* mask, int64_t batch,
                      int64_t horizon, int64_t n, int64_t n_rhs, void* stream) {
  return dispatch(op, dtype, L, E, x, mask, batch, horizon, n, n_rhs, static_cast<cudaStream_t>(stream), nullptr);
}

int socu_cholesky_run_info(socu_op op, socu_dtype dtype, void* L, void* E, void* x, const uint8_t* mask,
                           int32_t* info, int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, void* stream) {
  bool inv_op = false;
  const socu_op bop = base_op(op, &inv_op);
  if (info == nullptr && batch > 0) return SOCU_ERR_INVALID_ARGUMENT;
  if (bop != SOCU_OP_FACTOR && bop != SOCU_OP_FACTOR_AND_SOLVE) return SOCU_ERR_INVALID_ARGUMENT;
  return dispatch(op, dtype, L, E, x, mask, batch, horizon, n, n_rhs, static_cast<cudaStream_t>(stream), nullptr,
                  nullptr, nullptr, info);
}

int socu_launch_create(socu_launch_t* out, socu_op op, socu_dtype dtype, void* L, void* E, void* x,
                       const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs,
                       int use_cuda_graph, void* stream) {
  return socu_launch_create_tuned(out, op, dtype, L, E, x, mask, batch, horizon, n, n_rhs, use_cuda_graph, nullptr,
                                  stream);
}

int socu_launch_create_tuned(socu_launch_t* out, socu_op op, socu_dtype dtype, void* L, void* E, void* x,
                             const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs,
                             int use_cuda_graph, const socu_tuning* settings, void* stream) {
  return socu_launch_create_ex(out, op, dtype, L, E, x, mask, nullptr, batch, horizon, n, n_rhs, use_cuda_graph,
                               settings, stream);
}

int socu_launch_create_ex(socu_launch_t* out, socu_op op, socu_dtype dtype, void* L, void* E, void* x,
                          const uint8_t* mask, int32_t* info, int64_t batch, int64_t horizon, int64_t n,
                          int64_t n_rhs, int use_cuda_graph, const socu_tuning* settings, void* stream) {
  if (out == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (settings && !tuning_valid(*settings)) return SOCU_ERR_INVALID_ARGUMENT;
  bool inv_op = false;
  const socu_op bop = base_op(op, &inv_op);
  if (info != nullptr && bop != SOCU_OP_FACTOR && bop != SOCU_OP_FACTOR_AND_SOLVE) return SOCU_ERR_INVALID_ARGUMENT;
  long long kernels = 0;
  int st = dispatch(op, dtype, L, E, x, mask, batch, horizon, n, n_rhs, nullptr, &kernels, nullptr, settings, info);
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
  if (settings) h->over = *settings;
  h->info = info;
  if (use_cuda_graph && batch > 0) {
    st = capture(h);
    if (st != SOCU_OK) {
      delete h;
      return st;
    }
  }
  (void)stream;
  *out = h;
  return SOCU_OK;
}

int socu_launch_run(socu_launch_t h, void* stream) {
  if (h == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (h->exec) return cuda_status(cudaGraphLaunch(h->exec, st));
  return launch_enqueue(h, st);
}

int64_t socu_launch_kernel_count(socu_launch_t h) { return h ? h->kernels : 0; }

int64_t socu_launch_round_kernel_count(socu_launch_t h) { return h ? h->round_kernels : 0; }

size_t socu_refine_workspace_bytes(int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs) {
  if (batch < 0 || horizon <= 0 || n <= 0 || n_rhs <= 0) return 0;
  return refine_layout(batch, horizon, n, n_rhs).total;
}

int socu_refine_solve(const double* L, const double* E, const double* b, double* x, const uint8_t* mask,
                      int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, int max_iter, double tol,
                      void* workspace, size_t workspace_bytes, double* eta, int32_t* iters, void* stream) {
  Dims d;
  int v = refine_validate(L, E, b, x, batch, horizon, n, n_rhs, max_iter, tol, workspace, workspace_bytes, eta,
                          iters, &d);
  if (v != SOCU_OK || batch == 0) return v;
  const cudaError_t e = ensure_device(L);
  if (e != cudaSuccess) return cuda_status(e);
  const RefineArgs a = refine_args(L, E, b, x, mask, d, max_iter, tol, workspace, eta, iters);
  return refine_enqueue(a, static_cast<cudaStream_t>(stream), nullptr);
}

int socu_block_tridiag_grad(socu_dtype dtype, const void* x, const void* g, void* dD, void* dE, int64_t batch,
                            int64_t horizon, int64_t n, int64_t n_rhs, int64_t e_blocks, void* stream) {
  if (dtype != SOCU_FLOAT32 && dtype != SOCU_FLOAT64) return SOCU_ERR_INVALID_ARGUMENT;
  if (batch < 0 || horizon <= 0 || n <= 0 || n_rhs <= 0 || e_blocks < 0) return SOCU_ERR_INVALID_ARGUMENT;
  if (e_blocks < horizon - 1) return SOCU_ERR_INVALID_ARGUMENT;
  if (batch == 0) return SOCU_OK;
  if (x == nullptr || g == nullptr || dD == nullptr || (e_blocks > 0 && dE == nullptr)) return SOCU_ERR_INVALID_ARGUMENT;
  const size_t es = dtype == SOCU_FLOAT64 ? 8 : 4;
  const size_t smem = smem_grad_elems((int)n, (int)n_rhs) * es;
  if ((long long)smem > (long long)max_smem_optin()) return SOCU_ERR_UNSUPPORTED;
  const long long blocks = batch * (horizon > e_blocks ? horizon : e_blocks);
  if (!grid_ok(blocks)) return SOCU_ERR_UNSUPPORTED;
  cudaError_t e = ensure_device(x);
  if (e != cudaSuccess) return cuda_status(e);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (dtype == SOCU_FLOAT64) {
    GradArgs<double> a{static_cast<const double*>(x), static_cast<const double*>(g), static_cast<double*>(dD),
                       static_cast<double*>(dE), (int)batch, (int)horizon, (int)n, (int)n_rhs, (int)e_blocks};
    e = prepare(k_grad<double>, smem);
    if (e == cudaSuccess) k_grad<double><<<(unsigned)blocks, 256, smem, st>>>(a);
  } else {
    GradArgs<float> a{static_cast<const float*>(x), static_cast<const float*>(g), static_cast<float*>(dD),
                      static_cast<float*>(dE), (int)batch, (int)horizon, (int)n, (int)n_rhs, (int)e_blocks};
    e = prepare(k_grad<float>, smem);
    if (e == cudaSuccess) k_grad<float><<<(unsigned)blocks, 256, smem, st>>>(a);
  }
  return cuda_status(e != cudaSuccess ? e : cudaGetLastError());
}

constexpr int64_t kLowerBand = 16;

int64_t socu_lower_blocks_bytes(int64_t count, int64_t n, int64_t elem_bytes) {
  if (count < 0 || n <= 0 || elem_bytes <= 0) return 0;
  int64_t per = 0;
  for (int64_t r0 = 0; r0 < n; r0 += kLowerBand) {
    const int64_t rows = std::min(kLowerBand, n - r0), cols = std::min(r0 + kLowerBand, n);
    per += rows * cols;
  }
  return per * count * elem_bytes;
}

int socu_copy_lower_blocks_async(void* dst, const void* src, int64_t count, int64_t n, int64_t elem_bytes,
                                 void* stream) {
  if (dst == nullptr || src == nullptr || count < 0 || n <= 0 || elem_bytes <= 0) return SOCU_ERR_INVALID_ARGUMENT;
  if (count == 0) return SOCU_OK;
  const size_t pitch = (size_t)(n * elem_bytes);
  for (int64_t r0 = 0; r0 < n; r0 += kLowerBand) {
    const int64_t rows = std::min(kLowerBand, n - r0), cols = std::min(r0 + kLowerBand, n);
    // one 3-D copy per band: width = the band's columns, height = its rows,
    // depth = the blocks (slice pitch = one block)
    cudaMemcpy3DParms prm = {};
    const size_t off = (size_t)r0 * pitch;
    prm.srcPtr = make_cudaPitchedPtr(const_cast<char*>(static_cast<const char*>(src)) + off, pitch, pitch, (size_t)n);
    prm.dstPtr = make_cudaPitchedPtr(static_cast<char*>(dst) + off, pitch, pitch, (size_t)n);
    prm.extent = make_cudaExtent((size_t)(cols * elem_bytes), (size_t)rows, (size_t)count);
    prm.kind = cudaMemcpyDefault;
    const cudaError_t e = cudaMemcpy3DAsync(&prm, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return cuda_status(e);
  }
  return SOCU_OK;
}

int socu_block_tridiag_residual(const double* L, const double* E, const double* x, const double* b, double* r,
                                int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, void* stream) {
  Dims d;
  int v = validate(SOCU_OP_SOLVE, SOCU_FLOAT64, L, E, x, batch, horizon, n, n_rhs, &d);
  if (v != SOCU_OK) return v;
  if (batch == 0) return SOCU_OK;
  if (b == nullptr || r == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  if ((long long)smem_residual_elems(d.n) * (long long)sizeof(double) > (long long)max_smem_optin())
    return SOCU_ERR_UNSUPPORTED;
  cudaError_t e = ensure_device(L);
  if (e != cudaSuccess) return cuda_status(e);
  RefineArgs a{};
  a.L = L; a.E = E; a.b = b; a.x = const_cast<double*>(x); a.rout = r;
  a.B = d.B; a.N = d.N; a.n = d.n; a.m = d.m; a.S = d.S;
  const size_t sres = smem_residual_elems(d.n) * sizeof(double);
  if (residual_uses_rows(d.n)) {
    e = launch_residual_rows<false>(a, static_cast<cudaStream_t>(stream), false);
    if (e != cudaSuccess) return cuda_status(e);
  } else {
    e = prepare(k_residual<false>, sres);
    if (e != cudaSuccess) return cuda_status(e);
    const int nrc = ceil_div(d.n, kResRows);
    k_residual<false><<<(unsigned)((long long)d.B * d.N * nrc), 256, sres, static_cast<cudaStream_t>(stream)>>>(a);
  }
  return cuda_status(cudaGetLastError());
}

int socu_refine_launch_create(socu_launch_t* out, const double* L, const double* E, const double* b, double* x,
                              const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs,
                              int max_iter, double tol, void* workspace, size_t workspace_bytes, double* eta,
                              int32_t* iters, int use_cuda_graph, void* stream) {
  if (out == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  Dims d;
  int st = refine_validate(L, E, b, x, batch, horizon, n, n_rhs, max_iter, tol, workspace, workspace_bytes, eta,
                           iters, &d);
  if (st != SOCU_OK) return st;
  socu_launch_s* h = new (std::nothrow) socu_launch_s();
  if (!h) return SOCU_ERR_UNSUPPORTED;
  h->op = SOCU_OP_SOLVE;
  h->dtype = SOCU_FLOAT64;
  h->L = const_cast<double*>(L);
  h->E = const_cast<double*>(E);
  h->x = x;
  h->mask = mask;
  h->batch = batch;
  h->horizon = horizon;
  h->n = n;
  h->n_rhs = n_rhs;
  h->graph = nullptr;
  h->exec = nullptr;
  h->refine = true;
  h->ra = batch > 0 ? refine_args(L, E, b, x, mask, d, max_iter, tol, workspace, eta, iters) : RefineArgs{};
  long long kernels = 0;
  if (batch > 0) refine_enqueue(h->ra, nullptr, &kernels);
  h->kernels = kernels;
  if (use_cuda_graph && batch > 0) {
    st = cuda_status(ensure_device(L));
    if (st == SOCU_OK) st = capture_refine_while(h->ra, &h->graph);
    if (st == SOCU_OK) st = cuda_status(cudaGraphInstantiate(&h->exec, h->graph, 0));
    if (st != SOCU_OK) {
      if (h->exec) cudaGraphExecDestroy(h->exec);
      if (h->graph) cudaGraphDestroy(h->graph);
      delete h;
      return st;
    }
    // kernels per run: prologue with the first round and the loop test, then
    // one round (+ loop control) per further round executed
    long long cp = 0, ci = 0;
    refine_prologue(h->ra, nullptr, &cp);
    refine_iteration(h->ra, nullptr, &ci);
    h->kernels = cp + 1;
    h->round_kernels = ci + 1;
  }
  (void)stream;
  *out = h;
  return SOCU_OK;
}

size_t socu_refine_fallback_workspace_bytes(int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs) {
  if (batch < 0 || horizon <= 0 || n <= 0 || n_rhs <= 0) return 0;
  return fallback_layout(batch, horizon, n, n_rhs).total;
}

int socu_refine_fallback_launch_create(socu_launch_t* out, const double* L, const double* E, const double* b,
                                       double* x, const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n,
                                       int64_t n_rhs, int max_iter, double tol, void* workspace,
                                       size_t workspace_bytes, double* eta, int32_t* iters, uint8_t* used_fp64,
                                       void* stream) {
  if (out == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  Dims d;
  int st = refine_validate(L, E, b, x, batch, horizon, n, n_rhs, max_iter, tol, workspace, workspace_bytes, eta,
                           iters, &d);
  if (st != SOCU_OK) return st;
  if (batch > 0) {
    if (used_fp64 == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
    if (workspace_bytes < fallback_layout(batch, horizon, n, n_rhs).total) return SOCU_ERR_INVALID_ARGUMENT;
    Dims d64;
    const int v = validate(SOCU_OP_FACTOR_AND_SOLVE, SOCU_FLOAT64, L, E, x, batch, horizon, n, n_rhs, &d64);
    if (v != SOCU_OK) return v;
  }
  socu_launch_s* h = new (std::nothrow) socu_launch_s();
  if (!h) return SOCU_ERR_UNSUPPORTED;
  h->op = SOCU_OP_SOLVE;
  h->dtype = SOCU_FLOAT64;
  h->L = const_cast<double*>(L);
  h->E = const_cast<double*>(E);
  h->x = x;
  h->mask = mask;
  h->batch = batch;
  h->horizon = horizon;
  h->n = n;
  h->n_rhs = n_rhs;
  h->graph = nullptr;
  h->exec = nullptr;
  h->refine = true;
  if (batch == 0) {
    *out = h;
    return SOCU_OK;
  }
  h->ra = refine_args(L, E, b, x, mask, d, max_iter, tol, workspace, eta, iters);
  const FallbackLayout lay = fallback_layout(batch, horizon, n, n_rhs);
  char* w = static_cast<char*>(workspace);
  FallbackArgs f;
  f.L64 = reinterpret_cast<double*>(w + lay.l64);
  f.E64 = reinterpret_cast<double*>(w + lay.e64);
  f.fb = reinterpret_cast<uint8_t*>(w + lay.fb);
  f.any = reinterpret_cast<int*>(w + lay.any);
  f.used = used_fp64;
  st = cuda_status(ensure_device(L));
  if (st == SOCU_OK) st = capture_refine_while(h->ra, &h->graph, &f);
  if (st == SOCU_OK) st = cuda_status(cudaGraphInstantiate(&h->exec, h->graph, 0));
  if (st != SOCU_OK) {
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    delete h;
    return st;
  }
  long long cp = 0, ci = 0;
  refine_prologue(h->ra, nullptr, &cp);
  refine_iteration(h->ra, nullptr, &ci);
  h->kernels = cp + 1 + 2;   // prologue, loop test, fallback select + decide
  h->round_kernels = ci + 1;
  (void)stream;
  *out = h;
  return SOCU_OK;
}

int socu_tuning_set(socu_dtype dtype, int64_t n, int64_t n_rhs, const socu_tuning* settings) {
  if ((dtype != SOCU_FLOAT32 && dtype != SOCU_FLOAT64) || n <= 0 || n > 4096 || n_rhs < 0 || n_rhs > (1 << 20))
    return SOCU_ERR_INVALID_ARGUMENT;
  if (settings && !tuning_valid(*settings)) return SOCU_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> g(g_tune_mu);
  for (int i = 0; i < g_n_tune; ++i) {
    TuneSlot& t = g_tune[i];
    if (t.dtype == (int)dtype && t.n == (int)n && t.m == (int)n_rhs) {
      if (settings) {
        t.t = *settings;
      } else {
        g_tune[i] = g_tune[--g_n_tune];
      }
      return SOCU_OK;
    }
  }
  if (!settings) return SOCU_OK;
  if (g_n_tune >= kCacheSlots) return SOCU_ERR_UNSUPPORTED;
  g_tune[g_n_tune++] = TuneSlot{(int)dtype, (int)n, (int)n_rhs, *settings};
  return SOCU_OK;
}

int socu_tuning_get(socu_dtype dtype, int64_t n, int64_t n_rhs, socu_tuning* out) {
  if (out == nullptr || (dtype != SOCU_FLOAT32 && dtype != SOCU_FLOAT64) || n <= 0 || n_rhs < 0)
    return SOCU_ERR_INVALID_ARGUMENT;
  *out = tuning_lookup(dtype, (int)n, (int)n_rhs);
  return SOCU_OK;
}

int socu_tc_error(int* flag, int reset) {
  if (flag == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *flag = 0;
  cudaError_t e = cudaMemcpyFromSymbol(flag, g_tc_error, sizeof(int));
  if (e == cudaSuccess && reset) {
    const int zero = 0;
    e = cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int));
  }
  return cuda_status(e);
}

int socu_tuning_clear(void) {
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_n_tune = 0;
  return SOCU_OK;
}

int socu_launch_profile(socu_launch_t h, void* stream, double* ms, int64_t* launches) {
  if (h == nullptr || ms == nullptr || launches == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < SOCU_KIND_COUNT; ++k) {
    ms[k] = 0.0;
    launches[k] = 0;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  (void)cudaGetLastError();   // a stale error of an earlier, unrelated call is not this run's
  Prof prof;
  g_prof = &prof;
  int s = launch_enqueue(h, st);
  g_prof = nullptr;
  cudaError_t e = prof.err;
  if (s != SOCU_OK && e == cudaSuccess) prof.err_where = 3;
  if (e != cudaSuccess) g_last_cuda_error = (int)e;
  if (s == SOCU_OK && e == cudaSuccess && !prof.stop.empty()) {
    e = cudaEventSynchronize(prof.stop.back());
    if (e != cudaSuccess) prof.err_where = 4;
  }
  if (s == SOCU_OK && e == cudaSuccess && prof.start.size() == prof.stop.size()) {
    for (size_t i = 0; i < prof.start.size(); ++i) {
      float t = 0.f;
      const cudaError_t r = cudaEventElapsedTime(&t, prof.start[i], prof.stop[i]);
      if (r != cudaSuccess) {
        e = r;
        prof.err_where = 4;
        prof.err_kind = prof.kind[i];
        break;
      }
      const int k = prof.kind[i] >= 0 && prof.kind[i] < SOCU_KIND_COUNT ? prof.kind[i] : SOCU_KIND_COUNT - 1;
      ms[k] += t;
      launches[k] += 1;
    }
  }
  for (cudaEvent_t ev : prof.start) cudaEventDestroy(ev);
  for (cudaEvent_t ev : prof.stop) cudaEventDestroy(ev);
  g_prof_err_kind = prof.err_kind;
  g_prof_err_where = prof.err_where;
  if (s != SOCU_OK) return s;
  return cuda_status(e);
}

int socu_profile_error(int* kind, int* where) {
  if (kind == nullptr || where == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *kind = g_prof_err_kind;
  *where = g_prof_err_where;
  return SOCU_OK;
}

int socu_launch_destroy(socu_launch_t h) {
  if (h == nullptr) return SOCU_OK;
  if (h->exec) cudaGraphExecDestroy(h->exec);
  if (h->graph) cudaGraphDestroy(h->graph);
  delete h;
  return SOCU_OK;
}


int socu_refine_solve_noalloc(const double* L, const double* E, const double* b, double* x, const uint8_t* mask,
                              int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, int max_iter, double tol,
                              double* eta, int32_t* iters, void* stream) {
  if (batch < 0 || horizon <= 0 || n <= 0 || n_rhs <= 0) return SOCU_ERR_INVALID_ARGUMENT;
  if (refine_layout(batch, horizon, n, n_rhs).total > kNoAllocScratchBytes) return SOCU_ERR_SCRATCH_TOO_SMALL;
  Dims d;
  const int v = validate(SOCU_OP_SOLVE, SOCU_FLOAT32, L, E, x, batch, horizon, n, n_rhs, &d);
  if (v != SOCU_OK) return v;
  if (max_iter < 1 || max_iter > 1000 || !(tol >= 0.0)) return SOCU_ERR_INVALID_ARGUMENT;
  if (batch == 0) return SOCU_OK;
  if (b == nullptr || eta == nullptr || iters == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  if ((long long)smem_residual_elems(d.n) * (long long)sizeof(double) > (long long)max_smem_optin())
    return SOCU_ERR_UNSUPPORTED;
  cudaError_t e = ensure_device(L);
  if (e != cudaSuccess) return cuda_status(e);
  void* scratch = nullptr;
  const int st = noalloc_scratch(&scratch);
  if (st != SOCU_OK) return st;
  const RefineArgs a = refine_args(L, E, b, x, mask, d, max_iter, tol, scratch, eta, iters);
  // the same enqueue path as socu_refine_solve (level schedule on the stack,
  // kernel attributes from static caches): only the scratch differs
  return refine_enqueue(a, static_cast<cudaStream_t>(stream), nullptr);
}

// ---------------------------------------------------------------------------
// ragged batches
// ---------------------------------------------------------------------------
int socu_ragged_layout(const int64_t* horizon, const int64_t* n, const int64_t* n_rhs, int64_t count,
                       int64_t* off_L, int64_t* off_E, int64_t* off_x, int64_t* totals) {
  std::vector<RgInst> inst;
  long long tot[3];
  const int st = rg_layout(horizon, n, n_rhs, count, &inst, tot);
  if (st != SOCU_OK) return st;
  for (int64_t i = 0; i < count; ++i) {
    if (off_L) off_L[i] = inst[i].oL;
    if (off_E) off_E[i] = inst[i].oE;
    if (off_x) off_x[i] = inst[i].oX;
  }
  if (totals) {
    totals[0] = tot[0];
    totals[1] = tot[1];
    totals[2] = tot[2];
  }
  return SOCU_OK;
}

int socu_ragged_create(socu_ragged_t* out, socu_dtype dtype, int refine, const int64_t* horizon, const int64_t* n,
                       const int64_t* n_rhs, int64_t count, int max_iter) {
  if (out == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (dtype != SOCU_FLOAT32 && dtype != SOCU_FLOAT64) return SOCU_ERR_INVALID_ARGUMENT;
  if (refine && (dtype != SOCU_FLOAT64 || max_iter < 1 || max_iter > 1000)) return SOCU_ERR_INVALID_ARGUMENT;
  socu_ragged_s* r = new (std::nothrow) socu_ragged_s();
  if (!r) return SOCU_ERR_UNSUPPORTED;
  r->dtype = dtype;
  r->refine = refine != 0;
  r->max_iter = refine ? max_iter : 0;
  const int st = rg_create(r, horizon, n, n_rhs, count);
  if (st != SOCU_OK) {
    rg_free(r);
    delete r;
    return st;
  }
  *out = r;
  return SOCU_OK;
}

int socu_ragged_factor_and_solve(socu_ragged_t r, void* L, void* E, void* x, void* stream) {
  if (r == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  return rg_factor_and_solve(r, L, E, x, static_cast<cudaStream_t>(stream));
}

int socu_ragged_refine_solve(socu_ragged_t r, const double* L, const double* E, const double* b, double* x,
                             double tol, double* eta, int32_t* iters, void* stream) {
  if (r == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  return rg_refine_solve(r, L, E, b, x, tol, eta, iters, static_cast<cudaStream_t>(stream));
}

int socu_ragged_launch_create(socu_launch_t* out, socu_ragged_t r, void* L, void* E, const double* b, void* x,
                              double tol, double* eta, int32_t* iters, int use_cuda_graph, void* stream) {
  if (out == nullptr || r == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (r->count > 0) {
    if (L == nullptr || x == nullptr || (r->tot[1] > 0 && E == nullptr)) return SOCU_ERR_INVALID_ARGUMENT;
    if (r->refine && (b == nullptr || eta == nullptr || iters == nullptr || !(tol >= 0.0)))
      return SOCU_ERR_INVALID_ARGUMENT;
  }
  socu_launch_s* h = new (std::nothrow) socu_launch_s();
  if (!h) return SOCU_ERR_UNSUPPORTED;
  h->op = SOCU_OP_FACTOR_AND_SOLVE;
  h->dtype = r->refine ? SOCU_FLOAT64 : (socu_dtype)r->dtype;
  h->L = L;
  h->E = E;
  h->x = x;
  h->mask = nullptr;
  h->batch = r->count;
  h->graph = nullptr;
  h->exec = nullptr;
  h->rg = r;
  h->b = b;
  h->tol = tol;
  h->eta = eta;
  h->iters = iters;
  h->kernels = r->count > 0 ? 2 : 0;
  if (use_cuda_graph && r->count > 0) {
    const int st = capture(h);
    if (st != SOCU_OK) {
      delete h;
      return st;
    }
  }
  (void)stream;
  *out = h;
  return SOCU_OK;
}

int socu_ragged_error(socu_ragged_t r, int* flag) {
  if (r == nullptr || flag == nullptr) return SOCU_ERR_INVALID_ARGUMENT;
  *flag = 0;
  if (r->count == 0) return SOCU_OK;
  int s = rg_device(r);
  if (s != SOCU_OK) return s;
  return cuda_status(cudaMemcpy(flag, r->d_err, sizeof(int), cudaMemcpyDeviceToHost));
}

int64_t socu_ragged_grid(socu_ragged_t r) { return r ? r->grid : 0; }

int socu_ragged_set_wait_limit(socu_ragged_t r, int64_t timeout_ns) {
  if (r == nullptr || timeout_ns < 1000 || timeout_ns > 60000000000LL) return SOCU_ERR_INVALID_ARGUMENT;
  r->timeout_ns = timeout_ns;
  return SOCU_OK;
}

int socu_ragged_withhold_instance(socu_ragged_t r, int64_t instance) {
  if (r == nullptr || instance < 0 || instance >= r->count) return SOCU_ERR_INVALID_ARGUMENT;
  std::vector<unsigned long long> kept;
  kept.reserve(r->init.size());
  for (unsigned long long t : r->init) {
    int ii, ph, chunk;
    rg_decode(t, ii, ph, chunk);
    if (ii != (int)instance) kept.push_back(t);
  }
  if (kept.size() == r->init.size()) return SOCU_OK;
  int s = rg_device(r);
  if (s != SOCU_OK) return s;
  r->init.swap(kept);
  r->n_init = (unsigned)r->init.size();
  if (r->n_init == 0) return SOCU_OK;
  return cuda_status(cudaMemcpy(r->d_init, r->init.data(), sizeof(unsigned long long) * r->n_init,
                                cudaMemcpyHostToDevice));
}

int socu_ragged_destroy(socu_ragged_t r) {
  if (r == nullptr) return SOCU_OK;
  if (r->count > 0) rg_device(r);
  rg_free(r);
  delete r;
  return SOCU_OK;
}

}  // extern "C"
