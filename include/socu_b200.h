/*
 * socu_b200 — C ABI of the B200 (sm_100a) nested-dissection block-tridiagonal
 * SPD Cholesky.
 *
 * Plain pointers and sizes only.  Every array pointer is a CUDA device pointer
 * to a contiguous row-major buffer; `stream` is a cudaStream_t (NULL = legacy
 * default stream).  All entry points return an int status (SOCU_OK == 0,
 * negative on error) and never allocate on the hot path.
 *
 * Layouts (identical to socu; socu/block_tridiag_solver.py:739-774):
 *   L     (batch, horizon, n, n)        diagonal blocks; lower triangle read
 *   E     (batch, storage_len, n, n)    off-diagonal blocks, storage_len =
 *                                       socu_off_diag_storage_len(horizon);
 *                                       E[k] = Psi_{k+1,k} for k < horizon-1,
 *                                       slots >= horizon-1 MUST be zero
 *   x     (batch, horizon, n, n_rhs)    right-hand side in, result out
 *   mask  (batch,) uint8 or NULL        0 = leave that batch entry untouched
 * The factor is written in place into L and E with the reference's exact
 * block layout, so factors are interchangeable with socu's.
 */
#ifndef SOCU_B200_H
#define SOCU_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SOCU_OK 0
#define SOCU_ERR_INVALID_ARGUMENT (-1)
#define SOCU_ERR_CUDA (-2)
#define SOCU_ERR_UNSUPPORTED (-3)
#define SOCU_ERR_TIMEOUT (-4)
#define SOCU_ERR_SCRATCH_TOO_SMALL (-5)

typedef enum socu_dtype { SOCU_FLOAT32 = 0, SOCU_FLOAT64 = 1 } socu_dtype;

/* Operations 0-4 are the reference's five launches.  5-8 are an extension
 * (no counterpart in the reference) for factor reuse: SOCU_OP_FACTOR_INV
 * factors like SOCU_OP_FACTOR and also keeps W_i^T = C_i^{-T} in the strict
 * upper triangle of each L_i (as SOCU_OP_FACTOR_AND_SOLVE does); the *_INV
 * sweeps require such a factor and apply W_i as a matrix-vector product
 * instead of a triangular solve.  Blocks with n <= 64 only (larger n:
 * SOCU_ERR_UNSUPPORTED). */
typedef enum socu_op {
  SOCU_OP_FACTOR = 0,
  SOCU_OP_FACTOR_AND_SOLVE = 1,
  SOCU_OP_FORWARD_SUBSTITUTION = 2,
  SOCU_OP_BACKWARD_SUBSTITUTION = 3,
  SOCU_OP_SOLVE = 4,
  SOCU_OP_FACTOR_INV = 5,
  SOCU_OP_FORWARD_INV = 6,
  SOCU_OP_BACKWARD_INV = 7,
  SOCU_OP_SOLVE_INV = 8
} socu_op;

/* Library version string. */
const char* socu_version(void);

/* Human-readable text for a status code. */
const char* socu_status_string(int status);

/* The last CUDA error seen by this library in the calling thread (0 if none). */
int socu_last_cuda_error(void);

/* Diagnostics: the line of the library source that reported that error. */
int socu_last_cuda_error_line(void);

/* floor(log2(horizon)) + 1, or -1 for horizon <= 0.
 * Replaces calculate_recursive_iterations, socu/block_tridiag_solver.py:12-15. */
int64_t socu_recursive_iterations(int64_t horizon);

/* Number of n x n blocks E must hold, or -1 for horizon <= 0.
 * Replaces calculate_off_diag_storage_len, socu/block_tridiag_solver.py:18-23. */
int64_t socu_off_diag_storage_len(int64_t horizon);

/* Largest block size n supported for a dtype (shared-memory bound). */
int64_t socu_max_block_size(socu_dtype dtype, int64_t n_rhs);

/* One-shot operations, enqueued on `stream`.
 * Replace the callbacks returned by create_cholesky_factor_launch
 * (socu/block_tridiag_solver.py:739-923), create_cholesky_factor_and_solve_launch
 * (:926-1233), create_cholesky_forward_substitution_launch (:1236-1374),
 * create_cholesky_backward_substitution_launch (:1377-1517) and
 * create_cholesky_solve_launch (:1520-1727). */
int socu_cholesky_factor(socu_dtype dtype, void* L, void* E, const uint8_t* mask,
                         int64_t batch, int64_t horizon, int64_t n, void* stream);

int socu_cholesky_factor_and_solve(socu_dtype dtype, void* L, void* E, void* x,
                                   const uint8_t* mask, int64_t batch, int64_t horizon,
                                   int64_t n, int64_t n_rhs, void* stream);

int socu_cholesky_forward_substitution(socu_dtype dtype, const void* L, const void* E, void* x,
                                       const uint8_t* mask, int64_t batch, int64_t horizon,
                                       int64_t n, int64_t n_rhs, void* stream);

int socu_cholesky_backward_substitution(socu_dtype dtype, const void* L, const void* E, void* x,
                                        const uint8_t* mask, int64_t batch, int64_t horizon,
                                        int64_t n, int64_t n_rhs, void* stream);

int socu_cholesky_solve(socu_dtype dtype, const void* L, const void* E, void* x,
                        const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n,
                        int64_t n_rhs, void* stream);

/* Any socu_op (0-8) as a direct call; x is ignored for the two factor ops. */
int socu_cholesky_run(socu_op op, socu_dtype dtype, void* L, void* E, void* x, const uint8_t* mask, int64_t batch,
                      int64_t horizon, int64_t n, int64_t n_rhs, void* stream);

/* As socu_cholesky_run for the two factor ops (and SOCU_OP_FACTOR_INV), with a
 * per-instance numerical status: info (batch,) device int32, set to 0 for
 * every batch entry, then to 1 + i for entries whose factorisation failed,
 * i the first failing node in elimination order (lowest separator level,
 * then lowest block index): a pivot <= 0 (the Schur-complemented block is not
 * positive definite) or a non-finite value.  Blocks of a failed entry hold
 * non-finite values afterwards.  No counterpart in the reference, whose
 * potrf takes the square root of any pivot (socu/blas/potrf.py:97-117). */
int socu_cholesky_run_info(socu_op op, socu_dtype dtype, void* L, void* E, void* x, const uint8_t* mask,
                           int32_t* info, int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, void* stream);

/* Recorded launches bound to fixed buffers, optionally captured once into a
 * CUDA graph at creation (the recorded launches + create_cuda_graph_callback
 * of socu/block_tridiag_solver.py:784-790 and socu/utils.py:39-65).  The mask
 * pointer is bound, its contents may change between runs (also under a
 * graph).  `x` is ignored for SOCU_OP_FACTOR.  A launch object must not be
 * run from two host threads at once. */
typedef struct socu_launch_s* socu_launch_t;

int socu_launch_create(socu_launch_t* out, socu_op op, socu_dtype dtype, void* L, void* E,
                       void* x, const uint8_t* mask, int64_t batch, int64_t horizon,
                       int64_t n, int64_t n_rhs, int use_cuda_graph, void* stream);

int socu_launch_run(socu_launch_t launch, void* stream);

/* ---- launch settings and autotuning (no counterpart in the reference, whose
 * launches take block_dim / block_size per call,
 * socu/block_tridiag_solver.py:739-747, 776-781) ----
 * Every field 0 = not set (built-in heuristic).  node/update/sweep_threads:
 * threads per CTA of the node, Schur-update and sweep kernels (64, 128 or
 * 256).  sweep_tensor_cores: float sweeps on inverse-carrying factors use FP64
 * tensor-core (1) or SIMT (2) products.  update_tile: output tile of the
 * blocked Schur update for n > 64 (16 or 32; the reference's block_size).
 * ragged_units: level nodes per task chunk of a ragged batch (1..64).
 * update_tensor_cores: Schur updates of float factors (n <= 128) on the
 * tcgen05 tensor cores with 3xTF32 operands (1) or on the FP64 tensor pipe
 * (2, the default: exact products of the float operands, FP64 sums).
 * node_tensor_cores: the coupling and forward products of float level nodes
 * (n <= 128) on the tcgen05 tensor cores at every level (1), only on levels
 * with at least 4 nodes per SM (3), or SIMT (2, and the default); 4 keeps a
 * float level node with 64 < n <= 128 resident in tensor memory and runs the
 * trailing updates of its blocked Cholesky and coupling solves on the tensor
 * cores (3xTF32), the 32-column panels on SIMT cores. */
typedef struct socu_tuning {
  int32_t node_threads;
  int32_t update_threads;
  int32_t sweep_threads;
  int32_t sweep_tensor_cores;
  int32_t update_tile;
  int32_t ragged_units;
  int32_t update_tensor_cores;
  int32_t node_tensor_cores;
} socu_tuning;

/* As socu_launch_create, with per-launch settings (NULL: none) applied on top
 * of the tuned table.  The reference's block_dim maps to the three thread
 * counts, its block_size to update_tile. */
int socu_launch_create_tuned(socu_launch_t* out, socu_op op, socu_dtype dtype, void* L, void* E, void* x,
                             const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs,
                             int use_cuda_graph, const socu_tuning* settings, void* stream);

/* As socu_launch_create_tuned, with the per-instance factor status of
 * socu_cholesky_run_info (info may be NULL; non-NULL only for the factor ops),
 * rewritten by every run. */
int socu_launch_create_ex(socu_launch_t* out, socu_op op, socu_dtype dtype, void* L, void* E, void* x,
                          const uint8_t* mask, int32_t* info, int64_t batch, int64_t horizon, int64_t n,
                          int64_t n_rhs, int use_cuda_graph, const socu_tuning* settings, void* stream);

/* Install (settings != NULL) or remove the tuned entry for (dtype, n, n_rhs);
 * n_rhs = 0 is the entry for any n_rhs without one of its own.  Launches
 * created afterwards (and direct socu_cholesky_* calls, refined and ragged
 * solves, whose float factor uses the SOCU_FLOAT32 entries) read the table. */
int socu_tuning_set(socu_dtype dtype, int64_t n, int64_t n_rhs, const socu_tuning* settings);

/* The table's effective entry for (dtype, n, n_rhs) (zeros where unset). */
int socu_tuning_get(socu_dtype dtype, int64_t n, int64_t n_rhs, socu_tuning* out);

/* Remove every tuned entry. */
int socu_tuning_clear(void);

/* Kernel kinds of socu_launch_profile. */
typedef enum socu_kernel_kind {
  SOCU_KIND_NODE = 0,          /* level node: potrf + coupling solves (+ forward step) */
  SOCU_KIND_UPDATE = 1,        /* Schur updates and fill-in */
  SOCU_KIND_PULL = 2,          /* forward coupling updates fused into factor_and_solve */
  SOCU_KIND_FORWARD = 3,       /* forward sweep */
  SOCU_KIND_BACKWARD = 4,      /* backward sweep */
  SOCU_KIND_REFINE_SETUP = 5,  /* refinement: state reset, float copies, norms */
  SOCU_KIND_REFINE_UPDATE = 6, /* refinement: x += delta */
  SOCU_KIND_RESIDUAL = 7,      /* refinement: FP64 residual and norms */
  SOCU_KIND_REFINE_CHECK = 8,  /* refinement: convergence test (not a separate kernel any more: the
                                  residual kernel's last CTA per instance runs it) */
  SOCU_KIND_RAGGED = 9,        /* ragged batch: queue reset + persistent solver */
  SOCU_KIND_COUNT = 10
} socu_kernel_kind;

/* One eager (never graph) run of `launch` on `stream` with a CUDA event pair
 * around every kernel; synchronises, then ms[k] = summed device time and
 * launches[k] = kernel count of kind k (arrays of SOCU_KIND_COUNT).  A
 * refined solve runs all its max_iter rounds.  For measurement only: the
 * events add gaps between kernels. */
int socu_launch_profile(socu_launch_t launch, void* stream, double* ms, int64_t* launches);

/* After a failed socu_launch_profile in this thread: the kernel kind the
 * error was charged to (-1 if none) and where it arose: 0 pending before that
 * launch, 1 raised by the launch, 2 creating or recording a timing event, 3 a
 * non-launch call of the op, 4 synchronising on or reading the events. */
int socu_profile_error(int* kind, int* where);

/* Number of kernels one run enqueues (0 for a NULL launch).  For a
 * graph-captured refined solve: the kernels before the refinement loop. */
int64_t socu_launch_kernel_count(socu_launch_t launch);

/* Graph-captured refined solve: kernels per refinement round (the rounds run
 * in a conditional WHILE node until every instance converged); 0 otherwise. */
int64_t socu_launch_round_kernel_count(socu_launch_t launch);

int socu_launch_destroy(socu_launch_t launch);

/* ---- mixed precision with FP64 iterative refinement (no counterpart in the
 * reference, which only has plain f32/f64 paths) ----
 * Solves Psi x = b for FP64 inputs: a float copy of (L, E) is factored with the
 * same nested-dissection kernels, then x is refined in FP64 against the
 * original blocks until the normwise backward error
 *     eta = ||b - Psi x||_inf / (||Psi||_inf ||x||_inf + ||b||_inf) <= tol
 * or max_iter corrections were applied.  L, E and b are not modified.
 * eta (batch,) and iters (batch,) are device outputs; iters < 0 flags a
 * non-finite residual (float factor broke down) after -iters steps.
 * The workspace (>= socu_refine_workspace_bytes, 256-byte aligned device
 * memory) is owned by the caller; nothing is allocated here. */
size_t socu_refine_workspace_bytes(int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs);

int socu_refine_solve(const double* L, const double* E, const double* b, double* x, const uint8_t* mask,
                      int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, int max_iter, double tol,
                      void* workspace, size_t workspace_bytes, double* eta, int32_t* iters, void* stream);

/* Launch object for socu_refine_solve (buffers bound).  With use_cuda_graph
 * the refinement rounds are captured in a conditional WHILE graph node that
 * stops as soon as every instance is done; without it, and in
 * socu_refine_solve, max_iter rounds are enqueued and finished instances skip
 * their work. */
int socu_refine_launch_create(socu_launch_t* out, const double* L, const double* E, const double* b, double* x,
                              const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs,
                              int max_iter, double tol, void* workspace, size_t workspace_bytes, double* eta,
                              int32_t* iters, int use_cuda_graph, void* stream);

/* Graph-captured refined solve with an FP64 fallback (no counterpart in the
 * reference).  After the refinement loop, every active instance whose eta did
 * not reach tol -- refinement stalled, ran out of max_iter rounds, or the
 * float factor broke down -- is solved again by the plain FP64
 * factor_and_solve on working copies of its original blocks, and its eta is
 * recomputed; this stage sits in a conditional IF graph node that runs only
 * when some instance needs it.  used_fp64 (batch,) device output: 1 where x
 * comes from the FP64 path.  iters keeps the refinement count (negative on
 * breakdown).  The workspace (>= socu_refine_fallback_workspace_bytes,
 * 256-byte aligned) adds FP64 copies of L and E to the refinement workspace. */
size_t socu_refine_fallback_workspace_bytes(int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs);

int socu_refine_fallback_launch_create(socu_launch_t* out, const double* L, const double* E, const double* b,
                                       double* x, const uint8_t* mask, int64_t batch, int64_t horizon, int64_t n,
                                       int64_t n_rhs, int max_iter, double tol, void* workspace,
                                       size_t workspace_bytes, double* eta, int32_t* iters, uint8_t* used_fp64,
                                       void* stream);

/* Same solve as socu_refine_solve, for callers that cannot allocate device
 * memory while they solve: an XLA/JAX custom call (buffers come from XLA's
 * allocator, the handler must not cudaMalloc), a real-time control loop that
 * bans allocation after start-up (cudaMalloc/cudaFree can block and
 * synchronise the device), or code running inside CUDA stream capture, where
 * cudaMalloc is not allowed.  No counterpart in the reference.
 * Nothing is allocated: the float factor, the correction vector and the
 * per-instance refinement state live in one fixed array of
 * SOCU_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads
 * the library holds until the process exits.  Problems whose scratch
 * (socu_refine_workspace_bytes) exceeds it are rejected with
 * SOCU_ERR_SCRATCH_TOO_SMALL.  The first call on each device looks the
 * array's device address up (make that first call before any stream
 * capture).  All calls share the one array: every call re-initialises what it
 * reads, but calls whose work overlaps on the GPU (different streams, or
 * different host threads on the same device) race and corrupt each other.
 * The host cannot see convergence without a synchronisation, so every call
 * enqueues all max_iter refinement rounds; instances that have converged skip
 * the work of the remaining rounds (their kernels return at once), which
 * still costs the launches: pass the smallest max_iter that meets tol. */
#define SOCU_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)

int socu_refine_solve_noalloc(const double* L, const double* E, const double* b, double* x, const uint8_t* mask,
                              int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, int max_iter, double tol,
                              double* eta, int32_t* iters, void* stream);

/* Gradient of x = Psi^{-1} b with respect to the blocks of Psi (no counterpart
 * in the reference, which defines no derivative).  Given x and g = Psi^{-1} gx
 * (gx = dloss/dx, g obtained with socu_cholesky_solve on the stored factor):
 *   dD (batch, horizon, n, n): gradient w.r.t. the lower triangle of each D_i
 *       (the solver reads only lower(D_i)); zeros above the diagonal
 *   dE (batch, e_blocks, n, n): gradient w.r.t. E_i = Psi_{i+1,i} for
 *       i < horizon-1, zeros for the remaining storage slots
 * dloss/db equals g.  One fused kernel. */
int socu_block_tridiag_grad(socu_dtype dtype, const void* x, const void* g, void* dD, void* dE, int64_t batch,
                            int64_t horizon, int64_t n, int64_t n_rhs, int64_t e_blocks, void* stream);

/* ---- ragged batches (no counterpart in the reference, whose launches take
 * one (N, n, m) shape for the whole batch) ----
 * `count` independent systems, instance i with horizon[i] blocks of size n[i]
 * (1..64) and n_rhs[i] right-hand sides, packed back to back: instance i's
 * L is (horizon[i], n[i], n[i]) at element off_L[i] of one array, its E is
 * (calculate_off_diag_storage_len(horizon[i]), n[i], n[i]) at off_E[i], its
 * x/b is (horizon[i], n[i], n_rhs[i]) at off_x[i].  Each instance uses the
 * layouts and results of socu_cholesky_factor_and_solve.
 *
 * socu_ragged_layout: the offsets (arrays of `count`, any may be NULL) and
 * totals[3] = elements of the packed L, E, x arrays.  Host only. */
int socu_ragged_layout(const int64_t* horizon, const int64_t* n, const int64_t* n_rhs, int64_t count,
                       int64_t* off_L, int64_t* off_E, int64_t* off_x, int64_t* totals);

/* A ragged batch bound to the current device.  All the batch's systems are
 * solved by one persistent kernel that takes (instance, phase, chunk) tasks
 * from a device work queue; the queue, the instance descriptors and (refine)
 * the float workspace are allocated here, once.
 *   refine = 0: plain factor_and_solve in `dtype`.
 *   refine = 1: dtype must be SOCU_FLOAT64; float factor + FP64 refinement as
 *               socu_refine_solve, every instance iterating on its own until
 *               its eta <= tol or max_iter rounds.
 * A batch object runs one solve at a time (the queue is shared). */
typedef struct socu_ragged_s* socu_ragged_t;

int socu_ragged_create(socu_ragged_t* out, socu_dtype dtype, int refine, const int64_t* horizon, const int64_t* n,
                       const int64_t* n_rhs, int64_t count, int max_iter);

/* Plain path: factor L, E in place and overwrite x (b on input) with the solution. */
int socu_ragged_factor_and_solve(socu_ragged_t batch, void* L, void* E, void* x, void* stream);

/* Refine path: L, E, b untouched; eta (count,) and iters (count,) as in socu_refine_solve. */
int socu_ragged_refine_solve(socu_ragged_t batch, const double* L, const double* E, const double* b, double* x,
                             double tol, double* eta, int32_t* iters, void* stream);

/* Launch object for either path (b, tol, eta, iters only for refine), optionally
 * captured into a CUDA graph; run and destroy with socu_launch_run /
 * socu_launch_destroy.  The batch must outlive the launch. */
int socu_ragged_launch_create(socu_launch_t* out, socu_ragged_t batch, void* L, void* E, const double* b, void* x,
                              double tol, double* eta, int32_t* iters, int use_cuda_graph, void* stream);

/* Device error word of the last finished solve (synchronises): 0 ok,
 * 1 a queue wait exceeded its time bound, 2 queue overflow. */
int socu_ragged_error(socu_ragged_t batch, int* flag);

/* CTAs of the persistent launch (occupancy x SM count). */
int64_t socu_ragged_grid(socu_ragged_t batch);

/* Bound of one device-side queue wait, in nanoseconds of %globaltimer without
 * any queue progress (default 4e9, i.e. 4 s; range 1e3 .. 6e10).  A CTA whose
 * wait runs out sets error word 1 (socu_ragged_error) and returns, so a
 * stalled queue ends the launch instead of hanging it.  No counterpart in the
 * reference (its launches do not wait on each other). */
int socu_ragged_set_wait_limit(socu_ragged_t batch, int64_t timeout_ns);

/* Failure injection for tests of the bound above, host side only: leave the
 * first-phase tasks of `instance` out of the queue's initial contents, so that
 * this instance never starts and the queue stalls once the others are done.
 * The next solve then ends with error word 1.  No counterpart in the reference. */
int socu_ragged_withhold_instance(socu_ragged_t batch, int64_t instance);

int socu_ragged_destroy(socu_ragged_t batch);

/* Throughput probe of the FP64 tensor-core pipe (mma.sync m8n8k4 .f64 on
 * register operands, no memory traffic): `blocks` CTAs of `threads` threads,
 * `iters` steps of 8 independent chains per warp.  *flops receives the
 * launch's floating-point operations; time the launch with CUDA events on
 * `stream` to get the device's FP64 tensor peak (the roofline denominator of
 * the FP64 factor).  `sink` is a device double the kernel may write.  No
 * counterpart in the reference. */
int socu_dmma_peak_launch(int64_t blocks, int threads, int iters, double* sink, void* stream, double* flops);

/* Error word of the asynchronous units on the current device (synchronises):
 * 0 ok, 1 a tensor-core (tcgen05) wait ran out, 2 a TMA copy wait of the
 * resident sweeps ran out (that kernel skipped its result).  reset != 0 clears
 * it afterwards.  No counterpart in the reference. */
int socu_tc_error(int* flag, int reset);

/* Self-test of the tensor-core (tcgen05) building block of the float path:
 * one CTA computes D = A (m_rows x k_depth) * B (n_cols x k_depth)^T
 * (row-major float arrays; m_rows 64 or 128) with operands split into TF32
 * pieces (3xTF32), FP32 accumulation in tensor memory, and writes the
 * accumulator as it lies in tensor memory: D is (128 x n_cols), row t = TMEM
 * lane t.  n_cols in 16..128 (multiple of 16), k_depth a multiple of 8.
 * *error_flag (device int) is set to 1 if a tensor-core wait ran out.  No
 * counterpart in the reference. */
int socu_tc_selftest(const float* A, const float* B, float* D, int64_t m_rows, int64_t n_cols, int64_t k_depth,
                     int* error_flag, void* stream);

/* r = b - Psi x in FP64 against the original blocks (no counterpart in the
 * reference).  L and E as for the factor input (lower(L_i), level-0 slots). */
int socu_block_tridiag_residual(const double* L, const double* E, const double* x, const double* b, double* r,
                                int64_t batch, int64_t horizon, int64_t n, int64_t n_rhs, void* stream);

/* Copy the lower triangles of `count` consecutive row-major n x n blocks of
 * elem_bytes-byte elements (the only part of L that every factor and the
 * residual read) from src to dst, host or device memory on either side, in
 * 16-row bands (band k: rows 16k.., columns 0 .. 16k+15) on `stream`: a
 * caller streaming L from pinned host memory moves ~(n + 16) / 2n of the
 * bytes.  Elements above the band diagonal of dst are left as they are.  No
 * counterpart in the reference. */
int socu_copy_lower_blocks_async(void* dst, const void* src, int64_t count, int64_t n, int64_t elem_bytes,
                                 void* stream);
/* Bytes socu_copy_lower_blocks_async moves for those arguments. */
int64_t socu_lower_blocks_bytes(int64_t count, int64_t n, int64_t elem_bytes);

#ifdef __cplusplus
}
#endif

#endif /* SOCU_B200_H */
