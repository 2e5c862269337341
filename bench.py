"""Benchmark: batched solves/s of the mixed-precision + FP64-refinement solver
versus the plain FP64 path, at normwise relative backward error <= 1e-12.

Workload: N=1024 blocks, n=64, m=8 right-hand sides, diagonal shift s=10,
one system per GPU (README construction, seeded torch CPU generator, so both
arms solve bit-identical inputs).  A step is one full solve of that system
from its original blocks: float factor + refinement for the headline value,
FP64 factor_and_solve for the comparison line.  Further sections (same run,
same JSON line): the large stress shape N=16384, n=128, m=32; a ragged batch
of 4096 uneven systems; the differentiable solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank solves its own replica of the single system (the
path does not shard) and its own contiguous share of the ragged batch
(instances balanced by factor work); value = systems solved by all ranks /
max-over-ranks time.  The reference arm times the CPU oracle (NumPy
restatement of the reference algorithm) on the host cores, rank 0 only.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BLOCKS, BLOCK, NRHS, SHIFT, SEED = 1024, 64, 8, 10.0, 0
TOL, MAX_ITER = 1e-12, 10
METRIC = "batched solves/s: mixed+refine vs plain FP64 on 1 B200 at rel. backward err <=1e-12"
WORKLOAD = "N=1024 n=64 m=8 shift=10 single system per GPU (README generator, seed 0)"


def storage_len(N):
    return sum(N // (2 ** l) - 1 for l in range(N.bit_length()))


RAGGED_COUNT, RAGGED_SEED = 4096, 0
# DRAM bytes (read + write) per k_bwd<float, resident, inverse> launch, averaged
# over one backward sweep of this workload, from the ncu capture summarised in
# profiles/k_bwd_f32_inverse_sweep_N1024_n64_m8.md
TRAFFIC_BYTES = 5057908
TRAFFIC_NOTE = "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/k_bwd_f32_inverse_sweep_N1024_n64_m8.md"
# DRAM bytes (read + write) per k_node<float, y, inverse> launch of a float
# factor_and_solve of this shape, averaged over its 11 levels: ncu capture of
# `bench.py --ncu-case node` (4 systems, so that the float blocks exceed L2),
# 254.1 MB over the 11 launches of one pass, per system
# (profiles/k_node_f32_levels_N1024_n64_m8_B4.md)
NODE_TRAFFIC_BYTES = 254.13e6 / 4 / 11
NODE_TRAFFIC_NOTE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of the 11 k_node<float,1,1,wt> launches of "
                     "bench.py --ncu-case node (4 systems, inputs > L2), per system and launch; "
                     "profiles/k_node_f32_levels_N1024_n64_m8_B4.md")
RAGGED_WORKLOAD = ("4096 independent systems, N ~ U{8..256}, n in {8,16,32,48}, m in {1,4}, shift=10, "
                   "instance i seeded with 0 + i, one persistent launch per solve")


def make_problem_host():
    """The workload system as float64 CPU tensors (B=1): README construction
    from a seeded torch CPU generator.  Both arms start from these values."""
    from socu_b200.problems import readme_blocks
    return readme_blocks(N_BLOCKS, BLOCK, NRHS, shift=SHIFT, seed=SEED, batch=1, device="cpu")


def band_solve_fp64(L, E, b):
    """FP64 solve of one system by LAPACK's banded Cholesky (scipy
    solveh_banded, half-bandwidth 2n-1): the dense FP64 solution the forward
    errors are measured against (a dense matrix of N n unknowns does not fit)."""
    import scipy.linalg as la
    N, n = L.shape[0], L.shape[1]
    m = b.shape[-1]
    bw = 2 * n - 1
    ab = np.zeros((bw + 1, N * n))
    r, c = np.tril_indices(n)
    for i in range(N):
        # lower(D_i): ab[k, j] = A[j + k, j]
        ab[r - c, i * n + c] = L[i][r, c]
        if i < N - 1:
            rr, cc = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
            ab[(n + rr - cc).ravel(), (i * n + cc).ravel()] = E[i][rr, cc].ravel()
    return la.solveh_banded(ab, b.reshape(N * n, m), lower=True).reshape(N, n, m)


def forward_error(x, x_ref):
    """max |x - x_ref| / max |x_ref| (normwise, infinity norm)."""
    return float(np.abs(x - x_ref).max() / max(np.abs(x_ref).max(), 1e-300))


def algorithmic_factor_flops(N, n):
    """Nested-dissection factor flop count: per level, potrf n^3/3 per node,
    trsm n^3 per coupling side, syrk n^3 per coupling side, fill-in gemm 2 n^3."""
    s, total = 1, 0.0
    for _ in range(N.bit_length()):
        d = (N + s) // (2 * s)
        nodes = [s - 1 + 2 * s * t for t in range(d)]
        r = sum(1 for i in nodes if i + s < N)
        lft = sum(1 for i in nodes if i >= s)
        both = sum(1 for i in nodes if i + s < N and i >= s)
        total += d * n ** 3 / 3 + 2 * (r + lft) * n ** 3 + both * 2 * n ** 3
        s *= 2
    return total


def max_over_ranks(seconds, world, device):
    """Step time of the whole job: the slowest rank's figure (every rank calls
    this at the same points, in the same order)."""
    import torch
    import torch.distributed as dist
    v = torch.tensor([seconds], dtype=torch.float64, device=device)
    if world > 1:
        dist.all_reduce(v, op=dist.ReduceOp.MAX)
    return float(v)


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        # raw samples (the summary goes into the JSON line); SOCU_BENCH_CLOCKS_DIR keeps them elsewhere
        out_dir = os.environ.get("SOCU_BENCH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out_dir, f"bench_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for name, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle port (NumPy restatement of the reference algorithm)
# ---------------------------------------------------------------------------
CPU_SAMPLE_S = 10.0


def cpu_oracle_solves_per_s(L, E, b, budget_s=CPU_SAMPLE_S, max_reps=40):
    """Median time of full FP64 factor_and_solve runs of the oracle, repeated
    for about budget_s seconds of CPU work (at least 3 runs)."""
    from oracle import nd_cholesky as nd
    ts = []
    t_start = time.perf_counter()
    while len(ts) < 3 or (time.perf_counter() - t_start < budget_s and len(ts) < max_reps):
        t0 = time.perf_counter()
        nd.nd_factor_and_solve(L, E, b)
        ts.append(time.perf_counter() - t0)
    return 1.0 / statistics.median(ts), ts


def workload_config():
    return {"workload": WORKLOAD, "N": N_BLOCKS, "n": BLOCK, "m": NRHS, "shift": SHIFT, "tol": TOL,
            "max_iter": MAX_ITER, "l2": "256 MB flush before every timed step (GPU arm); host CPU run (reference)",
            "inputs": "README construction, torch CPU generator seed 0, identical in both arms"}


def run_reference(args, rank):
    if rank != 0:
        return
    L0, E0, b0 = make_problem_host()
    L, E, b = L0[0].numpy(), E0[0].numpy(), b0[0].numpy()
    cores = len(os.sched_getaffinity(0))
    from oracle import nd_cholesky as nd
    for _ in range(args.warmup):
        nd.nd_factor_and_solve(L, E, b)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, _, x = nd.nd_factor_and_solve(L, E, b)
        ts.append(time.perf_counter() - t0)
    eta = float(nd.backward_error(L, E, x, b)[0])
    sec = statistics.mean(ts)
    value = 1.0 / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": "one full FP64 factor_and_solve of the workload system per step "
                                   "(NumPy oracle restating socu's level loop; BLAS threads = host cores)"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "backward_error": eta,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


def dmma_peak_tflops(dev):
    """FP64 tensor-core (DMMA) throughput of this GPU: socu_dmma_peak_launch
    (register-only mma.sync m8n8k4 f64 chains, 2 CTAs x 256 threads per SM),
    best of 3 launches timed with CUDA events."""
    import ctypes

    import torch

    from socu_b200 import _lib
    lib = _lib.load()
    sink = torch.zeros(1, dtype=torch.float64, device=dev)
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    st = torch.cuda.current_stream(dev).cuda_stream
    best = 0.0
    for _ in range(4):
        fl = ctypes.c_double(0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        _lib.check(lib.socu_dmma_peak_launch(2 * sms, 256, 20000, sink.data_ptr(), st, ctypes.byref(fl)),
                   "socu_dmma_peak_launch")
        b.record()
        torch.cuda.synchronize(dev)
        best = max(best, fl.value / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best


def level_counts(N):
    """Per level: (d, r, l, both) = nodes, nodes with a right / left neighbour, with both."""
    s, out = 1, []
    for _ in range(N.bit_length()):
        d = (N + s) // (2 * s)
        nodes = [s - 1 + 2 * s * t for t in range(d)]
        r = sum(1 for i in nodes if i + s < N)
        lft = sum(1 for i in nodes if i >= s)
        both = sum(1 for i in nodes if i + s < N and i >= s)
        out.append((d, r, lft, both))
        s *= 2
    return out


def node_flops(N, n, m):
    """Algorithmic flops of the level-node work of a factor_and_solve: potrf
    n^3/3 per node, trsm n^3 per coupling side, forward step 2 n^2 m per node."""
    return sum(d * n ** 3 / 3 + (r + lft) * n ** 3 + 2 * d * n * n * m for d, r, lft, _ in level_counts(N))


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from socu_b200.block_tridiag_solver import (copy_lower_blocks, create_cholesky_backward_substitution_launch,
                                                create_cholesky_factor_and_solve_launch, create_cholesky_factor_launch)
    from socu_b200 import _lib as socu_lib

    def lower_blocks_bytes(t):
        n = int(t.shape[-1])
        return int(socu_lib.load().socu_lower_blocks_bytes(t.numel() // (n * n), n, t.element_size()))
    from socu_b200.mixed import backward_error, create_cholesky_refined_solve_launch

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    Lh0, Eh0, bh0 = make_problem_host()
    L0, E0, b0 = Lh0.to(dev), Eh0.to(dev), bh0.to(dev)
    x = torch.zeros_like(b0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    # mixed + refinement (headline), inputs read-only
    mixed = create_cholesky_refined_solve_launch(L0, E0, b0, x, tol=TOL, max_iter=MAX_ITER, use_cuda_graph=True)
    if args.profile:
        # profiler runs: ncu does not report kernels inside the conditional WHILE
        # graph node, so run the same kernels without a graph, with max_iter set to
        # the rounds the graph run needs (the graph only adds its loop-control kernels)
        mixed()
        torch.cuda.synchronize(dev)
        rounds = max(1, int(mixed.iterations.abs().max()))
        mixed = create_cholesky_refined_solve_launch(L0, E0, b0, x, tol=TOL, max_iter=rounds, use_cuda_graph=False)
    # plain FP64 factor_and_solve on working copies (in place); FP64 factor alone
    Lw, Ew, xw = L0.clone(), E0.clone(), b0.clone()
    plain = create_cholesky_factor_and_solve_launch(Lw, Ew, xw, use_cuda_graph=True)
    fac64 = create_cholesky_factor_launch(Lw, Ew, use_cuda_graph=True)
    # the float backward sweep of the mixed solve (HBM-bound secondary roofline)
    L32, E32 = L0.float(), E0.float()
    create_cholesky_factor_launch(L32, E32, dtype=torch.float32, keep_inverse=True)()
    b32 = b0.float()
    x32 = b32.clone()
    bwd32 = create_cholesky_backward_substitution_launch(L32, E32, x32, dtype=torch.float32, use_cuda_graph=True,
                                                         factor_has_inverse=True)
    sweep_launches = bwd32.kernel_count

    def time_steps(fn, reset, k):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(k)]
        for a, bev in evs:
            reset()
            flush.zero_()
            a.record()
            fn()
            bev.record()
        torch.cuda.synchronize(dev)
        return [a.elapsed_time(bev) * 1e-3 for a, bev in evs]

    def reset_plain():
        Lw.copy_(L0); Ew.copy_(E0); xw.copy_(b0)

    def reset_bwd():
        x32.copy_(b32)

    nothing = lambda: None
    # clocks are sampled over the whole measurement window (every timed region
    # below); nvidia-smi needs about a second before its first sample
    sampler = ClockSampler(local_rank)
    sampler.__enter__()
    time.sleep(1.5)
    for _ in range(args.warmup):
        mixed(); reset_plain(); plain(); reset_bwd(); bwd32(); reset_plain(); fac64()
    barrier()
    t_mixed = time_steps(mixed, nothing, args.steps)
    barrier()
    t_plain = time_steps(plain, reset_plain, args.steps)
    x_plain = xw.clone()
    t_fac64 = time_steps(fac64, reset_plain, args.steps)
    t_bwd = time_steps(bwd32, reset_bwd, args.steps)
    barrier()

    eta_dev = float(mixed.eta.max())
    iters = int(mixed.iterations.max())
    eta_check = float(backward_error(L0, E0, x, b0).max())
    eta_plain = float(backward_error(L0, E0, x_plain, b0).max())
    x_mixed = x.clone()

    # per-phase budget: one eager run of each solve with CUDA events around
    # every kernel (the mixed solve with exactly the rounds the graph ran)
    prof_mixed = create_cholesky_refined_solve_launch(L0, E0, b0, torch.zeros_like(b0), tol=TOL,
                                                      max_iter=max(1, abs(iters)), use_cuda_graph=False)
    reset_plain()
    phases_plain = plain.profile()
    phases_mixed = prof_mixed.profile()
    del prof_mixed
    dmma_tf = dmma_peak_tflops(dev)

    # the other shifts of this configuration: s = 1 and 0.1 make the README
    # matrix numerically indefinite (the diagonal factor blocks tril(randn) + s I
    # are numerically singular), so both paths must report the breakdown
    shift_sweep = {f"{SHIFT:g}": {"mixed_eta": eta_dev, "mixed_iterations": iters, "fp64_info": 0}}
    for s_alt in (1.0, 0.1):
        from socu_b200.problems import readme_blocks
        La, Ea, ba = readme_blocks(N_BLOCKS, BLOCK, NRHS, shift=s_alt, seed=SEED, batch=1, device=dev)
        xa = torch.zeros_like(ba)
        ra = create_cholesky_refined_solve_launch(La, Ea, ba, xa, tol=TOL, max_iter=3, use_cuda_graph=False)
        ra()
        info = torch.zeros(1, dtype=torch.int32, device=dev)
        create_cholesky_factor_and_solve_launch(La, Ea, ba, info=info)()
        torch.cuda.synchronize(dev)
        shift_sweep[f"{s_alt:g}"] = {"mixed_eta": float(ra.eta.max()), "mixed_iterations": int(ra.iterations.min()),
                                     "fp64_info": int(info[0]),
                                     "status": "breakdown reported (numerically indefinite)"
                                     if (int(info[0]) != 0 and not float(ra.eta.max()) <= TOL) else "solved"}
        del La, Ea, ba, xa, ra

    # e2e through the public API with host buffers (pinned), copies inside the timed region
    Lh = L0.cpu().pin_memory(); Eh = E0.cpu().pin_memory(); bh = b0.cpu().pin_memory()
    xh = torch.empty_like(x, device="cpu").pin_memory()
    # L travels as the lower triangles of its blocks (copy_lower_blocks: 16-row
    # bands), the only part any kernel reads; the rest of the device copy is
    # zeroed once, outside the timed region
    Ld, Ed, bd, xd = torch.zeros_like(L0), torch.empty_like(E0), torch.empty_like(b0), torch.empty_like(b0)
    e2e_run = create_cholesky_refined_solve_launch(Ld, Ed, bd, xd, tol=TOL, max_iter=MAX_ITER, use_cuda_graph=True)

    # the mixed solve reads only the N-1 coupling slots of E (the storage tail
    # is never touched), so only those cross the bus
    ncpl = N_BLOCKS - 1
    Ein = Eh[:, :ncpl]

    def e2e_step():
        copy_lower_blocks(Ld, Lh); Ed[:, :ncpl].copy_(Ein, non_blocking=True); bd.copy_(bh, non_blocking=True)
        e2e_run()
        xh.copy_(xd, non_blocking=True)

    for _ in range(2):
        e2e_step()
    t_e2e_serial = time_steps(e2e_step, nothing, max(3, args.steps // 2))
    h2d = lower_blocks_bytes(Lh) + Ein.numel() * 8 + bh.numel() * 8
    d2h = xh.numel() * 8

    # The same e2e steps as a streaming caller runs them: two device buffer
    # sets, the host->device copy of step k+1 and the device->host copy of
    # step k overlapping the solve of step k (three streams).  Every step
    # still copies its inputs in and its solution out inside the timed region.
    h2d_s, ks, d2h_s = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    bufs = [(torch.zeros_like(L0), torch.empty_like(E0), torch.empty_like(b0), torch.empty_like(b0)) for _ in range(2)]
    xhs = [torch.empty_like(x, device="cpu").pin_memory() for _ in range(2)]
    runs = [create_cholesky_refined_solve_launch(Lb, Eb, bb, xb, tol=TOL, max_iter=MAX_ITER, use_cuda_graph=True,
                                                 stream=ks) for (Lb, Eb, bb, xb) in bufs]
    copied = [torch.cuda.Event() for _ in range(2)]
    computed = [torch.cuda.Event() for _ in range(2)]
    done = [torch.cuda.Event() for _ in range(2)]

    def pipeline(k_steps):
        for ev in done:
            ev.record(d2h_s)
        for k in range(k_steps):
            j = k % 2
            Lb, Eb, bb, xb = bufs[j]
            h2d_s.wait_event(done[j])
            with torch.cuda.stream(h2d_s):
                copy_lower_blocks(Lb, Lh); Eb[:, :ncpl].copy_(Ein, non_blocking=True)
                bb.copy_(bh, non_blocking=True)
            copied[j].record(h2d_s)
            ks.wait_event(copied[j])
            runs[j]()
            computed[j].record(ks)
            d2h_s.wait_event(computed[j])
            with torch.cuda.stream(d2h_s):
                xhs[j].copy_(xb, non_blocking=True)
            done[j].record(d2h_s)

    pipeline(4)
    torch.cuda.synchronize(dev)
    k_pipe = max(4, args.steps)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    ev0.record(h2d_s)
    pipeline(k_pipe)
    ev1.record(d2h_s)
    torch.cuda.synchronize(dev)
    t_e2e = [ev0.elapsed_time(ev1) * 1e-3 / k_pipe]
    e2e_eta = max(float(r.eta.max()) for r in runs)
    del runs, bufs, xhs

    def agg(ts):
        return max_over_ranks(statistics.mean(ts), world, dev)

    sec_mixed, sec_plain, sec_bwd, sec_e2e = agg(t_mixed), agg(t_plain), agg(t_bwd), agg(t_e2e)
    sec_fac64 = agg(t_fac64)
    sec_e2e_serial = agg(t_e2e_serial)
    del e2e_run, Ld, Ed, bd, xd, Lw, Ew, xw, L32, E32, x32, b32
    torch.cuda.empty_cache()
    st = bench_stress(dev, args.steps, time_steps, agg, dmma_tf) if not args.skip_extra else None
    rg = bench_ragged(dev, args.steps, time_steps, agg, world, rank) if not args.skip_extra else None
    ad = bench_autograd(dev, args.steps, time_steps, agg) if not args.skip_extra else None
    barrier()
    sampler.__exit__(None, None, None)
    if rank != 0:
        return
    n, N, m = BLOCK, N_BLOCKS, NRHS
    S = storage_len(N)
    hbm_peak, bf16_peak, peak_src = measured_peaks()
    # accuracy against LAPACK's banded FP64 Cholesky of the same system
    Lh_np, Eh_np, bh_np = Lh0[0].numpy(), Eh0[0].numpy(), bh0[0].numpy()
    x_band = band_solve_fp64(Lh_np, Eh_np, bh_np)
    fwd_mixed = forward_error(x_mixed[0].cpu().numpy(), x_band)
    fwd_plain = forward_error(x_plain[0].cpu().numpy(), x_band)
    # dominant kernel of the mixed solve: the largest share of its profile
    dom = max(phases_mixed, key=lambda k: phases_mixed[k][0])
    node_ms, node_launches = phases_mixed["node"]
    nf = node_flops(N, n, m)
    node_ach = nf / node_launches / (node_ms * 1e-3 / node_launches) / 1e12
    # algorithmic bytes of one backward sweep: every diagonal block (with its
    # inverse) and every coupling slot read once, x read three times and
    # written once per node, 4-byte floats; per launch = sweep / launches
    sweep_bytes = ((N + S) * n * n + 4.0 * N * n * m) * 4
    bwd_ach = sweep_bytes / sweep_launches / (sec_bwd / sweep_launches) / 1e9
    fac_flops = algorithmic_factor_flops(N, n)
    fac64_tf = fac_flops / sec_fac64 / 1e12
    cores = len(os.sched_getaffinity(0))
    cpu_v, cpu_ts = cpu_oracle_solves_per_s(Lh_np, Eh_np, bh_np)
    value = world / sec_mixed

    def budget(ph):
        return {k: {"ms": round(v[0], 4), "launches": v[1]} for k, v in ph.items()}

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec_mixed * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor + f64 refinement", "data": "synthetic",
        "config": dict(workload_config(), parallelism=f"replicas x{world} (one system per GPU)"),
        "fp64_plain": {"value": world / sec_plain, "unit": "solves/s", "ms_per_step": sec_plain * 1e3,
                       "backward_error": eta_plain, "forward_error": fwd_plain,
                       "roofline": {"kernel": "FP64 factor (k_node<double> + k_update<double>, graph-launched)",
                                    "bound": "fp64 tensor (DMMA)", "achieved": fac64_tf, "peak": dmma_tf,
                                    "unit": "TFLOP/s", "frac": fac64_tf / dmma_tf,
                                    "peak_source": "measured in this run: socu_dmma_peak_launch (register-only "
                                                   "mma.sync m8n8k4 f64 chains); the device file has no FP64 figure",
                                    "algorithmic_flops": fac_flops, "ms": sec_fac64 * 1e3},
                       "phases": budget(phases_plain)},
        "mixed_over_fp64": sec_plain / sec_mixed,
        "backward_error": {"max": eta_dev, "recomputed": eta_check, "iterations": iters},
        "shift_sweep": dict(shift_sweep, note="fp64_info: 1 + first failing node of the plain FP64 factor, 0 = SPD"),
        "forward_error": {"mixed": fwd_mixed, "fp64_plain": fwd_plain,
                          "reference": "LAPACK banded FP64 Cholesky (scipy solveh_banded) of the same system"},
        "factor_flops_fp": fac_flops,
        "phases": dict(budget(phases_mixed), note="one eager run with CUDA events around every kernel, "
                       f"{abs(iters)} rounds; events add gaps, so the sum exceeds ms_per_step"),
        "roofline": {"kernel": f"k_node<float> (level nodes of the mixed solve: potrf + coupling solves + forward "
                               f"step, averaged over its launches; the kernel with the most device time in the "
                               f"mixed solve's ncu launch list; this run's eager profile: node "
                               f"{node_ms:.3f} ms in {node_launches} launches, backward sweeps "
                               f"{phases_mixed.get('backward', (0.0, 0))[0]:.3f} ms in "
                               f"{phases_mixed.get('backward', (0.0, 0))[1]}, "
                               f"largest phase {dom})",
                     "bound": "tensor", "achieved": node_ach, "peak": bf16_peak, "unit": "TFLOP/s",
                     "frac": node_ach / bf16_peak, "peak_source": f"{peak_src} (bf16 dense, MEASURED_PEAKS.json)",
                     "traffic": NODE_TRAFFIC_BYTES, "traffic_source": NODE_TRAFFIC_NOTE,
                     "algorithmic_flops_per_launch": nf / node_launches,
                     "ms_per_launch": node_ms / node_launches},
        "roofline_sweep": {"kernel": "k_bwd<float, resident, inverse> (backward sweep of the mixed solve; "
                                     f"{sweep_launches} launches per sweep, averaged)", "bound": "hbm",
                           "achieved": bwd_ach, "peak": hbm_peak, "unit": "GB/s", "frac": bwd_ach / hbm_peak,
                           "peak_source": peak_src, "traffic": TRAFFIC_BYTES,
                           "algorithmic_bytes": sweep_bytes / sweep_launches,
                           "ms_per_launch": sec_bwd / sweep_launches * 1e3, "traffic_source": TRAFFIC_NOTE},
        "fp64_dmma_peak_tflops": dmma_tf,
        "cpu_baseline": {"value": cpu_v, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": f"full FP64 factor_and_solve runs of the workload system for ~{CPU_SAMPLE_S:.0f} s, "
                                   f"median of {len(cpu_ts)} ({min(cpu_ts):.3f}-{max(cpu_ts):.3f} s)"},
        "e2e": {"value": world / sec_e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": sec_e2e * 1e3,
                "mode": "pipelined: two device buffer sets, copies of neighbouring steps overlap the solve "
                        "(inputs re-copied from pinned host memory every step: the lower triangles of L's "
                        "blocks in 16-row bands (copy_lower_blocks; no kernel reads above them), E[:N-1], b; "
                        "working set 2 x 71 MB plus workspaces > L2)",
                "backward_error_max": e2e_eta,
                "serial": {"value": world / sec_e2e_serial, "ms_per_step": sec_e2e_serial * 1e3,
                           "mode": "copy in, solve, copy out, one step at a time, L2 flushed before each"}},
        # graph run: the prologue holds the first round; the WHILE loop runs the others
        "gpu_launches": (mixed.kernel_count + max(abs(iters) - 1, 0) * mixed.round_kernel_count) * args.steps,
        "clocks": dict(sampler.summary(), window="100 ms samples over all timed regions of this run "
                                                  "(workload, e2e, stress, ragged, autograd) and their warm-ups"),
    }
    if st is not None:
        line["stress"] = st
    if rg is not None:
        line["ragged"] = rg
    if ad is not None:
        line["autograd"] = ad
    print(json.dumps(line), flush=True)


STRESS_N, STRESS_n, STRESS_m, STRESS_SHIFT, STRESS_SHIFT_LITERAL = 16384, 128, 32, 24.0, 0.05


def bench_stress(dev, steps, time_steps, agg, dmma_tf):
    """Large shape N=16384, n=128, m=32 (~6.4 GB of FP64 blocks): mixed +
    refinement against the plain FP64 path on the same system.  Shift 24
    instead of the literal 0.05, at which the README matrix is numerically
    indefinite (no Cholesky factors it); the literal shift is run once to
    report the breakdown status of both paths."""
    import torch

    from socu_b200.block_tridiag_solver import create_cholesky_factor_and_solve_launch, create_cholesky_factor_launch
    from socu_b200.mixed import backward_error, create_cholesky_refined_solve_launch
    from socu_b200.problems import readme_blocks

    N, n, m = STRESS_N, STRESS_n, STRESS_m
    L0, E0, b0 = readme_blocks(N, n, m, shift=STRESS_SHIFT, seed=SEED, batch=1, device=dev)
    x = torch.zeros_like(b0)
    mixed = create_cholesky_refined_solve_launch(L0, E0, b0, x, tol=TOL, max_iter=MAX_ITER, use_cuda_graph=True)
    Lw, Ew, xw = L0.clone(), E0.clone(), b0.clone()
    plain = create_cholesky_factor_and_solve_launch(Lw, Ew, xw, use_cuda_graph=True)
    fac64 = create_cholesky_factor_launch(Lw, Ew, use_cuda_graph=True)

    def reset():
        Lw.copy_(L0); Ew.copy_(E0); xw.copy_(b0)

    mixed(); reset(); plain(); reset(); fac64()
    torch.cuda.synchronize(dev)
    k = max(3, steps // 3)
    t_m = time_steps(mixed, lambda: None, k)
    t_p = time_steps(plain, reset, k)
    x_plain = xw.clone()
    t_f = time_steps(fac64, reset, k)
    eta_m = float(backward_error(L0, E0, x, b0).max())
    eta_p = float(backward_error(L0, E0, x_plain, b0).max())
    fwd = float((x - x_plain).abs().max() / x_plain.abs().max())
    iters = int(mixed.iterations.max())
    try:
        prof = create_cholesky_refined_solve_launch(L0, E0, b0, torch.zeros_like(b0), tol=TOL,
                                                    max_iter=max(1, abs(iters)), use_cuda_graph=False).profile()
        phases = {k: {"ms": round(v[0], 3), "launches": v[1]} for k, v in prof.items()}
    except RuntimeError as exc:   # the budget is a diagnostic: report instead of failing the line
        phases = {"error": str(exc)}
    sec_m, sec_p, sec_f = agg(t_m), agg(t_p), agg(t_f)
    fac_flops = algorithmic_factor_flops(N, n)
    del mixed, plain, fac64, Lw, Ew, xw, L0, E0, b0, x, x_plain
    torch.cuda.empty_cache()
    # the literal shift: both paths must report the breakdown rather than a number
    L1, E1, b1 = readme_blocks(N, n, m, shift=STRESS_SHIFT_LITERAL, seed=SEED, batch=1, device=dev)
    x1 = torch.zeros_like(b1)
    brk = create_cholesky_refined_solve_launch(L1, E1, b1, x1, tol=TOL, max_iter=3, use_cuda_graph=False)
    brk()
    eta_brk, it_brk = float(brk.eta.max()), int(brk.iterations.min())
    create_cholesky_factor_and_solve_launch(L1, E1, b1)()
    finite_plain = bool(torch.isfinite(b1).all())
    del brk, L1, E1, b1, x1
    torch.cuda.empty_cache()
    fac_tf = fac_flops / sec_f / 1e12
    return {
        "workload": f"N={N} n={n} m={m} single system, README construction with shift {STRESS_SHIFT:g}",
        "deviation": f"shift {STRESS_SHIFT_LITERAL:g} (as specified) is numerically indefinite: see breakdown",
        "mixed_refine": {"value": 1.0 / sec_m, "unit": "solves/s", "ms_per_step": sec_m * 1e3, "eta_max": eta_m,
                         "iterations": iters, "forward_error_vs_fp64_plain": fwd,
                         "phases": phases},
        "fp64_plain": {"value": 1.0 / sec_p, "unit": "solves/s", "ms_per_step": sec_p * 1e3, "eta_max": eta_p,
                       "factor_ms": sec_f * 1e3, "factor_tflops": fac_tf, "factor_frac_of_dmma_peak": fac_tf / dmma_tf},
        "mixed_over_fp64": sec_p / sec_m,
        "factor_flops": fac_flops,
        "breakdown_at_literal_shift": {"mixed_eta": eta_brk, "mixed_iterations": it_brk,
                                       "fp64_solution_finite": finite_plain},
    }


def bench_ragged(dev, steps, time_steps, agg, world=1, rank=0):
    """Uneven MPC-style batch in one persistent launch: FP64 plain and float
    factor + FP64 refinement.  The packed inputs (several GB) exceed L2.
    Under several ranks each rank solves its contiguous share of the
    instances (balanced by factor work, no exchange)."""
    import torch

    from socu_b200.problems import fill_ragged, ragged_shapes
    from socu_b200.ragged import (RaggedBatch, create_ragged_factor_and_solve_launch,
                                  create_ragged_refined_solve_launch, shard_instances)

    Ns, ns, ms = ragged_shapes(RAGGED_SEED, RAGGED_COUNT)
    flops = sum(algorithmic_factor_flops(int(N), int(n)) for N, n in zip(Ns, ns))
    lo, hi = shard_instances(Ns, ns, world, rank)
    Ns, ns, ms = Ns[lo:hi], ns[lo:hi], ms[lo:hi]
    plain_b = RaggedBatch(Ns, ns, ms, dtype=torch.float64, device=dev)
    L, E, b = plain_b.empty()
    fill_ragged(plain_b, L, E, b, seed=RAGGED_SEED + lo)
    mixed_b = RaggedBatch(Ns, ns, ms, dtype=torch.float64, device=dev, refine=True, max_iter=MAX_ITER)
    x = torch.zeros_like(b)
    run_m = create_ragged_refined_solve_launch(mixed_b, L, E, b, x, tol=TOL)
    Lw, Ew, xw = L.clone(), E.clone(), b.clone()
    run_p = create_ragged_factor_and_solve_launch(plain_b, Lw, Ew, xw)

    def reset():
        Lw.copy_(L); Ew.copy_(E); xw.copy_(b)

    for _ in range(2):
        run_m(); reset(); run_p()
    torch.cuda.synchronize(dev)
    k = max(3, steps // 2)
    t_m = time_steps(run_m, lambda: None, k)
    t_p = time_steps(run_p, reset, k)
    errs = (mixed_b.error_flag(), plain_b.error_flag())
    sec_m, sec_p = agg(t_m), agg(t_p)
    # per-instance forward error of the mixed solution against the plain FP64 one
    reset()
    run_p()
    sizes = torch.as_tensor(Ns * ns * ms, device=dev)
    inst = torch.repeat_interleave(torch.arange(len(Ns), device=dev), sizes)
    dx = torch.zeros(len(Ns), dtype=torch.float64, device=dev).scatter_reduce(0, inst, (x - xw).abs(), "amax")
    xm = torch.zeros(len(Ns), dtype=torch.float64, device=dev).scatter_reduce(0, inst, xw.abs(), "amax")
    fwd = float((dx / xm.clamp_min(1e-300)).max())
    out = {
        "workload": RAGGED_WORKLOAD,
        "mixed_refine": {"value": RAGGED_COUNT / sec_m, "unit": "solves/s", "ms_per_step": sec_m * 1e3,
                         "eta_max": float(run_m.eta.max()), "iterations_max": int(run_m.iterations.max()),
                         "iterations_mean": float(run_m.iterations.double().mean()),
                         "forward_error_vs_fp64_plain_max": fwd},
        "fp64_plain": {"value": RAGGED_COUNT / sec_p, "unit": "solves/s", "ms_per_step": sec_p * 1e3,
                       "factor_gflops": flops / sec_p / 1e9},
        "instances_per_rank": [lo, hi],
        "mixed_over_fp64": sec_p / sec_m,
        "persistent_ctas": plain_b.grid,
        "queue_errors": list(errs),
        "packed_bytes_fp64": (L.numel() + E.numel() + 2 * b.numel()) * 8,
        "gpu_launches_per_solve": 2,
    }
    del run_m, run_p, L, E, b, x, Lw, Ew, xw
    return out


def bench_autograd(dev, steps, time_steps, agg):
    """Differentiable solve on 256 systems of N=128, n=16, m=1 (FP64): forward
    solve, loss = sum(w * x), backward (adjoint solve on the stored factor and
    the fused dD/dE kernel).  A step is one forward + backward pass."""
    import torch

    from socu_b200.autograd import block_tridiag_solve
    from socu_b200.problems import readme_blocks

    B, N, n, m = 256, 128, 16, 1
    L, E, b = readme_blocks(N, n, m, shift=10.0, seed=SEED, batch=B, device=dev)
    D = L.clone().requires_grad_(True)
    Ec = E[:, :N - 1].clone().requires_grad_(True)
    bb = b.clone().requires_grad_(True)
    w = torch.randn(B, N, n, m, dtype=torch.float64, device=dev, generator=torch.Generator(device=dev).manual_seed(1))

    def step():
        D.grad = Ec.grad = bb.grad = None
        x = block_tridiag_solve(D, Ec, bb)
        (w * x).sum().backward()

    for _ in range(3):
        step()
    torch.cuda.synchronize(dev)
    sec = agg(time_steps(step, lambda: None, max(3, steps // 2)))
    return {"workload": "256 systems, N=128, n=16, m=1, FP64, loss = sum(w*x), forward + backward",
            "value": B / sec, "unit": "solves/s (forward + backward)", "ms_per_step": sec * 1e3}


NCU_CASES = {
    # the mixed solve's float factor_and_solve on 4 systems of the workload shape (L, E float: 200 MB > L2)
    "node": dict(B=4, N=1024, n=64, m=8, shift=10.0),
    # the stress block size at a reduced horizon (FP64 blocks ~0.8 GB)
    "stress": dict(B=1, N=2048, n=128, m=32, shift=24.0),
}


def run_ncu_case(name):
    """Small eager workloads for ncu captures of single kernels (not a bench
    line): two factor_and_solve runs in float and two in FP64 of the case's
    shape, for n > 64 one float factor_and_solve with the tensor-memory node
    and the tensor-core Schur update, then one mixed solve without its CUDA
    graph (ncu does not report kernels inside conditional graph nodes)."""
    import torch

    from socu_b200.block_tridiag_solver import create_cholesky_factor_and_solve_launch
    from socu_b200.mixed import create_cholesky_refined_solve_launch
    from socu_b200.problems import readme_blocks

    c = NCU_CASES[name]
    L, E, b = readme_blocks(c["N"], c["n"], c["m"], shift=c["shift"], seed=SEED, batch=c["B"], device="cuda")
    for dt in (torch.float32, torch.float64):
        for _ in range(2):
            # copies: the FP64 inputs must stay intact for the next pass and the mixed solve
            Lw, Ew, xw = L.to(dt, copy=True), E.to(dt, copy=True), b.to(dt, copy=True)
            create_cholesky_factor_and_solve_launch(Lw, Ew, xw, dtype=dt)()
            torch.cuda.synchronize()
    if c["n"] > 64:
        # the tensor-memory float node (k_node_tm) with the tensor-core Schur update
        from socu_b200.block_tridiag_solver import _launch_with_settings
        Lw, Ew, xw = L.float(), E.float(), b.float()
        _launch_with_settings("factor_and_solve", Lw, Ew, xw, torch.float32,
                              {"node_tensor_cores": 4, "update_tensor_cores": 1}, use_cuda_graph=False)()
        torch.cuda.synchronize()
    x = torch.zeros_like(b)
    run = create_cholesky_refined_solve_launch(L, E, b, x, tol=TOL, max_iter=3, use_cuda_graph=False)
    run()
    torch.cuda.synchronize()
    print(json.dumps({"ncu_case": name, **c, "eta_max": float(run.eta.max())}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-extra", "--skip-ragged", dest="skip_extra", action="store_true",
                    help="omit the stress, ragged-batch and autograd measurements")
    ap.add_argument("--profile", action="store_true",
                    help="for profiler runs only: the mixed solve runs without its CUDA graph")
    ap.add_argument("--ncu-case", choices=sorted(NCU_CASES), default=None,
                    help="run a small eager workload for ncu kernel captures instead of the benchmark")
    args = ap.parse_args()
    if args.ncu_case:
        run_ncu_case(args.ncu_case)
        return
    args.warmup = max(args.warmup, 3) if args.impl == "ours" else args.warmup
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
