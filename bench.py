"""Benchmark: batched solves/s of the mixed-precision + FP64-refinement solver
versus the plain FP64 path, at normwise relative backward error <= 1e-12.

Workload: N=1024 blocks, n=64, m=8 right-hand sides, diagonal shift s=10,
one system per GPU (README generator, seeded).  A step is one full solve of
that system from its original blocks: float factor + refinement for the
headline value, FP64 factor_and_solve for the comparison line.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun every rank solves its own replica (the path does not shard);
value = systems solved by all ranks / max-over-ranks time.  The reference arm
times the CPU oracle (NumPy restatement of the reference algorithm) on the
host cores, rank 0 only.
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
TRAFFIC_BYTES = 5005218
TRAFFIC_NOTE = "ncu dram__bytes_read.sum + dram__bytes_write.sum, profiles/k_bwd_f32_inverse_sweep_N1024_n64_m8.md"
RAGGED_WORKLOAD = ("4096 independent systems, N ~ U{8..256}, n in {8,16,32,48}, m in {1,4}, shift=10, "
                   "instance i seeded with 0 + i, one persistent launch per solve")


def make_problem_gpu(dev):
    """The workload system on the device (README construction, torch generator)."""
    from socu_b200.problems import readme_blocks
    return readme_blocks(N_BLOCKS, BLOCK, NRHS, shift=SHIFT, seed=SEED, batch=1, device=dev)


def make_problem_host():
    """The workload system on the host for the reference arm (NumPy generator, same construction)."""
    from oracle.generators import readme_problem
    return readme_problem(N_BLOCKS, BLOCK, NRHS, shift=SHIFT, seed=SEED)


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
def cpu_oracle_solves_per_s(L, E, b, reps):
    from oracle import nd_cholesky as nd
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        nd.nd_factor_and_solve(L, E, b)
        ts.append(time.perf_counter() - t0)
    return 1.0 / statistics.median(ts), ts


def run_reference(args, rank):
    if rank != 0:
        return
    L, E, b = make_problem_host()
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
        "config": {"workload": WORKLOAD, "N": N_BLOCKS, "n": BLOCK, "m": NRHS, "shift": SHIFT,
                   "l2": "host CPU run"},
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
def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from socu_b200.block_tridiag_solver import (create_cholesky_backward_substitution_launch,
                                                create_cholesky_factor_and_solve_launch, create_cholesky_factor_launch)
    from socu_b200.mixed import backward_error, create_cholesky_refined_solve_launch

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    L0, E0, b0 = make_problem_gpu(dev)
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
    # plain FP64 factor_and_solve on working copies (in place)
    Lw, Ew, xw = L0.clone(), E0.clone(), b0.clone()
    plain = create_cholesky_factor_and_solve_launch(Lw, Ew, xw, use_cuda_graph=True)
    # the dominant kernel of the mixed solve: the float backward sweep on a
    # factor that carries its diagonal inverses (k_bwd<float, resident, inverse>),
    # one launch per level, timed as whole graph-launched sweeps
    L32, E32 = L0.float(), E0.float()
    create_cholesky_factor_launch(L32, E32, dtype=torch.float32, keep_inverse=True)()
    b32 = b0.float()
    x32 = b32.clone()
    fac32 = create_cholesky_backward_substitution_launch(L32, E32, x32, dtype=torch.float32, use_cuda_graph=True,
                                                         factor_has_inverse=True)
    sweep_launches = fac32.kernel_count

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

    def reset_fac():
        x32.copy_(b32)

    nothing = lambda: None
    # clocks are sampled over the whole measurement window (every timed region
    # below); nvidia-smi needs about a second before its first sample
    sampler = ClockSampler(local_rank)
    sampler.__enter__()
    time.sleep(1.5)
    for _ in range(args.warmup):
        mixed(); reset_plain(); plain(); reset_fac(); fac32()
    barrier()
    t_mixed = time_steps(mixed, nothing, args.steps)
    barrier()
    t_plain = time_steps(plain, reset_plain, args.steps)
    t_fac = time_steps(fac32, reset_fac, args.steps)
    barrier()

    eta_dev = float(mixed.eta.max())
    iters = int(mixed.iterations.max())
    eta_check = float(backward_error(L0, E0, x, b0).max())
    x_plain = xw.clone()
    eta_plain = float(backward_error(L0, E0, x_plain, b0).max())

    # e2e through the public API with host buffers (pinned), copies inside the timed region
    Lh = L0.cpu().pin_memory(); Eh = E0.cpu().pin_memory(); bh = b0.cpu().pin_memory()
    xh = torch.empty_like(x, device="cpu").pin_memory()
    Ld, Ed, bd, xd = torch.empty_like(L0), torch.empty_like(E0), torch.empty_like(b0), torch.empty_like(b0)
    e2e_run = create_cholesky_refined_solve_launch(Ld, Ed, bd, xd, tol=TOL, max_iter=MAX_ITER, use_cuda_graph=True)

    # the mixed solve reads only the N-1 coupling slots of E (the storage tail
    # is never touched), so only those cross the bus
    ncpl = N_BLOCKS - 1
    Ein = Eh[:, :ncpl]

    def e2e_step():
        Ld.copy_(Lh, non_blocking=True); Ed[:, :ncpl].copy_(Ein, non_blocking=True); bd.copy_(bh, non_blocking=True)
        e2e_run()
        xh.copy_(xd, non_blocking=True)

    for _ in range(2):
        e2e_step()
    t_e2e_serial = time_steps(e2e_step, nothing, max(3, args.steps // 2))
    h2d = Lh.numel() * 8 + Ein.numel() * 8 + bh.numel() * 8
    d2h = xh.numel() * 8

    # The same e2e steps as a streaming caller runs them: two device buffer
    # sets, the host->device copy of step k+1 and the device->host copy of
    # step k overlapping the solve of step k (three streams).  Every step
    # still copies its inputs in and its solution out inside the timed region.
    h2d_s, ks, d2h_s = torch.cuda.Stream(dev), torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    bufs = [(torch.empty_like(L0), torch.empty_like(E0), torch.empty_like(b0), torch.empty_like(b0)) for _ in range(2)]
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
                Lb.copy_(Lh, non_blocking=True); Eb[:, :ncpl].copy_(Ein, non_blocking=True)
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

    sec_mixed, sec_plain, sec_fac, sec_e2e = agg(t_mixed), agg(t_plain), agg(t_fac), agg(t_e2e)
    sec_e2e_serial = agg(t_e2e_serial)
    del e2e_run, Ld, Ed, bd, xd, Lw, Ew, xw, L32, E32, x32, b32
    torch.cuda.empty_cache()
    rg = bench_ragged(dev, args.steps, time_steps, agg) if not args.skip_ragged else None
    ad = bench_autograd(dev, args.steps, time_steps, agg) if not args.skip_ragged else None
    barrier()
    sampler.__exit__(None, None, None)
    if rank != 0:
        return
    n, N, m = BLOCK, N_BLOCKS, NRHS
    S = storage_len(N)
    # algorithmic bytes of one backward sweep: every diagonal block (with its
    # inverse) and every coupling slot read once, x read three times and
    # written once per node, 4-byte floats; per launch = sweep / launches
    sweep_bytes = ((N + S) * n * n + 4.0 * N * n * m) * 4
    fac_bytes = sweep_bytes / sweep_launches
    sec_fac = sec_fac / sweep_launches
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak, peak_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        hbm_peak, peak_src = float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    achieved = fac_bytes / sec_fac / 1e9
    cores = len(os.sched_getaffinity(0))
    cpu_v, cpu_ts = cpu_oracle_solves_per_s(L0[0].cpu().numpy(), E0[0].cpu().numpy(), b0[0].cpu().numpy(), reps=2)
    value = world / sec_mixed
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sec_mixed * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 factor + f64 refinement", "data": "synthetic",
        "config": {"workload": WORKLOAD, "N": N, "n": n, "m": m, "shift": SHIFT, "tol": TOL,
                   "max_iter": MAX_ITER, "l2": "256 MB flush before every timed step",
                   "parallelism": f"replicas x{world} (one system per GPU)"},
        "fp64_plain": {"value": world / sec_plain, "unit": "solves/s", "ms_per_step": sec_plain * 1e3,
                       "backward_error": eta_plain},
        "mixed_over_fp64": sec_plain / sec_mixed,
        "backward_error": {"max": eta_dev, "recomputed": eta_check, "iterations": iters},
        "factor_flops_fp": algorithmic_factor_flops(N, n),
        "roofline": {"kernel": "k_bwd<float, resident, inverse> (backward sweep of the mixed solve; "
                               f"{sweep_launches} launches per sweep, averaged)", "bound": "hbm",
                     "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "peak_source": peak_src, "traffic": TRAFFIC_BYTES,
                     "algorithmic_bytes": fac_bytes, "ms_per_launch": sec_fac * 1e3,
                     "traffic_source": TRAFFIC_NOTE},
        "cpu_baseline": {"value": cpu_v, "unit": "solves/s", "cores": cores, "kind": "port",
                         "sample": "one FP64 factor_and_solve of the workload system, median of 2 "
                                   f"({[round(t, 3) for t in cpu_ts]} s)"},
        "e2e": {"value": world / sec_e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": sec_e2e * 1e3,
                "mode": "pipelined: two device buffer sets, copies of neighbouring steps overlap the solve "
                        "(inputs L, E[:N-1], b re-copied from pinned host memory every step; working set "
                        "2 x 71 MB plus workspaces > L2)",
                "backward_error_max": e2e_eta,
                "serial": {"value": world / sec_e2e_serial, "ms_per_step": sec_e2e_serial * 1e3,
                           "mode": "copy in, solve, copy out, one step at a time, L2 flushed before each"}},
        # graph run: the prologue holds the first round; the WHILE loop runs the others
        "gpu_launches": (mixed.kernel_count + max(abs(iters) - 1, 0) * mixed.round_kernel_count) * args.steps,
        "clocks": dict(sampler.summary(), window="100 ms samples over all timed regions of this run "
                                                  "(workload, e2e, ragged) and their warm-ups"),
    }
    if rg is not None:
        line["ragged"] = rg
    if ad is not None:
        line["autograd"] = ad
    print(json.dumps(line), flush=True)


def bench_ragged(dev, steps, time_steps, agg):
    """Uneven MPC-style batch in one persistent launch: FP64 plain and float
    factor + FP64 refinement.  The packed inputs (several GB) exceed L2."""
    import torch

    from socu_b200.problems import fill_ragged, ragged_shapes
    from socu_b200.ragged import (RaggedBatch, create_ragged_factor_and_solve_launch,
                                  create_ragged_refined_solve_launch)

    Ns, ns, ms = ragged_shapes(RAGGED_SEED, RAGGED_COUNT)
    plain_b = RaggedBatch(Ns, ns, ms, dtype=torch.float64, device=dev)
    L, E, b = plain_b.empty()
    fill_ragged(plain_b, L, E, b, seed=RAGGED_SEED)
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
    flops = sum(algorithmic_factor_flops(int(N), int(n)) for N, n in zip(Ns, ns))
    out = {
        "workload": RAGGED_WORKLOAD,
        "mixed_refine": {"value": RAGGED_COUNT / sec_m, "unit": "solves/s", "ms_per_step": sec_m * 1e3,
                         "eta_max": float(run_m.eta.max()), "iterations_max": int(run_m.iterations.max()),
                         "iterations_mean": float(run_m.iterations.double().mean())},
        "fp64_plain": {"value": RAGGED_COUNT / sec_p, "unit": "solves/s", "ms_per_step": sec_p * 1e3,
                       "factor_gflops": flops / sec_p / 1e9},
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--skip-ragged", action="store_true", help="omit the ragged-batch and autograd measurements")
    ap.add_argument("--profile", action="store_true",
                    help="for profiler runs only: the mixed solve runs without its CUDA graph")
    args = ap.parse_args()
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
