"""Autotuner for the launch settings of the nested-dissection solver.

No counterpart in the reference: its factories take ``block_dim`` (threads
per tile block) and ``block_size`` (tile size of the blocked kernels) per call,
with defaults from a fixed table (``optimal_problem_settings``,
socu/block_tridiag_solver.py:26-60, 776-781).  Here the native library reads
launch settings from a table keyed on (dtype, n, n_rhs) (``socu_tuning_set``);
this module fills that table by measurement and keeps the results in an
on-disk cache, so a process tunes a shape once and later processes reuse it.

Settings (``socu_tuning``; 0 = built-in heuristic):
    node_threads, update_threads, sweep_threads   threads per CTA: 64, 128, 256
    sweep_tensor_cores   float sweeps on inverse-carrying factors: 1 FP64
                         tensor-core products, 2 SIMT row dots
    update_tile          output tile of the blocked Schur update (n > 64): 16, 32
    ragged_units         level nodes per task chunk of a ragged batch: 1..64
    update_tensor_cores  Schur updates of float factors (n <= 128) on the
                         tcgen05 tensor cores, 3xTF32 (1), or not (2)
    node_tensor_cores    products of float level nodes (n <= 128) on the
                         tcgen05 tensor cores at every level (1), on wide
                         levels only (3), or SIMT (2); 64 < n <= 128: the
                         node resident in tensor memory, trailing updates on
                         the tensor cores (4)

Search: coordinate descent from the built-in heuristics.  Each knob in turn
is tried at every value with the others held at the best so far; a candidate
is timed as the median of graph-launched runs of the tuned operation on a
synthetic system of the requested shape (README construction, inputs restored
by a device copy outside the timed region).  A candidate replaces the
incumbent only when it is faster by more than ``min_gain`` (default 2 %), so
noise does not churn the table.

Cache: JSON at ``$SOCU_TUNE_CACHE`` (default ``~/.cache/socu_b200/tune.json``),
entries keyed by device name, dtype, n and n_rhs.  ``load_cache()`` installs
the entries for the current device into the library; the factories call it
once per process.  ``SOCU_AUTOTUNE=1`` makes the factories tune shapes that
have no entry on first use (slow: one tuning run per new shape).
"""
from __future__ import annotations

import ctypes
import json
import os
import pathlib
import statistics
import threading

import torch

from . import _lib

__all__ = ["cache_path", "load_cache", "save_entry", "tune", "candidates", "current_settings", "install",
           "KNOBS", "maybe_autotune"]

KNOBS = ("update_tensor_cores", "node_tensor_cores", "node_threads", "sweep_tensor_cores", "sweep_threads",
         "update_threads", "update_tile")
_VALUES = {
    "node_threads": (0, 64, 128, 256),
    "update_threads": (0, 128, 256),
    "sweep_threads": (0, 64, 128, 256),
    "sweep_tensor_cores": (0, 1, 2),
    "update_tile": (0, 16, 32),
    "update_tensor_cores": (0, 1, 2),
    "node_tensor_cores": (0, 1, 3),
}
_loaded = set()
_tuned = set()
_lock = threading.Lock()


def cache_path() -> pathlib.Path:
    p = os.environ.get("SOCU_TUNE_CACHE")
    if p:
        return pathlib.Path(p)
    return pathlib.Path.home() / ".cache" / "socu_b200" / "tune.json"


def _dtype_name(dtype) -> str:
    return "float64" if dtype in (torch.float64, "float64") else "float32"


def _lib_dtype(dtype) -> int:
    return _lib.FLOAT64 if _dtype_name(dtype) == "float64" else _lib.FLOAT32


def _read(path: pathlib.Path) -> dict:
    try:
        with open(path) as f:
            data = json.load(f)
        if isinstance(data, dict) and data.get("version") == 1 and isinstance(data.get("entries"), list):
            return data
    except (OSError, ValueError):
        pass
    return {"version": 1, "entries": []}


def install(dtype, n: int, n_rhs: int, settings: dict | None):
    """Put one entry into the library's table (None removes it)."""
    lib = _lib.load()
    if settings is None:
        _lib.check(lib.socu_tuning_set(_lib_dtype(dtype), int(n), int(n_rhs), None), "socu_tuning_set")
        return
    t = _lib.Tuning.from_dict(settings)
    _lib.check(lib.socu_tuning_set(_lib_dtype(dtype), int(n), int(n_rhs), ctypes.byref(t)), "socu_tuning_set")


def current_settings(dtype, n: int, n_rhs: int) -> dict:
    """The library's effective entry for (dtype, n, n_rhs) (zeros where unset)."""
    t = _lib.Tuning()
    _lib.check(_lib.load().socu_tuning_get(_lib_dtype(dtype), int(n), int(n_rhs), ctypes.byref(t)),
               "socu_tuning_get")
    return t.as_dict()


def load_cache(device=None, path=None, device_name=None) -> int:
    """Install the cached entries for `device`'s GPU model (or for the model
    named `device_name`); returns how many.  Each (file, model) pair is read
    once per process."""
    if device_name is None:
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        device_name = torch.cuda.get_device_name(dev)
    name = device_name
    path = pathlib.Path(path) if path is not None else cache_path()
    key = (str(path), name)
    with _lock:
        if key in _loaded:
            return 0
        _loaded.add(key)
    count = 0
    for e in _read(path)["entries"]:
        if e.get("device") != name:
            continue
        install(e["dtype"], e["n"], e["n_rhs"], e["settings"])
        count += 1
    return count


def save_entry(device_name: str, dtype, n: int, n_rhs: int, settings: dict, ms: float, shape, path=None):
    """Add or replace one cache entry (atomic rewrite of the file)."""
    path = pathlib.Path(path) if path is not None else cache_path()
    path.parent.mkdir(parents=True, exist_ok=True)
    data = _read(path)
    key = (device_name, _dtype_name(dtype), int(n), int(n_rhs))
    data["entries"] = [e for e in data["entries"]
                       if (e.get("device"), e.get("dtype"), e.get("n"), e.get("n_rhs")) != key]
    data["entries"].append({"device": device_name, "dtype": _dtype_name(dtype), "n": int(n), "n_rhs": int(n_rhs),
                            "settings": {k: int(settings.get(k, 0)) for k in _lib.Tuning.FIELDS},
                            "ms": float(ms), "shape": [int(v) for v in shape]})
    tmp = path.with_suffix(path.suffix + f".tmp{os.getpid()}")
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def candidates(n: int, n_rhs: int, dtype) -> dict:
    """Values worth trying per knob for this shape (knobs that cannot matter are
    left out: the blocked update tile exists only for n > 64, and the sweep
    product switch only for float factors with n <= 64)."""
    out = {}
    for k in KNOBS:
        vals = list(_VALUES[k])
        if k == "update_tile" and n <= 64:
            continue
        if k == "sweep_tensor_cores" and (n > 64 or _dtype_name(dtype) == "float64"):
            continue
        if k == "update_tensor_cores" and (n > 128 or _dtype_name(dtype) == "float64"):
            continue
        if k == "node_tensor_cores" and (n > 128 or _dtype_name(dtype) == "float64"):
            continue
        if k == "node_tensor_cores" and n > 64:
            vals = vals + [4]
        out[k] = vals
    return out


def _time_op(op, dtype, settings, L0, E0, b0, reps, warmup):
    """Median device time (ms) of one graph-launched run with `settings`."""
    from .block_tridiag_solver import _launch_with_settings

    L, E, x = L0.clone(), E0.clone(), b0.clone()
    run = _launch_with_settings(op, L, E, x, dtype, settings)

    def reset():
        L.copy_(L0); E.copy_(E0); x.copy_(b0)

    ts = []
    for k in range(warmup + reps):
        reset()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        run()
        b.record()
        torch.cuda.synchronize()
        if k >= warmup:
            ts.append(a.elapsed_time(b))
    return statistics.median(ts), x


def tune(n: int, n_rhs: int, dtype=torch.float64, horizon: int = 256, batch: int = 1, op: str = "factor_and_solve",
         device=None, reps: int = 7, warmup: int = 2, min_gain: float = 0.02, save: bool = True, path=None,
         check=True):
    """Tune the settings of `op` ("factor_and_solve" or "solve") for blocks of
    size n with n_rhs right-hand sides in `dtype`, on a synthetic (batch,
    horizon) system; install the winner (key (dtype, n, n_rhs)) and, with
    `save`, write it to the cache.  Every candidate's result is checked against
    the default settings' result (relative difference <= 1e-10 for float64,
    1e-4 for float32) when `check` is set.  Returns (settings, ms, trials)."""
    from .problems import readme_blocks

    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    tdt = torch.float64 if _dtype_name(dtype) == "float64" else torch.float32
    L0, E0, b0 = readme_blocks(horizon, n, n_rhs, shift=10.0 + 0.25 * n ** 0.5, seed=0, batch=batch, device=dev)
    L0, E0, b0 = L0.to(tdt), E0.to(tdt), b0.to(tdt)
    if op == "solve":
        from .block_tridiag_solver import create_cholesky_factor_launch
        create_cholesky_factor_launch(L0, E0, dtype=tdt)()
    best = {k: 0 for k in _lib.Tuning.FIELDS}
    trials = []
    best_ms, x_ref = _time_op(op, tdt, best, L0, E0, b0, reps, warmup)
    trials.append((dict(best), best_ms))
    tol = 1e-10 if tdt == torch.float64 else 1e-4
    scale = float(x_ref.abs().max()) or 1.0
    for knob, values in candidates(n, n_rhs, tdt).items():
        for v in values:
            if v == best[knob]:
                continue
            trial = dict(best)
            trial[knob] = v
            ms, x = _time_op(op, tdt, trial, L0, E0, b0, reps, warmup)
            if check:
                err = float((x - x_ref).abs().max()) / scale
                if not err <= tol:
                    raise RuntimeError(f"autotune: settings {trial} changed the result by {err:.3e}")
            trials.append((trial, ms))
            if ms < best_ms * (1.0 - min_gain):
                best, best_ms = trial, ms
    install(tdt, n, n_rhs, best)
    if save:
        save_entry(torch.cuda.get_device_name(dev), tdt, n, n_rhs, best, best_ms, (batch, horizon), path)
    return best, best_ms, trials


_state = threading.local()


def maybe_autotune(dtype, n: int, n_rhs: int, device):
    """Factory hook: install cached entries once; with SOCU_AUTOTUNE=1 tune a
    shape (dtype, n, n_rhs) that has neither a cache entry nor a tuning run in
    this process.  Launches created by a tuning run do not tune again."""
    load_cache(device)
    if os.environ.get("SOCU_AUTOTUNE", "") not in ("1", "true", "yes") or getattr(_state, "busy", False):
        return
    key = (_dtype_name(dtype), int(n), int(n_rhs))
    name = torch.cuda.get_device_name(torch.device(device))
    with _lock:
        if key in _tuned:
            return
        cached = any((e.get("device"), e.get("dtype"), e.get("n"), e.get("n_rhs")) == (name, *key)
                     for e in _read(cache_path())["entries"])
        _tuned.add(key)
    if cached:
        return
    _state.busy = True
    try:
        tune(n, max(int(n_rhs), 1), dtype, device=device)
    finally:
        _state.busy = False
