"""Build ``socu_b200/lib/libsocu_b200.so`` with nvcc for sm_100a.

    python -m socu_b200.build            # build if sources changed
    python -m socu_b200.build --force    # always rebuild

The CUDA runtime is linked statically so the library does not depend on the
libcudart version a host process (e.g. PyTorch) happens to load.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "lib"
OUT = OUT_DIR / "libsocu_b200.so"
STAMP = OUT_DIR / ".build_stamp"

SOURCES = ["capi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _digest() -> str:
    h = hashlib.sha256()
    for p in sorted(CSRC.glob("*")) + [ROOT / "include" / "socu_b200.h", pathlib.Path(__file__)]:
        if p.is_file():
            h.update(p.name.encode())
            h.update(p.read_bytes())
    return h.hexdigest()


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    digest = _digest()
    if not force and OUT.exists() and STAMP.exists() and STAMP.read_text() == digest:
        return OUT
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
           "-Xcompiler", "-fPIC", "-shared", "-cudart", "static",
           "-I", str(ROOT / "include"),
           "-o", str(OUT) + ".tmp", *[str(CSRC / s) for s in SOURCES]]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building libsocu_b200.so")
    if verbose:
        sys.stderr.write(res.stdout + res.stderr)
    os.replace(str(OUT) + ".tmp", OUT)
    STAMP.write_text(digest)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
