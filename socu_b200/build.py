"""Build ``socu_b200/lib/libsocu_b200.so`` with nvcc for sm_100a.

    python -m socu_b200.build            # build if sources changed
    python -m socu_b200.build --force    # always rebuild

The CUDA runtime is linked statically so the library does not depend on the
libcudart version a host process (e.g. PyTorch) happens to load.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import hashlib
import os
import pathlib
import shutil
import subprocess
import sys
import tempfile

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "lib"
OUT = OUT_DIR / "libsocu_b200.so"
STAMP = OUT_DIR / ".build_stamp"

SOURCES = ["capi.cu", "peak.cu", "tc_selftest.cu"]
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


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd))
    res = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
    return res.returncode


def build(force: bool = False, verbose: bool = False) -> pathlib.Path:
    digest = _digest()
    if not force and OUT.exists() and STAMP.exists() and STAMP.read_text() == digest:
        return OUT
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    nvcc = nvcc_path()
    flags = [*ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
             "-I", str(ROOT / "include")]
    if verbose:
        flags.insert(0, "-Xptxas=-v")
    with tempfile.TemporaryDirectory(prefix="socu_build_") as tmp:
        objs = [os.path.join(tmp, pathlib.Path(src).stem + ".o") for src in SOURCES]
        # translation units compile in parallel, then one link step
        with concurrent.futures.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
            codes = list(ex.map(lambda so: _run([nvcc, *flags, "-c", "-o", so[1], str(CSRC / so[0])], verbose),
                                zip(SOURCES, objs)))
        if any(codes):
            raise RuntimeError("nvcc failed building libsocu_b200.so")
        if _run([nvcc, *ARCH, "-shared", "-cudart", "static", "-o", str(OUT) + ".tmp", *objs], verbose):
            raise RuntimeError("nvcc failed linking libsocu_b200.so")
    os.replace(str(OUT) + ".tmp", OUT)
    STAMP.write_text(digest)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))
