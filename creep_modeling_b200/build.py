"""Builds the sm_100a shared library ``_build/libevp_b200.so`` with nvcc.

The library is compiled in-tree (no JIT cache) so that it travels with the
repository to the GPU machine.  Objects are rebuilt only when a source or
header is newer than the object.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT = PKG / "_build"
LIB = OUT / "libevp_b200.so"
INCLUDE = PKG.parent / "include"

SOURCES = ["evp_solver.cu", "evp_engine.cu", "evp_control.cu", "evp_kernels.cu", "evp_fft.cu", "evp_green.cu",
           "evp_deck.cpp", "evp_server.cpp"]
# per-file extra flags: the device-side iteration tail keeps plain multiply-then-add rounding
EXTRA_FLAGS = {"evp_control.cu": ["-fmad=false"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3", f"-I{INCLUDE}"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libevp_b200.so")


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [INCLUDE / "evp.h"]


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *_deps()])


def build(force: bool = False, verbose: bool = False) -> Path:
    OUT.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    env = dict(os.environ)
    jobs = []
    objs = []
    for name in SOURCES:
        src = CSRC / name
        obj = OUT / (name + ".o")
        objs.append(obj)
        if force or _stale(obj, src):
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, *EXTRA_FLAGS.get(name, []), "-c", str(src), "-o", str(obj)]
            if name.endswith(".cpp"):
                cmd = [nvcc, "-x", "cu", *ARCH, *NVCC_FLAGS, "-c", str(src), "-o", str(obj)]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        return r

    with ThreadPoolExecutor(max_workers=max(1, len(jobs))) as ex:
        list(ex.map(run, jobs))
    if jobs or not LIB.exists():
        link = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        run(link)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
