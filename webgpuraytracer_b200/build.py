"""Builds the native library libwgpt.so (CUDA kernels for sm_100a + C ABI + host builders).

The kernels are compiled without contraction of multiply-adds (-fmad=false) and with IEEE
division and square root, so that their arithmetic is reproducible bit for bit on the CPU.
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
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libwgpt.so"
CU_SOURCES = ["tracer.cu", "wavefront.cu", "denoise.cu", "api.cu", "kpcn.cu", "probe.cu"]
CXX_SOURCES = ["builders.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr",
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-Wall"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    if r.stderr.strip() and os.environ.get("WGPT_BUILD_VERBOSE"):
        sys.stderr.write(r.stderr)


def _stale(target: Path, deps: list[Path]) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def build(force: bool = False, ptxas_verbose: bool = False) -> Path:
    """Compiles every source that changed and links libwgpt.so; returns its path."""
    OUT_DIR.mkdir(exist_ok=True)
    headers = list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list((PKG.parent / "include").glob("*.h"))
    nvcc = _nvcc()
    objs: list[Path] = []
    jobs = []
    for src in CU_SOURCES:
        s = CSRC / src
        o = OUT_DIR / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            flags = NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else [])
            jobs.append([nvcc] + flags + ["-c", str(s), "-o", str(o)])
    for src in CXX_SOURCES:
        s = CSRC / src
        o = OUT_DIR / (src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", str(s), "-o", str(o)])
    with ThreadPoolExecutor(max_workers=4) as ex:
        list(ex.map(_run, jobs))
    if force or jobs or _stale(LIB, objs):
        _run([nvcc] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + ["-lcudart"])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv))
