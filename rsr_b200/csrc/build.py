"""Builds librsrgpu.so (all CUDA kernels + the C ABI) for sm_100a.

Each translation unit is compiled by its own nvcc process, in parallel, into
rsr_b200/_build/, then linked into rsr_b200/librsrgpu.so.  -fmad=false keeps
every multiply and add separately rounded, as the reference evaluates them.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
PKG = HERE.parent
ROOT = PKG.parent
BUILD = PKG / "_build"
LIB = PKG / "librsrgpu.so"

SOURCES = ["runtime.cu", "kernels_plain.cu", "kernels_reg.cu", "kernels_grad.cu", "kernels_adj.cu", "encoder.cpp",
           "serving.cu", "lbfgs.cu", "nelder_mead.cu", "cma_es.cu", "ingest.cu", "noalloc.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-lineinfo", "-fmad=false",
              "-prec-div=true", "-prec-sqrt=true", "-Xcompiler", "-fPIC,-fvisibility=hidden,-ffp-contract=off",
              "-I", str(ROOT / "include"), "-I", str(HERE)]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, verbose: bool) -> Path:
    out = BUILD / (Path(src).stem + ".o")
    path = HERE / src
    deps = [path] + list(HERE.glob("*.h")) + list(HERE.glob("*.cuh")) + [ROOT / "include" / "rsr_gpu.h"]
    if out.exists() and out.stat().st_mtime > max(d.stat().st_mtime for d in deps):
        return out
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", str(path), "-o", str(out)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return out


def build(verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    srcs = [s for s in SOURCES if (HERE / s).exists()]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if LIB.exists() and LIB.stat().st_mtime > max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", str(tmp)] + [str(o) for o in objs] + \
          ["-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
