"""Build the CUDA library in-tree (sm_100a only).

    python fast-atari-rs_b200/build.py        # incremental
    python fast-atari-rs_b200/build.py --force

Produces fast-atari-rs_b200/lib/libfast_atari.so from csrc/*.cu with nvcc.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libfast_atari.so"
SOURCES = ["fa_kernels.cu", "fa_api.cu", "fa_pool.cu", "fa_noalloc.cu", "fa_autotune.cu", "fa_env.cu", "fa_serve.cu",
           "fa_serve_kernel.cu", "fa_render.cu"]
# The serving kernel reads state rows that a concurrently running launch may
# have written: its global loads are cached in L2 only (the coherence point).
EXTRA = {"fa_serve_kernel.cu": ["-Xptxas", "-dlcm=cg"]}
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-I", str(ROOT / "include")]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.h")) + sorted(CSRC.glob("*.cuh")) + \
        [ROOT / "include" / "fast_atari.h"]


def build(force: bool = False, verbose: bool = False) -> Path:
    newest = max(p.stat().st_mtime for p in _deps())
    if LIB.exists() and not force and LIB.stat().st_mtime >= newest:
        return LIB
    OBJ.mkdir(parents=True, exist_ok=True)
    LIB.parent.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()

    def compile_one(src: str) -> Path:
        out = OBJ / (Path(src).stem + ".o")
        cmd = [nvcc, *ARCH, *FLAGS, *EXTRA.get(src, []), "-c", str(CSRC / src), "-o", str(out)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose:
            sys.stderr.write(r.stderr)
        return out

    with ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart_static", "-lpthread", "-ldl", "-lrt"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
