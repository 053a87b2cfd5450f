"""Build libwsb.so (the CUDA kernels and the C ABI) in-tree for sm_100a.

    python -m warpsphboundaries_b200.build          # regenerate the kernel tables, compile, link

The library lands in warpsphboundaries_b200/_build/libwsb.so, where `_lib.py` loads it.
"""
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_build"
LIB = OUT_DIR / "libwsb.so"
SOURCES = ["surface.cu", "topology.cu", "fused.cu", "radial.cu", "mesh.cu", "triangle.cu", "disk.cu", "fem.cu",
           "serve.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found (set NVCC or install the CUDA toolkit)")


def generate_tables():
    from . import kernels
    text = kernels.emit_header()
    p = CSRC / "kernel_tables.h"
    if not p.exists() or p.read_text() != text:
        p.write_text(text)


def flags(extra=()):
    return ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", *ARCH, *extra]


def build(verbose=False, force=False, ptxas_verbose=False):
    """compile every source to an object and link libwsb.so; returns the library path."""
    generate_tables()
    OUT_DIR.mkdir(exist_ok=True)
    nvcc = nvcc_path()
    deps = [CSRC / "common.cuh", CSRC / "kernel_tables.h", PKG.parent / "include" / "wsb.h"]
    objs = []
    for src in SOURCES:
        s = CSRC / src
        o = OUT_DIR / (src + ".o")
        objs.append(o)
        newest = max(p.stat().st_mtime for p in deps + [s])
        if force or not o.exists() or o.stat().st_mtime < newest:
            cmd = [nvcc, *flags(["-Xptxas", "-v"] if ptxas_verbose else []), "-c", str(s), "-o", str(o)]
            if verbose:
                print(" ".join(cmd), flush=True)
            r = subprocess.run(cmd, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
            if ptxas_verbose:
                print(r.stderr)
    if force or not LIB.exists() or LIB.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    peak = OUT_DIR / "libwsbpeak.so"
    src = CSRC / "peak.cu"
    if force or not peak.exists() or peak.stat().st_mtime < src.stat().st_mtime:
        cmd = [nvcc, *flags(), "-shared", "-o", str(peak), str(src)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on peak.cu:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_verbose="--ptxas" in sys.argv))
