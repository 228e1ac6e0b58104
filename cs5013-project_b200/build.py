"""Builds libvann.so (CUDA kernels + C ABI) in-tree for sm_100a.

    python cs5013-project_b200/build.py [--verbose]

Each .cu under csrc/ is compiled to an object in parallel, then linked into
cs5013-project_b200/vann/libvann.so with the CUDA runtime linked statically.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "vann", "libvann.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-ccbin", "g++",
         "--expt-relaxed-constexpr", "-Wno-deprecated-gpu-targets"]
SOURCES = ["search.cu", "search_f32.cu", "search_bf16.cu", "search_fp8.cu", "search_u8.cu", "search_pq.cu", "pq.cu",
           "prune.cu",
           "prune_tc.cu", "prune_rev.cu", "staged.cu", "formats.cu", "graph_ops.cu", "index.cu", "server.cu",
           "rerank.cu"]
HEADERS = ["common.cuh", "kernels.h", "search_impl.cuh", "search_reg.cuh", "search_dispatch.cuh"]


def _stale(obj: str, src: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    deps = [src] + [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(HERE, "..", "include", "vann.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, verbose: bool) -> str:
    s = os.path.join(CSRC, src)
    o = os.path.join(OBJ, src.replace(".cu", ".o"))
    if not _stale(o, s):
        return o
    cmd = [NVCC, *ARCH, *FLAGS, "-c", s, "-o", o]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose:
        sys.stderr.write(r.stderr)
    return o


def build(verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-Xcompiler", "-fPIC", "-ccbin", "g++", "-o", OUT, *objs,
               "-cudart", "static"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv))
