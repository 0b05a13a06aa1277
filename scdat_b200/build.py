"""Build libscdat_b200.so in-tree with nvcc for sm_100a.

    python -m scdat_b200.build          # incremental
    python -m scdat_b200.build --force  # rebuild everything

Objects go to scdat_b200/_build/, the library to scdat_b200/libscdat_b200.so, and the C++20
host layer over it (scdat_b200/host/) to scdat_b200/libscdat_host.so.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libscdat_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CXX = os.environ.get("CXX", "g++")
HOST_DIR = os.path.join(HERE, "host")
HOST_LIB = os.path.join(HERE, "libscdat_host.so")

SOURCES = ["capi.cu", "push_f64.cu", "push_mixed.cu", "field.cu", "utils.cu", "pcg_csr.cu", "pcg_noalloc.cu",
           "batch_field.cu", "batch_host.cu", "surface.cu", "adjoint.cu", "mg.cu", "mesh_setup.cpp",
           "mg_setup.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", f"-I{os.path.join(ROOT, 'include')}"]


# The precision form's push runs a particle's sub-steps in whichever of its pass kernels reaches
# them (the pass split depends on the pass-1 form and the list capacities), and its results are
# bitwise independent of that split only if every kernel evaluates the same IEEE operations:
# so no multiply-add contraction in that file (explicit fmaf calls are kept).
PER_FILE_FLAGS = {"push_mixed.cu": ["--fmad=false"]}


def _headers_mtime() -> float:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(os.path.join(ROOT, "include", "scdat_b200.h"))
    return max(os.path.getmtime(h) for h in hs)


def _compile(src: str, force: bool, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, src + ".o")
    srcp = os.path.join(CSRC, src)
    if not force and os.path.exists(obj):
        if os.path.getmtime(obj) >= max(os.path.getmtime(srcp), _headers_mtime()):
            return obj
    cmd = [NVCC, *ARCH, *FLAGS, *PER_FILE_FLAGS.get(src, []), "-c", srcp, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC, "-x", "c++", *FLAGS, "-c", srcp, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, len(SOURCES))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose_ptxas), SOURCES))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-Xcompiler", "-fPIC"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_host(force)
    return LIB


def build_host(force: bool = False) -> str:
    """The C++20 host layer: g++ over scdat_b200/host/*.cpp, linked to the C-ABI library."""
    srcs = [os.path.join(HOST_DIR, f) for f in sorted(os.listdir(HOST_DIR)) if f.endswith(".cpp")]
    deps = srcs + [os.path.join(HOST_DIR, f) for f in os.listdir(HOST_DIR) if f.endswith(".hpp")]
    deps += [LIB, os.path.join(ROOT, "include", "scdat_b200.h")]
    if not force and os.path.exists(HOST_LIB) and os.path.getmtime(HOST_LIB) >= max(os.path.getmtime(d) for d in deps):
        return HOST_LIB
    cmd = [CXX, "-std=c++20", "-O2", "-fPIC", "-shared", "-Wall", "-Wextra", *srcs, f"-I{os.path.join(ROOT, 'include')}",
           f"-I{HOST_DIR}", f"-L{HERE}", "-lscdat_b200", "-Wl,-rpath,$ORIGIN", "-o", HOST_LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"host layer build failed:\n{r.stdout}\n{r.stderr}")
    return HOST_LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv))
