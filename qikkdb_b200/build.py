"""Build recipe of the native libraries (run in-tree; the built .so files sit next to this file).

* ``libqdbgb.so``   - the CUDA GROUP BY path (sm_100a only) behind the C ABI of include/qdb_gb.h.
* ``libqdbgen.so``  - the multithreaded, counter-based synthetic data generators (host C++).

Usage: ``python -m qikkdb_b200.build [--force]``.  Objects are compiled in parallel and only rebuilt when a
source or header is newer than the library.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
]
CUDA_SOURCES = [
    "runtime.cu", "groupby.cu", "results.cu", "exchange.cu", "filter.cu", "reconstruct.cu", "hostpipe.cu",
    "agg_i32.cu", "agg_i64.cu", "agg_f32.cu", "agg_f64.cu", "agg_comp.cu", "fast_i32.cu", "fast_i64.cu", "fast_f32.cu",
    "fast_f64.cu", "fast_comp.cu", "fast_i32_mod.cu", "fast_i64_mod.cu", "batch.cu", "batch_kernels.cu",
    "serve.cu", "orderby.cu", "scalar.cu", "groupby_string.cu", "compression.cu",
]
EXTRA_CUDA_SOURCES: list[str] = []

LIB_NAME = "libqdbgb.so"
GEN_NAME = "libqdbgen.so"


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build qikkdb_b200")


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _newest(paths: list[str]) -> float:
    return max((os.path.getmtime(p) for p in paths if os.path.exists(p)), default=0.0)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("command failed: " + " ".join(cmd) + "\n" + res.stdout + res.stderr)


def _compile(src: str, obj: str, force: bool) -> str:
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(
            os.path.getmtime(src), _newest(_headers())):
        return obj
    _run([nvcc(), *NVCC_FLAGS, "-I", INCLUDE, "-c", src, "-o", obj])
    return obj


def build_cuda(force: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    lib = os.path.join(HERE, LIB_NAME)
    sources = [os.path.join(CSRC, s) for s in CUDA_SOURCES + EXTRA_CUDA_SOURCES]
    objs = [os.path.join(BUILD, os.path.basename(s) + ".o") for s in sources]
    jobs = jobs or max(1, min(len(sources), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(lambda so: _compile(so[0], so[1], force), zip(sources, objs)))
    if force or not os.path.exists(lib) or os.path.getmtime(lib) < _newest(objs):
        _run([nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", lib, *objs,
              "-Xcompiler", "-fPIC", "-cudart", "static"])
    return lib


def build_datagen(force: bool = False) -> str:
    src = os.path.join(CSRC, "datagen.cpp")
    lib = os.path.join(HERE, GEN_NAME)
    if force or not os.path.exists(lib) or os.path.getmtime(lib) < os.path.getmtime(src):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", lib, src])
    return lib


def build_all(force: bool = False) -> None:
    build_datagen(force)
    build_cuda(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", os.path.join(HERE, LIB_NAME), os.path.join(HERE, GEN_NAME))
