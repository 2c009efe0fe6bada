"""Build recipe of liblomacte_b200.so (sm_100a) in-tree.

nvcc compiles the CUDA kernels for sm_100a only and the host C++ with
OpenMP; the shared library lands next to this file so it travels with the
source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "liblomacte_b200.so")
SOURCES = ["lmc_y_d.cu", "lmc_y_c.cu", "lmc_y_b.cu", "lmc_y_a.cu", "lmc_ytpm.cu", "lmc_fft_c.cu", "lmc_fft_b.cu",
           "lmc_fft_a.cu", "lmc_api.cu", "lmc_dispatch.cu", "lmc_ykernels.cu", "lmc_noalloc.cu", "lmc_yop.cu", "lmc_host.cpp"]
HEADERS = ["lmc_internal.h", "lmc_kernels.cuh", "lmc_device.cuh", "lmc_fft_impl.cuh", "lmc_async.cuh",
           "lmc_ykernels.cuh", "lmc_ylaunch.h", "lmc_ytpm.cuh", "lmc_stats.cuh"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "lomacte_b200.h"))
    return any(os.path.getmtime(p) > t for p in deps)


FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-gencode", "arch=compute_100a,code=sm_100a",
         "-Xcompiler", "-fPIC,-fopenmp"]


def _compile(src: str, obj: str, verbose: bool) -> str:
    cmd = [nvcc(), "-ccbin", host_cxx()] + FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}{r.stderr}")
    return r.stderr


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object in parallel, then link the shared
    library (sm_100a device code only)."""
    if not force and not _stale():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    odir = os.path.join(HERE, "_build")
    os.makedirs(odir, exist_ok=True)
    objs = [os.path.join(odir, os.path.splitext(f)[0] + ".o") for f in SOURCES]
    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        logs = list(ex.map(lambda a: _compile(a[0], a[1], verbose), zip(SOURCES, objs)))
    if verbose:
        for f, l in zip(SOURCES, logs):
            sys.stderr.write(f"==== {f}\n{l}")
    cmd = [nvcc(), "-ccbin", host_cxx(), "-shared", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-fopenmp", "-o", LIB + ".tmp"] + objs + ["-lcublas", "-lgomp"]
    r = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc link of liblomacte_b200 failed")
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
