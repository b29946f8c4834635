"""Build recipe of the native library ``libufem_b200.so`` (sm_100a only).

``python -m coolfluid3_b200.build`` compiles every CUDA source under ``csrc/``
with nvcc for ``sm_100a`` and links the shared library in-tree, next to this
file, so that it travels with the package.  Object files go to ``_build/``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libufem_b200.so")
SOURCES = ["assembly.cu", "krylov.cu", "host.cu", "batch.cu", "restart.cu", "bcfunction.cu", "pipeline.cu",
           "semi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-O3",
              "-Xcompiler", "-Wall,-Wno-unused-function"]


def nvcc() -> str:
    path = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(path):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libufem_b200.so")
    return path


def _compile(src: str, ptxas_verbose: bool) -> tuple[str, str]:
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc(), *ARCH, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", obj]
    if ptxas_verbose:
        cmd += ["-Xptxas", "-v"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{proc.stdout}\n{proc.stderr}")
    return obj, proc.stdout + proc.stderr


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [
        os.path.join(HERE, "..", "include", "ufem_b200.h"), __file__]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, ptxas_verbose: bool = False, quiet: bool = False) -> str:
    """Compile and link the library; return its path."""
    if not force and not needs_build():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        results = list(ex.map(lambda s: _compile(s, ptxas_verbose), SOURCES))
    if ptxas_verbose and not quiet:
        for _, log in results:
            sys.stdout.write(log)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"link failed:\n{proc.stdout}\n{proc.stderr}")
    os.replace(tmp, LIB)
    if not quiet:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, ptxas_verbose="-v" in sys.argv)
