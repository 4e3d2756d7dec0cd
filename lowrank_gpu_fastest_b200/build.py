"""Build recipe for the native library ``liblrd.so`` (sm_100a only).

``nvcc -gencode arch=compute_100a,code=sm_100a`` cross-compiles without a GPU,
so the library is built in-tree here and travels with the package. The CUDA
runtime is linked statically; the library shares the device's primary context
with PyTorch, so device pointers and streams pass between them unchanged.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "liblrd.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O2",
         "--expt-relaxed-constexpr", "-Xptxas", "-O3"]


def sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))
            if f.endswith((".cu", ".cuh", ".h"))] + [os.path.join(INCLUDE, "lrd.h")]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(s) > t for s in sources())


def build(force: bool = False, verbose: bool = False, extra: list | None = None) -> str:
    """Compile ``csrc/lrd_api.cu`` (which includes the kernel headers) into
    ``liblrd.so`` next to this file; a no-op when it is newer than every source."""
    if not force and not needs_build():
        return LIB
    cmd = [NVCC, *ARCH_FLAGS, *FLAGS, *(extra or []), "-I", INCLUDE,
           os.path.join(CSRC, "lrd_api.cu"), "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else None)
