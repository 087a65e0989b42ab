"""Build libssfft.so in-tree for sm_100a.

    python -m materialite_b200.csrc.build

Compiles ``ssfft.cu`` (which includes the kernel headers of this directory),
``noalloc.cu``, ``server.cu`` and ``voronoi.cu`` with nvcc into ``materialite_b200/libssfft.so``.
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3",
              "-std=c++17", "-shared", "-Xcompiler", "-fPIC,-O2"]


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.isfile(cand) else "nvcc"


def sources():
    return sorted(os.path.join(HERE, f) for f in os.listdir(HERE)
                  if f.endswith((".cu", ".cuh")))


def build(force=False, verbose=False):
    out = os.path.join(PKG, "libssfft.so")
    srcs = sources() + [os.path.join(os.path.dirname(PKG), "include", "ssfft.h")]
    if (not force and os.path.isfile(out)
            and os.path.getmtime(out) >= max(os.path.getmtime(s) for s in srcs)):
        return out
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", out] + [os.path.join(HERE, f) for f in
                                                 ("ssfft.cu", "noalloc.cu", "server.cu", "voronoi.cu")]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
