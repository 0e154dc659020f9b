"""Build the sm_100a shared library ``ddpcm_b200/lib/libddcosmo_gpu.so``.

The library is compiled in-tree with nvcc for ``compute_100a``/``sm_100a``
(B200).  cudart is linked statically and no other CUDA library is linked:
every kernel, the dense contractions included, is this library's own (the
driver's TMA descriptor encoder is reached through cudart's entry-point
query).
Host code is compiled with ``-ffp-contract=off`` so that the Lebedev grid and
the normalisation tables follow the written operation order.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libddcosmo_gpu.so")
SOURCES = ["ddc_api.cu", "ddc_kernels.cu", "ddc_tc.cu", "ddc_guess.cu", "ddc_noalloc.cu",
           "ddc_zfar.cu"]
HEADERS = ["ddc_internal.h", "lebedev_orbits.inc"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for p in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if p and (os.path.sep not in p or os.path.exists(p)):
            return p
    return "nvcc"


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "ddcosmo_gpu.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force=False, verbose=False):
    """Compile the library if any source is newer than it. Returns its path."""
    if not force and not _stale():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    cmd = [nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-Xptxas", "-warn-spills" if verbose else "-O3",
           "-I", os.path.join(HERE, "..", "include"),
           "-Xlinker", "--no-undefined",  # a missing definition fails the build, not the load
           "-o", LIB + ".tmp", *[os.path.join(CSRC, s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
