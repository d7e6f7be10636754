"""Builds libctc_b200.so in-tree for sm_100a (nvcc cross-compiles; no GPU needed)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libctc_b200.so")

# kernels.cu compiles clist.cu, dpd.cu, fsi.cu, integrate.cu and membrane.cu
# as one translation unit, with the persistent batched step built from their
# kernel bodies
SOURCES = ["api.cu", "api_adjoint.cu", "api_batch.cu", "api_objects.cu", "kernels.cu", "clist_noalloc.cu", "cnt.cu",
           "io_ply.cu", "io_bop.cu", "wall.cu", "api_wall.cu", "exch.cu", "membrane_vjp.cu"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    # the reference builds with -use_fast_math (src/make/main.mk:26); the same
    # flag gives the same rsqrtf/powf and flush-to-zero behaviour
    "-use_fast_math",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc():
    for c in ("/usr/local/cuda/bin/nvcc", "nvcc"):
        if os.path.sep not in c or os.path.exists(c):
            return c
    return "nvcc"


def build(verbose=False):
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "ctc_b200.h"))
    if os.path.exists(LIB) and all(os.path.getmtime(d) <= os.path.getmtime(LIB) for d in deps):
        return LIB
    cmd = [nvcc()] + NVCC_FLAGS + ["-o", LIB] + srcs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
