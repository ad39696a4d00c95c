"""Compiles the CUDA library in-tree for sm_100a (``python -m torchcompactradius_b200.build``)."""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
REPO = os.path.dirname(HERE)
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
              "-shared", "-static-global-template-stub=true", "-I" + os.path.join(REPO, "include")]

LIBS = {
    "libtcr_b200.so": ["tcr_search.cu", "tcr_scatter.cu"],
}


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def build(force=False, verbose=False):
    """Builds every library whose sources are newer than the .so; returns the paths."""
    out = []
    for lib, srcs in LIBS.items():
        dst = os.path.join(HERE, lib)
        deps = [os.path.join(CSRC, s) for s in srcs] + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                                                         if f.endswith(".cuh")]
        deps.append(os.path.join(REPO, "include", "tcr_b200.h"))
        if force or not os.path.exists(dst) or any(os.path.getmtime(d) > os.path.getmtime(dst) for d in deps):
            cmd = [_nvcc()] + NVCC_FLAGS + ["-o", dst] + [os.path.join(CSRC, s) for s in srcs]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
        out.append(dst)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
