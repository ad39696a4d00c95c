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


OPS_LIB = "libtcr_torch_ops.so"
OPS_SRC = "tcr_torch_ops.cpp"


def build_ops(force=False, verbose=False):
    """Builds the TORCH_LIBRARY operator layer (tcr_torch_ops.cpp, linked to libtcr_b200.so) into
    the package directory; returns its path."""
    dst = os.path.join(HERE, OPS_LIB)
    deps = [os.path.join(CSRC, OPS_SRC), os.path.join(REPO, "include", "tcr_b200.h"), os.path.join(HERE, "libtcr_b200.so")]
    if not force and os.path.exists(dst) and all(os.path.getmtime(d) <= os.path.getmtime(dst) for d in deps[:2]):
        return dst
    import shutil

    bdir = os.path.join(HERE, "_build", "ops")
    os.makedirs(bdir, exist_ok=True)
    env = os.environ.copy()
    # The system g++ links libstdc++ dynamically, the one copy torch uses; a toolchain whose
    # library path holds only the static archive would give this library a second, uninitialised
    # copy of the C++ runtime (its stream and locale state), so the system compiler is used.
    if os.path.exists("/usr/bin/g++"):
        env["CXX"] = "/usr/bin/g++"
    # torch's extension builder loads what it built into the calling process; it runs in a child
    # so that this process registers the operators once, from the package copy (ops.load).
    script = f"""
from torch.utils import cpp_extension
cpp_extension.load(name="tcr_torch_ops", sources=[{os.path.join(CSRC, OPS_SRC)!r}],
                   extra_include_paths=[{os.path.join(REPO, "include")!r}],
                   extra_cflags=["-O2", "-std=c++17"],
                   extra_ldflags=["-L" + {HERE!r}, "-ltcr_b200",
                                  # $$ reaches the linker as one $ through ninja, quotes keep the shell off it
                                  "'-Wl,-rpath,$$ORIGIN'", "'-Wl,-rpath,$$ORIGIN/../..'"],
                   with_cuda=True, is_python_module=False, build_directory={bdir!r}, verbose={bool(verbose)!r})
"""
    subprocess.check_call([sys.executable, "-c", script], env=env)
    shutil.copy2(os.path.join(bdir, "tcr_torch_ops.so"), dst)
    return dst


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
    if "--ops" in sys.argv:
        print(build_ops(force="--force" in sys.argv, verbose=True))
