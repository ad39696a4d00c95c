"""Build recipe for the reference's own C++ CPU operators (test infrastructure only).

Compiles the torchCompactRadius CPU sources where they lie (``src/torchCompactRadius/cppSrc``
of the reference checkout named by ``--reference`` or ``TCR_REFERENCE``) with ``torch.utils.cpp_extension.load``
into ``oracle/_ref/``.  The reference's own build system (``setup.py``/``dsl.py``) is not used:
the sources compile as they are, with the flags its ``setup.py:127-139`` gives the host compiler
(``-O2 -fopenmp``).  Nothing is copied out of the reference tree; only the compiled ``.so``
lands in ``oracle/_ref/`` (git-ignored, but it travels with the repository snapshot).

The resulting library registers ``torch.ops.torchCompactRadius_cpu.{countNeighbors,
buildNeighborList, computeHashIndices, ...}`` (reference ``cppSrc/cppWrapper.cpp:38-59``).
It is loaded only by the tests, by ``__graft_entry__.smoke`` and by ``bench.py``'s reference /
CPU-baseline arms, as the checker; the product path never touches it.

Usage: ``python oracle/build_ref.py --reference <checkout>`` (or ``TCR_REFERENCE=<checkout>``)
"""
import argparse
import glob
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB_NAME = "torchCompactRadius_cpu"


def ref_library_path():
    """Path of the built reference operator library, or None when it has not been built."""
    cands = sorted(glob.glob(os.path.join(OUT, LIB_NAME + "*.so")))
    return cands[0] if cands else None


def build(reference_root, verbose=False):
    src = os.path.join(reference_root, "src", "torchCompactRadius", "cppSrc")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference sources not found at {src}")
    os.makedirs(OUT, exist_ok=True)
    build_dir = os.path.join(OUT, "build")
    os.makedirs(build_dir, exist_ok=True)
    # /opt's gcc lacks libgomp.spec; the system g++ links OpenMP fine.
    if os.path.exists("/usr/bin/g++"):
        os.environ["CXX"] = "/usr/bin/g++"
        os.environ["CC"] = "/usr/bin/gcc"
    os.environ.setdefault("MAX_JOBS", str(os.cpu_count() or 4))
    from torch.utils import cpp_extension

    sources = sorted(glob.glob(os.path.join(src, "*.cpp")) + glob.glob(os.path.join(src, "*", "*.cpp")))
    cpp_extension.load(
        name=LIB_NAME,
        sources=sources,
        extra_include_paths=[src],
        extra_cflags=["-O2", "-fopenmp", "-Wno-sign-compare", "-Wno-unused-variable", "-w"],
        extra_ldflags=["-fopenmp"],
        build_directory=build_dir,
        is_python_module=False,
        verbose=verbose,
    )
    built = os.path.join(build_dir, LIB_NAME + ".so")
    dst = os.path.join(OUT, LIB_NAME + ".so")
    shutil.copy2(built, dst)
    return dst


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("TCR_REFERENCE"),
                    help="reference checkout (default: the TCR_REFERENCE environment variable)")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give --reference or set TCR_REFERENCE")
    print(build(a.reference, a.v))
