"""Build libqfb.so (the sm_100a CUDA engine) in-tree with nvcc.

    python -m qforte_b200.build            # build if sources are newer
    python -m qforte_b200.build --force    # rebuild
    python -m qforte_b200.build --verbose-ptxas   # also print registers / spills

The library is a plain C-ABI shared object (include/qfb.h); the Python package
loads it with ctypes.  It is compiled for sm_100a only.
"""

import argparse
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libqfb.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libqfb.so")
    return cand


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(ROOT, "include", "qfb.h")]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose_ptxas=False, quiet=False):
    if not force and not needs_build():
        return LIB
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared",
           "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
           "-Xcompiler", "-O2", "-I", os.path.join(ROOT, "include"),
           "-o", LIB + ".tmp", *sources()]
    if verbose_ptxas:
        cmd[1:1] = ["-Xptxas", "-v"]
    if not quiet:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    build(force=a.force or a.verbose_ptxas, verbose_ptxas=a.verbose_ptxas)


if __name__ == "__main__":
    main()
