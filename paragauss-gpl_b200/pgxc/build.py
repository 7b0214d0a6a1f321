"""Compile libpgxc.so for sm_100a (B200) in-tree with nvcc."""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libpgxc.so")
SOURCES = ["pgxc_api.cu", "kernels_fp64.cu", "kernels_aux.cu", "mixed.cu", "noalloc.cu", "screened.cu",
           "screened_mixed.cu", "symmetry.cu", "gradient.cu", "grid.cu", "mgga.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC"]
OBJDIR = os.path.join(PKG, "_build")


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    for d in (CSRC, os.path.join(os.path.dirname(PKG), "include")):
        for f in os.listdir(d):
            if os.path.getmtime(os.path.join(d, f)) > t:
                return True
    return False


def build(force=False, verbose=False):
    """Compile every source to an object (in parallel), then link the library."""
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    cc = nvcc()

    def compile_one(src):
        obj = os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")
        cmd = [cc] + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True, cwd=CSRC)
        return obj

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    cmd = [cc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared"] + objs + ["-o", LIB]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
