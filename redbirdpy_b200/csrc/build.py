"""Build the CUDA library ``redbirdpy_b200/librbb200.so`` for sm_100a.

    python redbirdpy_b200/csrc/build.py [--debug]

Every ``*.cu`` file in this directory is compiled by nvcc into an object under
``_build/`` at the repository root (in parallel) and the objects are linked
into one shared library placed next to the package's Python files, where
``redbirdpy_b200/_lib.py`` loads it.  The library exports the C ABI declared
in ``include/redbird_b200.h``.
"""

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(PKG, "librbb200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def compile_one(src, debug):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) > max(
        os.path.getmtime(p) for p in [src] + glob.glob(os.path.join(HERE, "*.cuh")) +
        [os.path.join(ROOT, "include", "redbird_b200.h")]
    ):
        return obj
    flags = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
             "-I", os.path.join(ROOT, "include")]
    if debug:
        flags += ["-DRB_DEBUG"]
    cmd = [nvcc()] + ARCH + flags + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s" % (src, r.stderr))
    return obj


def build(debug=False, verbose=True):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(HERE, "*.cu")))
    with cf.ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: compile_one(s, debug), srcs))
    tmp = LIB + ".tmp"
    cmd = [nvcc()] + ARCH + ["-shared", "-o", tmp] + objs + ["-cudart", "static"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stderr)
    os.replace(tmp, LIB)
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(debug="--debug" in sys.argv)
