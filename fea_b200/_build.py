"""Build the fea_b200 native library in-tree with nvcc (sm_100a only).

    python fea_b200/_build.py [--verbose]

(run by path: ``python -m`` would import the package first, and the
package raises ImportError while the library is missing)

Produces ``fea_b200/libfea_b200.so`` (static CUDA runtime, no torch
dependency).  Objects go to ``fea_b200/_build/``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libfea_b200.so")

CU_SOURCES = ["capi.cu", "assemble.cu", "pcg.cu", "explicit.cu", "adjoint.cu"]
CPP_SOURCES = ["plan.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _compile(src, verbose):
    out = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    path = os.path.join(CSRC, src)
    flags = ["-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I", os.path.join(ROOT, "include")]
    if src.endswith(".cu"):
        cmd = [nvcc(), "-c", path, "-o", out, "-lineinfo", "--expt-relaxed-constexpr"] + ARCH + flags
        if verbose:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd = [nvcc(), "-c", "-x", "c++", path, "-o", out] + flags + ["-Xcompiler", "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    return out, r.stderr


def build(verbose=False, force=False):
    srcs = CU_SOURCES + CPP_SOURCES
    deps = [os.path.join(CSRC, s) for s in srcs] + [os.path.join(CSRC, "common.cuh"),
                                                   os.path.join(ROOT, "include", "fea_b200.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in deps):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        results = list(ex.map(lambda s: _compile(s, verbose), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for _, log in results:
            sys.stderr.write(log)
    tmp = LIB + ".tmp"
    cmd = [nvcc(), "-shared", "-o", tmp] + objs + ARCH + ["-Xcompiler", "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed: %s\n%s" % (r.stdout, r.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="--verbose" in sys.argv, force=True))
