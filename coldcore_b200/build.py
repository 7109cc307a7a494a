"""Build the engine's shared library (sm_100a) in-tree.

``build()`` compiles every ``csrc/*.cu`` translation unit with nvcc for
``sm_100a`` into ``_build/`` at the repository root and links
``coldcore_b200/libcoldcore_covering.so``.  Object files are rebuilt only
when a source or header is newer.
"""
import concurrent.futures
import glob
import os
import subprocess

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(ROOT, "_build", "obj")
LIB = os.path.join(PKG, "libcoldcore_covering.so")
SPARSE_LIB = os.path.join(PKG, "libcoldcore_sparse.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
         "-Xcompiler", "-fvisibility=hidden", "-I",
         os.path.join(ROOT, "include")]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, headers, extra):
    obj = os.path.join(OBJ, os.path.basename(src).replace(".cu", ".o"))
    if not _newer(obj, [src] + headers):
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode:
        raise RuntimeError(f"nvcc failed on {src}:\n{r.stdout}\n{r.stderr}")
    return obj, r.stderr


def build(verbose=False, extra=()):
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.h")) +
                     glob.glob(os.path.join(ROOT, "include", "*", "*.h")))
    with concurrent.futures.ThreadPoolExecutor(len(srcs)) as ex:
        res = list(ex.map(lambda s: _compile(s, headers, list(extra)), srcs))
    objs = [o for o, _ in res]
    if verbose:
        for _, log in res:
            if log:
                print(log)
    if _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    build_sparse(verbose, extra)
    return LIB


def build_sparse(verbose=False, extra=()):
    """The explicit-incidence engine (plugin ABI 2), its own library as in
    the reference: ``csrc/sparse/*.cu`` -> ``libcoldcore_sparse.so``."""
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "sparse", "*.cu")))
    headers = [os.path.join(ROOT, "include", "coldcore_b200", "sparse.h")]
    res = [_compile(s, headers, list(extra)) for s in srcs]
    objs = [o for o, _ in res]
    if verbose:
        for _, log in res:
            if log:
                print(log)
    if _newer(SPARSE_LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", SPARSE_LIB] + objs
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return SPARSE_LIB


if __name__ == "__main__":
    import sys
    print(build(verbose="-v" in sys.argv))
