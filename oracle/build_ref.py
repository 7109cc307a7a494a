#!/usr/bin/env python3
"""Build the reference's own plugins for sm_100a (test and comparison
infrastructure only).

The reference's ABI-v1 plugin is one CUDA translation unit,
``src/plugins/covering/dct_hc.cu`` (with the ``dctcore_*.cuh`` headers
beside it).  This recipe compiles it where it lies, with nvcc directly (not
the reference's CMake build), into ``oracle/_ref/libref_covering.so``:

    python oracle/build_ref.py            # ~3 minutes

The library exports the same ``dct_*`` symbols as this engine, so the GPU
tests can pin the engine's fields against the reference's own kernels on
the same B200, and ``bench.py`` can time the reference's kernels on the
cells they accept (axes <= 16, n <= 16, <= 65,535 occurrences).

Likewise the ABI-2 plugin, ``src/plugins/sparse/sparse.cu`` (one file),
becomes ``oracle/_ref/libref_sparse.so`` (``build_sparse``), the
reference side of the explicit-incidence comparison.  Nothing here is
linked into the engine; the reference source stays outside the
repository, and the built libraries are git-ignored.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_ref")
OUT = os.path.join(OUT_DIR, "libref_covering.so")
SPARSE_OUT = os.path.join(OUT_DIR, "libref_sparse.so")


def ref_src():
    """The reference checkout's ``src/`` directory: ``COLDCORE_REF_SRC``.
    Unset means no source here; a prebuilt library is then used as is."""
    path = os.environ.get("COLDCORE_REF_SRC")
    if not path:
        raise FileNotFoundError(
            "COLDCORE_REF_SRC is unset: point it at the reference "
            "checkout's src/ directory to build the reference plugins")
    return path


def build(force=False):
    try:
        src = os.path.join(ref_src(), "plugins", "covering", "dct_hc.cu")
    except FileNotFoundError:
        if os.path.exists(OUT):
            return OUT
        raise
    if not os.path.exists(src):
        if os.path.exists(OUT):
            return OUT                    # prebuilt; no source here
        raise FileNotFoundError(src)
    if os.path.exists(OUT) and not force and \
            os.path.getmtime(OUT) >= os.path.getmtime(src):
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["nvcc", "-O3", "-std=c++17",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-shared", "-Xcompiler", "-fPIC",
           "-I", os.path.join(ref_src(), "include"),
           src, "-o", OUT + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


def build_sparse(force=False):
    try:
        src = os.path.join(ref_src(), "plugins", "sparse", "sparse.cu")
    except FileNotFoundError:
        if os.path.exists(SPARSE_OUT):
            return SPARSE_OUT
        raise
    if not os.path.exists(src):
        if os.path.exists(SPARSE_OUT):
            return SPARSE_OUT
        raise FileNotFoundError(src)
    if os.path.exists(SPARSE_OUT) and not force and \
            os.path.getmtime(SPARSE_OUT) >= os.path.getmtime(src):
        return SPARSE_OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["nvcc", "-O3", "-std=c++17",
           "-gencode", "arch=compute_100a,code=sm_100a",
           "-shared", "-Xcompiler", "-fPIC", src, "-o", SPARSE_OUT + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(SPARSE_OUT + ".tmp", SPARSE_OUT)
    return SPARSE_OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
    print(build_sparse(force="--force" in sys.argv))
