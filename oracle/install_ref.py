#!/usr/bin/env python3
"""Install the reference's own Python package and test files beside the
repository (test infrastructure only).

    COLDCORE_REF_SRC=<reference checkout>/src python oracle/install_ref.py

* ``baseline/_ref/coldcore``: the reference package, installed by pip with
  no index and no dependencies from a scratch copy of the checkout (its
  setuptools build writes into the source tree, which may be read-only):
  ``pip install --no-index --no-build-isolation --no-deps --target
  baseline/_ref <copy>``;
* ``baseline/_ref/tests``: the checkout's ``tests/*.py`` and its
  ``conftest.py``, unchanged.

Both are git-ignored and travel with the working tree, so a GPU host
without the checkout can run the reference's binding (``coldcore.gpu``)
and its GPU test files against this engine's library
(``tests/test_gpu_reference_binding.py``).  Nothing in the engine imports
them.
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
TARGET = os.path.join(ROOT, "baseline", "_ref")


def install():
    src = os.environ.get("COLDCORE_REF_SRC")
    if not src or not os.path.isdir(os.path.join(src, "coldcore")):
        raise FileNotFoundError(
            "COLDCORE_REF_SRC must name the reference checkout's src/ "
            "directory")
    checkout = os.path.dirname(os.path.abspath(src))
    with tempfile.TemporaryDirectory() as tmp:
        copy = os.path.join(tmp, "ref")
        shutil.copytree(checkout, copy, ignore=shutil.ignore_patterns(
            ".git", "build", "paper", "__pycache__"))
        if os.path.isdir(TARGET):
            shutil.rmtree(TARGET)
        subprocess.run([sys.executable, "-m", "pip", "install", "--no-index",
                        "--no-build-isolation", "--no-deps", "--quiet",
                        "--target", TARGET, copy], check=True, cwd=tmp)
    tests = os.path.join(TARGET, "tests")
    os.makedirs(tests, exist_ok=True)
    for name in sorted(os.listdir(os.path.join(checkout, "tests"))):
        if name.endswith(".py"):
            shutil.copy2(os.path.join(checkout, "tests", name), tests)
    return TARGET


if __name__ == "__main__":
    print(install())
