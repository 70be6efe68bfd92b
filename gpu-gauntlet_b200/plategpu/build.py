"""In-tree build of libplategpu.so (nvcc cross-compiles sm_100a without a GPU)."""
from __future__ import annotations

import os
import subprocess

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "csrc")


def build_library(verbose: bool = False) -> str:
    """Runs the csrc Makefile; returns the path of the shared library."""
    subprocess.run(["make", "-C", CSRC] + ([] if verbose else ["-s"]), check=True)
    from . import _lib
    return _lib.LIB_PATH
