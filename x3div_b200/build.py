"""Build recipe for the in-tree CUDA library (sm_100a) and its checker."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build(jobs: int = 8) -> str:
    """Compile x3div_b200/_lib/libx3d_b200.so with nvcc for sm_100a and return its path."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "csrc")], check=True)
    return os.path.join(HERE, "_lib", "libx3d_b200.so")
