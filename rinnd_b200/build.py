"""Build recipe for librinnd_b200.so (sm_100a) -- nvcc via rinnd_b200/csrc/Makefile."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build(jobs: int = 8) -> str:
    """Compile every CUDA source for sm_100a into rinnd_b200/librinnd_b200.so."""
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", CSRC], check=True)
    return os.path.join(HERE, "librinnd_b200.so")


if __name__ == "__main__":
    print(build())
