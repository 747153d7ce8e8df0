"""Builds the in-tree CUDA library (sm_100a) and the CPU oracle used by the tests."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def build(jobs: int = 8, oracle: bool = True) -> str:
    subprocess.run(["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "csrc")], check=True)
    if oracle:
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    return os.path.join(HERE, "_build", "libspaqr_b200.so")


if __name__ == "__main__":
    print(build())
