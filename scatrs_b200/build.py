"""Builds libscatrs_b200.so for sm_100a in this directory (nvcc cross-compiles without a GPU)."""

from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libscatrs_b200.so")


def build(verbose: bool = False) -> str:
    """Runs the Makefile of csrc/ (a no-op when the library is up to date)."""
    r = subprocess.run(["make", "-C", os.path.join(HERE, "csrc")], capture_output=True, text=True)
    if verbose or r.returncode != 0:
        print(r.stdout[-4000:], r.stderr[-4000:])
    r.check_returncode()
    return LIB


if __name__ == "__main__":
    build(verbose=True)
