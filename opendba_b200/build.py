"""Builds the native library in-tree (sm_100a only)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")


def build_library(verbose_ptxas: bool = False) -> str:
    cmd = ["make", "-s", "-C", CSRC, "-j8"]
    if verbose_ptxas:
        cmd.append("VERBOSE_PTXAS=1")
    subprocess.run(cmd, check=True)
    return os.path.join(HERE, "libopendba_b200.so")


if __name__ == "__main__":
    print(build_library())
