"""Builds libstophys_b200.so in-tree (nvcc, sm_100a) with the committed Makefile."""
from __future__ import annotations

import os
import subprocess
from pathlib import Path

CSRC = Path(__file__).resolve().parent / "csrc"


def build(jobs: int = 0, force: bool = False) -> Path:
    if force:
        subprocess.run(["make", "-C", str(CSRC), "clean"], check=True, capture_output=True)
    j = jobs or max(1, min(8, os.cpu_count() or 1))
    subprocess.run(["make", "-C", str(CSRC), f"-j{j}"], check=True)
    return CSRC.parent / "libstophys_b200.so"


if __name__ == "__main__":
    print(build())
