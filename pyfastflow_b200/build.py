"""Build libpff.so in-tree (nvcc, sm_100a)."""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))


def build(jobs: int = 8, extra: str = "") -> str:
    cmd = ["make", "-s", f"-j{jobs}", "-C", os.path.join(HERE, "csrc")]
    if extra:
        cmd.append(f"EXTRA={extra}")
    subprocess.run(cmd, check=True)
    return os.path.join(HERE, "libpff.so")


if __name__ == "__main__":
    print(build())
