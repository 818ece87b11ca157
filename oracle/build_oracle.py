"""Build ``oracle/_build/libcubam_oracle.so`` from ``oracle/cpu_decoder.c`` (gcc, zlib, pthreads).

TEST INFRASTRUCTURE ONLY: the oracle for large inputs and the timed CPU baseline.
"""

from __future__ import annotations

import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_build"
LIB = OUT / "libcubam_oracle.so"
SRC = HERE / "cpu_decoder.c"


def build(force: bool = False) -> Path:
    if LIB.exists() and not force and LIB.stat().st_mtime > SRC.stat().st_mtime:
        return LIB
    OUT.mkdir(exist_ok=True)
    tmp = OUT / "libcubam_oracle.tmp.so"
    cmd = ["gcc", "-O3", "-march=x86-64-v2", "-shared", "-fPIC", "-pthread", str(SRC), "-o", str(tmp), "-lz"]
    subprocess.run(cmd, check=True)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
