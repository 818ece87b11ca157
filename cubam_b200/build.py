"""Build the native library ``cubam_b200/_lib/libcubam_b200.so`` with nvcc for sm_100a.

``python cubam_b200/build.py`` (or :func:`build`) compiles every ``.cu`` file of
``cubam_b200/csrc`` into one shared library in the source tree; a stamp of the
sources' hash skips the build when nothing changed.
"""

from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
OUT_DIR = PKG / "_lib"
LIB = OUT_DIR / "libcubam_b200.so"
HEADER = PKG.parent / "include" / "cubam_b200.h"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared"]


SYNTH_SRC = CSRC / "host" / "synth.c"
SYNTH_LIB = OUT_DIR / "libcubam_synth.so"


def build_synth(force: bool = False) -> Path:
    """The host library of the synthetic BAM generator (gcc, zlib, pthreads)."""
    if not force and SYNTH_LIB.exists() and SYNTH_LIB.stat().st_mtime > SYNTH_SRC.stat().st_mtime:
        return SYNTH_LIB
    OUT_DIR.mkdir(exist_ok=True)
    tmp = OUT_DIR / f".libcubam_synth.{os.getpid()}.so"
    cmd = ["gcc", "-O3", "-shared", "-fPIC", "-pthread", str(SYNTH_SRC), "-o", str(tmp), "-lz", "-lm"]
    subprocess.run(cmd, check=True)
    tmp.replace(SYNTH_LIB)
    return SYNTH_LIB


SYNTH_MAIN = CSRC / "host" / "synth_main.c"
SYNTH_EXE = OUT_DIR / "cubam_synth"


def build_synth_exe(force: bool = False) -> Path:
    """The generator as an executable (``synth_main.c``): a process of its own writes the file."""
    newest = max(SYNTH_SRC.stat().st_mtime, SYNTH_MAIN.stat().st_mtime)
    if not force and SYNTH_EXE.exists() and SYNTH_EXE.stat().st_mtime > newest:
        return SYNTH_EXE
    OUT_DIR.mkdir(exist_ok=True)
    tmp = OUT_DIR / f".cubam_synth.{os.getpid()}"
    cmd = ["gcc", "-O3", "-pthread", str(SYNTH_SRC), str(SYNTH_MAIN), "-o", str(tmp), "-lz", "-lm"]
    subprocess.run(cmd, check=True)
    tmp.replace(SYNTH_EXE)
    return SYNTH_EXE


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + [HEADER]


def _digest() -> str:
    h = hashlib.sha256()
    for p in _sources():
        h.update(p.name.encode())
        h.update(p.read_bytes())
    h.update(" ".join(ARCH + FLAGS).encode())
    return h.hexdigest()


def nvcc() -> str:
    found = shutil.which("nvcc")
    if found:
        return found
    cand = Path(os.environ.get("CUDA_HOME", "/usr/local/cuda")) / "bin" / "nvcc"
    if cand.exists():
        return str(cand)
    raise RuntimeError("nvcc not found: the cubam_b200 native library cannot be built")


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library unless it is up to date; returns its path."""
    stamp = OUT_DIR / "libcubam_b200.sha256"
    digest = _digest()
    if not force and LIB.exists() and stamp.exists() and stamp.read_text().strip() == digest:
        return LIB
    OUT_DIR.mkdir(exist_ok=True)
    tmp = OUT_DIR / f".libcubam_b200.{os.getpid()}.so"
    cmd = [nvcc(), *ARCH, *FLAGS, *map(str, sorted(CSRC.glob("*.cu"))), "-o", str(tmp)]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=CSRC)
    tmp.replace(LIB)
    stamp.write_text(digest)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
    print(build_synth(force="--force" in sys.argv))
    print(build_synth_exe(force="--force" in sys.argv))
