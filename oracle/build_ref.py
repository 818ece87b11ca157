"""Build ``oracle/_ref/libref_kernels.so``: the reference's reader kernels compiled for the CPU.

TEST INFRASTRUCTURE ONLY.  Reads ``src/cubam/_kernels.py`` of the reference
checkout (``$CUBAM_REFERENCE``, else a directory ``reference`` beside this
repository's root), takes its
``SOURCE`` string unchanged into ``oracle/_ref/ref_kernels.inc`` and compiles it
with ``oracle/ref_shim.cpp``.  Everything it writes stays under ``oracle/_ref/``
(git-ignored).  Without a reference checkout it does nothing.
"""

from __future__ import annotations

import ast
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"


def reference_root() -> Path:
    """The reference checkout: ``$CUBAM_REFERENCE``, else ``reference`` next to this repository."""
    env = os.environ.get("CUBAM_REFERENCE")
    return Path(env) if env else HERE.parent.parent / "reference"


def build(force: bool = False) -> Path | None:
    src = reference_root() / "src" / "cubam" / "_kernels.py"
    if not src.exists():
        return None
    OUT.mkdir(exist_ok=True)
    lib = OUT / "libref_kernels.so"
    shim = HERE / "ref_shim.cpp"
    if lib.exists() and not force and lib.stat().st_mtime > max(src.stat().st_mtime, shim.stat().st_mtime):
        return lib
    tree = ast.parse(src.read_text())
    code = next(
        n.value.value
        for n in tree.body
        if isinstance(n, ast.Assign) and any(getattr(t, "id", None) == "SOURCE" for t in n.targets)
    )
    (OUT / "ref_kernels.inc").write_text(code)
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-w", f"-I{OUT}", str(shim), "-o", str(lib)]
    subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    p = build(force="--force" in sys.argv)
    print(p if p else "no reference checkout: nothing built")
