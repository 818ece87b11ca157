"""Write app_imports.json: every name cubam's application layer imports from cubam, by module.

The application layer is every module of ``src/cubam`` but the reader's own (``__init__``,
``bam``, ``bgzf``, ``_kernels``, ``_memory``): ``apps/*.py``, ``cells``, ``filters``, ``intervals``,
``_contigs``, ``bigwig``, ``_cellsnp``, ``cli``.  Reads them from a cubam checkout (``$CUBAM_REFERENCE``, else the directory
``reference`` beside this repository) with :mod:`ast`; nothing is executed.
"""

import ast
import json
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = Path(os.environ.get("CUBAM_REFERENCE", HERE.parents[2] / "reference"))


def main() -> None:
    names: dict[str, set[str]] = {}
    pkg = ROOT / "src" / "cubam"
    reader = {"__init__.py", "bam.py", "bgzf.py", "_kernels.py", "_memory.py"}
    files = sorted(pkg.glob("apps/*.py")) + sorted(f for f in pkg.glob("*.py") if f.name not in reader)
    for f in files:
        for node in ast.walk(ast.parse(f.read_text())):
            if isinstance(node, ast.ImportFrom) and node.module and node.module.split(".")[0] == "cubam":
                names.setdefault(node.module, set()).update(a.name for a in node.names)
    out = {m: sorted(v) for m, v in sorted(names.items())}
    (HERE / "app_imports.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
