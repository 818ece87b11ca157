"""A package named ``cubam`` over this library, for programs written against cubam's reader.

cubam's applications import the reader by its own names: ``from cubam.bam import RecordBatch,
read_bam, _strings_at``, ``from cubam.bgzf import BgzfWriter, BLOCK_DATA``, ``from cubam._kernels
import launch, copy_spans``, ``from cubam import memory_pool`` (``src/cubam/apps/*.py``).  The
directory ``shim/`` holds a package ``cubam`` whose modules ``cubam``, ``cubam.bam``, ``cubam.bgzf``,
``cubam._kernels`` and ``cubam._memory`` give those names from this library.  :func:`install` puts
it first on ``sys.path``.

cubam's application layer -- ``cells``, ``filters``, ``intervals``, ``_contigs``, ``bigwig``,
``_cellsnp``, ``cli`` and ``apps`` -- is not part of the reader and is not rebuilt here: given the
directory of cubam's own ``cubam`` package, :func:`install` appends it to the shim package's
``__path__``, so those modules load from cubam's sources while every reader name they import
(``from cubam.bam import _fnv1a`` and the like) resolves to this library.
"""

from __future__ import annotations

import sys
from pathlib import Path

#: the directory that holds the shim package ``cubam``
SHIM_DIR = Path(__file__).resolve().with_name("shim")
#: modules of the shim (the reader)
READER_MODULES = ("cubam", "cubam.bam", "cubam.bgzf", "cubam._kernels", "cubam._memory")
#: cubam's application layer, loaded from cubam's own sources when :func:`install` is given them
APP_LAYER = ("cubam.cells", "cubam.filters", "cubam.intervals", "cubam._contigs", "cubam.bigwig",
             "cubam._cellsnp", "cubam.cli", "cubam.apps")


def install(app_layer: str | Path | None = None):
    """Make ``import cubam`` load the shim; returns the package.

    ``app_layer`` is the directory of cubam's own ``cubam`` package (``src/cubam`` of a checkout):
    its modules that the shim does not define load from there.  Raises RuntimeError when another
    ``cubam`` is already imported in this process.
    """
    mod = sys.modules.get("cubam")
    if mod is not None and Path(mod.__file__).resolve().parent.parent != SHIM_DIR:
        raise RuntimeError(f"a package named cubam is already imported from {mod.__file__}")
    if str(SHIM_DIR) not in sys.path:
        sys.path.insert(0, str(SHIM_DIR))
    import cubam

    if app_layer is not None:
        d = str(Path(app_layer).resolve())
        if d not in cubam.__path__:
            cubam.__path__.append(d)
    return cubam


def uninstall() -> None:
    """Drop the shim from ``sys.path`` and every ``cubam`` module from ``sys.modules``."""
    while str(SHIM_DIR) in sys.path:
        sys.path.remove(str(SHIM_DIR))
    for name in [m for m in sys.modules if m == "cubam" or m.startswith("cubam.")]:
        del sys.modules[name]
