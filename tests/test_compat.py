"""The ``cubam`` compatibility package: every name cubam's application layer imports resolves."""

import json
import sys
from pathlib import Path

import pytest

from cubam_b200 import _lib, compat

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture
def shim():
    compat.uninstall()
    yield compat.install
    compat.uninstall()


def test_every_reader_name_the_apps_import_resolves(shim):
    import importlib

    shim()
    imports = json.loads((GOLDEN / "app_imports.json").read_text())
    checked = 0
    for module, names in imports.items():
        if module not in compat.READER_MODULES:
            assert any(module == m or module.startswith(m + ".") for m in compat.APP_LAYER), module
            continue
        mod = importlib.import_module(module)
        assert Path(mod.__file__).resolve().is_relative_to(compat.SHIM_DIR)
        for name in names:
            if f"{module}.{name}" in compat.APP_LAYER:  # a submodule of the application layer
                continue
            assert hasattr(mod, name), f"{module}.{name}"
            checked += 1
    assert checked >= 30


def test_names_are_this_library(shim):
    cubam = shim()
    import cubam_b200
    from cubam_b200 import bam, bgzf

    assert cubam.read_bam is cubam_b200.read_bam and cubam.memory_pool is cubam_b200.memory_pool
    import cubam.bam
    import cubam.bgzf

    assert cubam.bam._fnv1a is bam._fnv1a and cubam.bam.RecordBatch is bam.RecordBatch
    assert cubam.bgzf.BgzfWriter is bgzf.BgzfWriter and cubam.bgzf.BLOCK_DATA == 0xFF00
    assert cubam.bgzf.EOF_BLOCK == bgzf.EOF_BLOCK


def test_application_layer_loads_from_a_package_directory(shim, tmp_path):
    """Modules the shim does not define load from the given directory, and the reader names they
    import come from this library."""
    pkg = tmp_path / "cubam"
    (pkg / "apps").mkdir(parents=True)
    (pkg / "cells.py").write_text("from cubam.bam import _fnv1a\nfrom cubam import memory_pool\n")
    (pkg / "apps" / "__init__.py").write_text("")
    (pkg / "apps" / "demo.py").write_text("from cubam._kernels import launch, copy_spans\n"
                                          "from cubam.cells import _fnv1a as h\n")
    shim(pkg)
    import cubam.apps.demo
    import cubam.cells
    from cubam_b200 import bam

    assert cubam.cells._fnv1a is bam._fnv1a
    assert cubam.apps.demo.h is bam._fnv1a
    assert Path(cubam.apps.demo.launch.__code__.co_filename).resolve().is_relative_to(compat.SHIM_DIR)


def test_launch_maps_to_exported_entry_points(shim):
    shim()
    import cubam._kernels as k

    exported = set(_lib.exported_symbols())
    assert set(k.KERNELS.values()) <= exported
    k.launch("decode_fixed", 0)  # no items: no launch, as cubam
    with pytest.raises(NotImplementedError, match="vcy_segments"):
        k.launch("vcy_segments", 5, None)
    assert k.kernel("name_hash").name == "name_hash"


def test_install_refuses_another_cubam(shim, monkeypatch, tmp_path):
    fake = type(sys)("cubam")
    fake.__file__ = str(tmp_path / "cubam" / "__init__.py")
    monkeypatch.setitem(sys.modules, "cubam", fake)
    with pytest.raises(RuntimeError, match="already imported"):
        compat.install()


def test_launch_arguments_from_cupy_style_objects(shim):
    """cubam passes CuPy arrays and NumPy scalars: arrays become their device pointers through
    __cuda_array_interface__, scalars become integers, and a host tensor is refused."""
    import numpy as np
    import torch

    shim()
    import cubam._kernels as k

    class CupyLike:
        def __init__(self, ptr):
            self.__cuda_array_interface__ = {"data": (ptr, False), "shape": (4,), "typestr": "|u1", "version": 3}

    assert k._arg(CupyLike(0x7F0000001000)) == 0x7F0000001000
    assert k._arg(np.int64(12)) == 12 and k._arg(np.uint8(ord("C"))) == 67
    assert k._arg(None) is None
    with pytest.raises(TypeError, match="GPU"):
        k._arg(torch.zeros(4))
