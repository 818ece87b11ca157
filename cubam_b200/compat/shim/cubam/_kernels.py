"""cubam's kernel launcher (``src/cubam/_kernels.py:627-660``) over this library's C ABI.

cubam compiles one CUDA source with CuPy and launches its kernels by name: ``launch(name, n,
*args)`` with the kernel's own argument list.  Here each name that this library implements maps to
its ``cb_*`` entry point, which takes the same arguments in the same order (plus the stream: the
current torch stream), so a call written for cubam runs on this library's kernels.  Arrays may be
torch tensors or any object with ``__cuda_array_interface__`` (CuPy arrays); scalars may be Python
or NumPy numbers.

Kernels of cubam's application layer (``vcy_segments``, ``natural_name``, ``record_sizes_at``,
``gather_spans``, the bigWig writers) are not part of the reader: they run from cubam's own
``_kernels.py`` when its package directory was given to :func:`cubam_b200.compat.install` (which
needs CuPy, as cubam does), and raise NotImplementedError otherwise.
"""

from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import torch

from cubam_b200 import _lib
from cubam_b200.bgzf import stream_ptr

#: cubam kernel name -> this library's entry point (same arguments, same order)
KERNELS = {
    "copy_spans": "cb_copy_spans",
    "decode_fixed": "cb_decode_fixed",
    "name_hash": "cb_name_hash",
    "aligned_len": "cb_aligned_length",
    "blocks": "cb_blocks",
    "base_at": "cb_base_at",
    "hash_spans": "cb_hash_spans",
    "pack_acgt": "cb_pack_acgt",
    "unpack_acgt": "cb_unpack_acgt",
    "crc32_spans": "cb_crc32_spans",
    "adler32_spans": "cb_adler32_spans",
    "find_tag": "cb_find_tags",
}


def _arg(a):
    """A device pointer or an integer for a ctypes argument."""
    if a is None:
        return None
    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            raise TypeError("kernel arrays must be on the GPU")
        return a.data_ptr()
    cai = getattr(a, "__cuda_array_interface__", None)
    if cai is not None:
        return int(cai["data"][0])
    return int(a)


def _find_tag(b, off, n, t0, t1, type_, voff, vlen, ival, stream):
    """cubam's one-tag ``find_tag`` (``src/cubam/_kernels.py:334-388``) as a one-name ``cb_find_tags``."""
    names = bytes([int(t0), int(t1)])
    return _lib.lib.cb_find_tags(_arg(b), _arg(off), int(n), names, 1, _arg(type_), _arg(voff), _arg(vlen),
                                 _arg(ival), stream)


_reference = None


def _reference_kernels():
    """cubam's own ``_kernels`` module, from a package directory appended to ``cubam.__path__``."""
    global _reference
    if _reference is None:
        pkg = sys.modules["cubam"]
        for d in list(pkg.__path__)[1:]:
            src = Path(d) / "_kernels.py"
            if src.is_file():
                spec = importlib.util.spec_from_file_location("cubam._reference_kernels", src)
                mod = importlib.util.module_from_spec(spec)
                spec.loader.exec_module(mod)
                _reference = mod
                break
    return _reference


def launch(name: str, n: int, *args, threads_per_item: int = 1) -> None:
    """Launch kernel ``name`` over ``n`` items with cubam's argument list for it."""
    if not n:
        return
    fn = KERNELS.get(name)
    if fn is None:
        ref = _reference_kernels()
        if ref is None:
            raise NotImplementedError(
                f"kernel {name!r} belongs to cubam's application layer, not to the reader; "
                "pass cubam's package directory to cubam_b200.compat.install() to run it from there")
        ref.launch(name, n, *args, threads_per_item=threads_per_item)
        return
    stream = stream_ptr()
    if name == "find_tag":
        rc = _find_tag(*args, stream)
    else:
        rc = getattr(_lib.lib, fn)(*[_arg(a) for a in args], stream)
    _lib.check(rc, fn)


class _Kernel:
    """A kernel by name, called as CuPy's RawKernel is: ``kernel(grid, block, args)``."""

    def __init__(self, name: str):
        self.name = name

    def __call__(self, grid, block, args) -> None:
        n = 1
        for g in tuple(grid) + tuple(block):
            n *= int(g)
        launch(self.name, n, *args)


def kernel(name: str) -> _Kernel:
    """Kernel ``name`` (``src/cubam/_kernels.py:627-634``)."""
    return _Kernel(name)


def _device_index(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.int64).contiguous()
    return torch.as_tensor(x, dtype=torch.int64, device=device).contiguous()


def copy_spans(src, dst, src_off, dst_off, size) -> None:
    """``dst[dst_off[i]:][:size[i]] = src[src_off[i]:][:size[i]]`` on the GPU
    (``src/cubam/_kernels.py:645-660``)."""
    dev = src.device if isinstance(src, torch.Tensor) else torch.device("cuda")
    so, do, sz = (_device_index(x, dev) for x in (src_off, dst_off, size))
    launch("copy_spans", int(sz.numel()), src, dst, so, do, sz, int(sz.numel()), threads_per_item=32)
