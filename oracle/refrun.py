"""Run the reference's own reader code on the CPU: TEST INFRASTRUCTURE ONLY.

cubam's reader (``src/cubam/bam.py``, ``src/cubam/bgzf.py``,
``src/cubam/_kernels.py``) needs CuPy, cuDF and nvCOMP, none of which exist
here.  This module imports the reference checkout unchanged and stands in for
those three:

- ``cupy`` is a numpy-backed module with the calls the reader makes (arrays
  with ``.get()``, ``.set()`` and ``.data.ptr``);
- ``cubam._kernels.kernel`` launches the reference's kernels compiled for the
  CPU by ``oracle/build_ref.py`` (``oracle/_ref/libref_kernels.so``);
- ``cubam.bgzf._nvcomp_decompress`` inflates each member with zlib (raw
  DEFLATE, RFC 1951), writing to the addresses the reader passes, with
  nvCOMP's status/actual-size outputs;
- ``cubam.bam._string_series`` returns the strings as a list of ``bytes``
  instead of a cuDF column.

Everything else is the reference's code path.  Used only by
``tests/golden/make_golden.py`` (to write the golden vectors) and by CPU tests
that skip when no reference checkout is present.
"""

from __future__ import annotations

import ctypes
import os
import sys
import types
import zlib
from pathlib import Path

import numpy as np

from oracle import build_ref

_lib = None


class _Ptr:
    def __init__(self, p):
        self.ptr = p


class FakeArray(np.ndarray):
    """A numpy array with the CuPy methods the reader calls."""

    def get(self, out=None):
        a = np.asarray(self).copy()
        if out is not None:
            out[...] = a
            return out
        return a

    def set(self, x):
        np.asarray(self)[...] = np.asarray(x)

    @property
    def data(self):  # noqa: D401  (CuPy's device pointer)
        return _Ptr(self.ctypes.data)

    def copy(self, order="C"):
        return np.array(np.asarray(self), copy=True).view(FakeArray)


def _w(x):
    if isinstance(x, np.ndarray):
        return x.view(FakeArray)
    return x


def _fake_cupy() -> types.ModuleType:
    cp = types.ModuleType("cupy")
    for t in ("uint8", "int8", "int16", "uint16", "int32", "uint32", "int64", "uint64", "bool_", "float32"):
        setattr(cp, t, getattr(np, t))
    cp.ndarray = FakeArray

    def wrap(f):
        return lambda *a, **k: _w(f(*a, **k))

    for name in (
        "empty",
        "zeros",
        "ones",
        "arange",
        "cumsum",
        "sort",
        "stack",
        "where",
        "flatnonzero",
        "searchsorted",
        "concatenate",
        "minimum",
        "maximum",
        "unique",
        "full",
    ):
        setattr(cp, name, wrap(getattr(np, name)))
    cp.asarray = lambda a, dtype=None: _w(np.asarray(a, dtype=dtype))
    cuda = types.ModuleType("cupy.cuda")
    cuda.alloc_pinned_memory = lambda n: bytearray(n)
    cuda.get_current_stream = lambda: _Ptr(0)
    runtime = types.ModuleType("cupy.cuda.runtime")
    runtime.memGetInfo = lambda: (80 << 30, 80 << 30)
    cuda.runtime = runtime
    cp.cuda = cuda
    return cp


_CTYPE = {
    np.dtype(np.int64): ctypes.c_int64,
    np.dtype(np.uint64): ctypes.c_uint64,
    np.dtype(np.int32): ctypes.c_int32,
    np.dtype(np.uint32): ctypes.c_uint32,
    np.dtype(np.uint8): ctypes.c_uint8,
    np.dtype(np.int8): ctypes.c_int8,
    np.dtype(np.uint16): ctypes.c_uint16,
    np.dtype(np.int16): ctypes.c_int16,
}


def _launcher(name):
    def call(grid, block, args):
        keep = []
        argv = (ctypes.c_void_p * len(args))()
        for i, a in enumerate(args):
            if isinstance(a, np.ndarray):
                v = ctypes.c_void_p(a.ctypes.data)
            elif isinstance(a, np.generic):
                v = _CTYPE[a.dtype](a.item())
            else:
                raise TypeError(f"argument {i} of {name}: {type(a)}")
            keep.append(v)
            argv[i] = ctypes.cast(ctypes.pointer(v), ctypes.c_void_p)
        rc = _lib.ref_launch(name.encode(), ctypes.c_longlong(grid[0] * block[0]), argv)
        if rc:
            raise RuntimeError(f"kernel {name} is not in the host build")

    return call


def _fake_nvcomp_decompress():
    def fn(in_ptr, in_size, out_size, actual, m, _tmp, _tmp_bytes, out_ptr, _opts, status, _stream):
        u64 = ctypes.c_uint64 * m
        ip = u64.from_address(in_ptr)
        isz = u64.from_address(in_size)
        osz = u64.from_address(out_size)
        op = u64.from_address(out_ptr)
        act = u64.from_address(actual)
        st = (ctypes.c_int32 * m).from_address(status)
        for i in range(m):
            payload = ctypes.string_at(ip[i], isz[i])
            d = zlib.decompressobj(-15)
            try:
                out = d.decompress(payload, osz[i] + 1)
                ok = d.eof and len(out) <= osz[i]
            except zlib.error:
                out, ok = b"", False
            out = out[: osz[i]]
            ctypes.memmove(op[i], out, len(out))
            act[i] = len(out)
            st[i] = 0 if ok else 1
        return 0

    return fn


def load(reference: str | os.PathLike | None = None):
    """Import the reference's ``cubam`` with the stand-ins in place; returns the module, or None without a checkout."""
    global _lib
    root = Path(reference) if reference else build_ref.reference_root()
    if not (root / "src" / "cubam" / "bam.py").exists():
        return None
    lib = build_ref.build()
    if lib is None:
        return None
    if _lib is None:
        _lib = ctypes.CDLL(str(lib))
        _lib.ref_launch.argtypes = [ctypes.c_char_p, ctypes.c_longlong, ctypes.c_void_p]
        _lib.ref_launch.restype = ctypes.c_int
    if "cupy" not in sys.modules or not hasattr(sys.modules["cupy"], "ndarray"):
        sys.modules["cupy"] = _fake_cupy()
    src = str(root / "src")
    if src not in sys.path:
        sys.path.insert(0, src)
    import cubam  # noqa: F401
    import cubam._kernels as K
    import cubam.bam as B
    import cubam.bgzf as G

    K.kernel = _launcher
    G._nvcomp_decompress = _fake_nvcomp_decompress

    def strings(chars, offsets):
        c = np.asarray(chars).tobytes()
        o = np.asarray(offsets).astype(np.int64)
        return [c[o[i] : o[i + 1]] for i in range(o.size - 1)]

    B._string_series = strings
    return cubam


def reference_tests_dir(reference: str | os.PathLike | None = None) -> Path:
    root = Path(reference) if reference else build_ref.reference_root()
    return root / "tests"
