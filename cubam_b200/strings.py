"""String columns on the GPU: the bytes of all strings and their offsets.

cubam returns cuDF STRING columns built from the same two buffers
(``src/cubam/bam.py:115-134``).  :class:`StringColumn` keeps them as device
tensors; :meth:`StringColumn.to_cudf` builds the cuDF column when cuDF is
installed, and :meth:`StringColumn.to_arrow` gives a pyarrow array (through
the host), so code written for cuDF's ``.to_arrow().to_pylist()`` works.
"""

from __future__ import annotations

import numpy as np
import torch


class StringColumn:
    """``chars[offsets[i]:offsets[i + 1]]`` for i in ``range(len(self))``; offsets are int32 below 2^31 - 1 bytes."""

    def __init__(self, chars: torch.Tensor, offsets: torch.Tensor):
        self.chars = chars
        self.offsets = offsets

    def __len__(self) -> int:
        return int(self.offsets.numel()) - 1

    def to_arrow(self):
        import pyarrow as pa

        n = len(self)
        off = self.offsets.cpu().numpy()
        total = int(off[-1]) if n >= 0 and off.size else 0
        chars = self.chars[:total].cpu().numpy().tobytes() if total else b""
        typ = pa.string() if off.dtype == np.int32 else pa.large_string()
        return pa.Array.from_buffers(typ, n, [None, pa.py_buffer(off.tobytes()), pa.py_buffer(chars)])

    def to_pylist(self) -> list:
        return self.to_arrow().to_pylist()

    def to_bytes_list(self) -> list[bytes]:
        off = self.offsets.cpu().numpy().astype(np.int64)
        chars = self.chars.cpu().numpy().tobytes()
        return [chars[off[i] : off[i + 1]] for i in range(len(self))]

    def to_cudf(self):
        """The cuDF STRING column of these buffers (needs cuDF and pylibcudf)."""
        import cudf
        import cupy as cp
        import pylibcudf as plc

        chars = cp.from_dlpack(self.chars)
        offsets = cp.from_dlpack(self.offsets)
        col = plc.Column(
            plc.DataType(plc.TypeId.STRING),
            len(self),
            plc.gpumemoryview(chars),
            None,
            0,
            0,
            [plc.Column.from_cuda_array_interface(offsets)],
        )
        return cudf.Series.from_pylibcudf(col)

    def __repr__(self) -> str:
        return f"StringColumn(n={len(self)}, bytes={int(self.offsets[-1]) if len(self) >= 0 else 0})"
