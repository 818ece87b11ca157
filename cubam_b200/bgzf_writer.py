"""BGZF files written from data on the B200: the write side of cubam's ``src/cubam/bgzf.py``.

Same names, arguments and results as the reference (``_deflate_spans`` ``:248``,
``_crc32_spans`` ``:364``, ``_adler32_spans`` ``:369``, ``_bgzf_compress`` ``:380``,
``BgzfWriter`` ``:425-539``), with torch tensors where the reference has cupy arrays, on this
package's kernels instead of nvCOMP:

- ``cb_deflate_spans`` compresses every span to one raw DEFLATE stream (one CTA per span: hashing,
  match finding, a parallel greedy/lazy parse, Huffman codes, bit emission, all in shared memory),
  takes the CRC32 of each span on the way, and packs the streams one after another -- as BGZF
  members (header, stream, CRC32, ISIZE) for :func:`_bgzf_compress`.  A span is written as the
  smallest of a dynamic-Huffman, a fixed-Huffman and a stored block, so every member fits BGZF's
  64 KiB and incompressible data costs 5 bytes per span, as the reference's stored fallback.
- ``cb_crc32_spans`` / ``cb_adler32_spans``: one warp per span.

``level`` is 0 (Huffman coding only), 1 (greedy matching) or 2 and up (matching with one position
of lazy lookahead); the reference's levels are nvCOMP's algorithms 0-5, with level 2 its writer's
default.  The output depends only on the input bytes and the level.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np
import torch

from cubam_b200 import _lib
from cubam_b200.bgzf import BLOCK_DATA, EOF_BLOCK, read_struct, stream_ptr

#: Largest span of a raw DEFLATE stream (the reference's limit, ``src/cubam/bgzf.py:304``)
MAX_DEFLATE_SPAN = 1 << 16
#: Spans per native call (1 GiB of 64 KiB spans): bounds the workspace, 64 KiB of output slot per
#: span plus 256 KiB of tokens per resident CTA (about 1.1 GB at this size)
SPANS_PER_CALL = 16384


def _as_index(x, device) -> torch.Tensor:
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=torch.int64).contiguous()
    return torch.as_tensor(np.asarray(x, dtype=np.int64), device=device)


def _as_bytes(data) -> torch.Tensor:
    if isinstance(data, (bytes, bytearray, memoryview)):
        data = torch.frombuffer(bytearray(data), dtype=torch.uint8) if len(data) else torch.empty(0, dtype=torch.uint8)
    if not isinstance(data, torch.Tensor):
        data = torch.as_tensor(np.asarray(data, dtype=np.uint8))
    if data.dtype != torch.uint8:
        raise TypeError("data must be uint8")
    if not data.is_cuda:
        data = data.cuda()
    return data.contiguous()


def _check_spans(data: torch.Tensor, off: torch.Tensor, size: torch.Tensor, limit: int, what: str) -> int:
    """Total bytes of the spans; ValueError for a span outside ``data`` or longer than ``limit``."""
    if off.numel() != size.numel():
        raise ValueError("off and size differ in length")
    if off.numel() == 0:
        return 0
    lo, hi, smax, smin, total = (
        int(v) for v in torch.stack([off.min(), (off + size).max(), size.max(), size.min(), size.sum()]).cpu()
    )
    if smax > limit:
        raise ValueError(f"{what} hold at most {limit:,} bytes")
    if lo < 0 or smin < 0 or hi > data.numel():
        raise ValueError("a span lies outside the data")
    return total


def _deflate_call(data, off, size, level: int, bgzf: bool, total_in: int):
    """One native call: ``(out, out_off, out_size, crc)`` of the spans, packed."""
    n = int(off.numel())
    dev = data.device
    ws = torch.empty(_lib.lib.cb_deflate_workspace_bytes(n), dtype=torch.uint8, device=dev)
    cap = total_in + 36 * n
    out = torch.empty(max(cap, 1), dtype=torch.uint8, device=dev)
    out_off = torch.empty(n, dtype=torch.int64, device=dev)
    out_size = torch.empty(n, dtype=torch.int64, device=dev)
    crc = torch.empty(n, dtype=torch.int32, device=dev)
    summary = torch.zeros(ctypes.sizeof(_lib.DeflateSummary), dtype=torch.uint8, device=dev)
    rc = _lib.lib.cb_deflate_spans(
        data.data_ptr(), off.data_ptr(), size.data_ptr(), n, int(level), int(bgzf), out.data_ptr(), cap,
        out_off.data_ptr(), out_size.data_ptr(), crc.data_ptr(), summary.data_ptr(), ws.data_ptr(), ws.numel(),
        stream_ptr(),
    )
    _lib.check(rc, "cb_deflate_spans")
    s = read_struct(summary, _lib.DeflateSummary)
    if s.status == _lib.ARG:
        raise ValueError("a span is longer than a DEFLATE stream may hold")
    if s.status != _lib.OK:
        raise RuntimeError(f"cb_deflate_spans failed (status {s.status})")
    return out[: s.total], out_off, out_size, crc.view(torch.uint32)


def _deflate_many(data, off, size, level: int, bgzf: bool, max_chunks: int | None):
    max_chunks = max_chunks or SPANS_PER_CALL
    n = int(off.numel())
    limit = BLOCK_DATA if bgzf else MAX_DEFLATE_SPAN
    total = _check_spans(data, off, size, limit, "BGZF blocks" if bgzf else "Deflate chunks")
    parts = []
    for k in range(0, n, max_chunks):
        o, s = off[k : k + max_chunks], size[k : k + max_chunks]
        parts.append(_deflate_call(data, o, s, level, bgzf, total if n <= max_chunks else int(s.sum())))
    if len(parts) == 1:
        return parts[0]
    base = np.cumsum([0] + [int(p[0].numel()) for p in parts[:-1]])
    return (
        torch.cat([p[0] for p in parts]),
        torch.cat([p[1] + int(b) for p, b in zip(parts, base, strict=True)]),
        torch.cat([p[2] for p in parts]),
        torch.cat([p[3] for p in parts]),
    )


def _deflate_spans(data, off, size, level: int = 1, max_chunks: int | None = None):
    """Raw DEFLATE streams of ``data[off[i] : off[i] + size[i]]`` (device uint8), each at most 65,536 bytes.

    Returns ``(out, out_off, out_size)``: the streams packed in one device buffer, with their
    offsets and sizes (``src/cubam/bgzf.py:248-277``).  ``max_chunks`` spans go to each native
    call (default :data:`SPANS_PER_CALL`).
    """
    data = _as_bytes(data)
    off, size = _as_index(off, data.device), _as_index(size, data.device)
    if off.numel() == 0:
        e = torch.empty(0, dtype=torch.int64, device=data.device)
        return torch.empty(0, dtype=torch.uint8, device=data.device), e, e.clone()
    out, out_off, out_size, _ = _deflate_many(data, off, size, level, False, max_chunks)
    return out, out_off, out_size


def _crc32_spans(data, off, size) -> torch.Tensor:
    """CRC32 (as ``zlib.crc32``) of ``data[off[i] : off[i] + size[i]]``, one uint32 per span."""
    return _checksum(_lib.lib.cb_crc32_spans, "cb_crc32_spans", data, off, size)


def _adler32_spans(data, off, size) -> torch.Tensor:
    """Adler-32 (as ``zlib.adler32``) of ``data[off[i] : off[i] + size[i]]``, one uint32 per span."""
    return _checksum(_lib.lib.cb_adler32_spans, "cb_adler32_spans", data, off, size)


def _checksum(fn, name: str, data, off, size) -> torch.Tensor:
    data = _as_bytes(data)
    off, size = _as_index(off, data.device), _as_index(size, data.device)
    _check_spans(data, off, size, 1 << 62, "spans")
    n = int(off.numel())
    out = torch.empty(n, dtype=torch.int32, device=data.device)
    if n:
        _lib.check(fn(data.data_ptr(), off.data_ptr(), size.data_ptr(), n, out.data_ptr(), stream_ptr()), name)
    return out.view(torch.uint32)


def _bgzf_compress(data, level: int = 2, block_off=None, block_size=None, return_offsets: bool = False):
    """``data`` (device uint8) as BGZF blocks, without the EOF block (``src/cubam/bgzf.py:380-422``).

    Blocks hold :data:`BLOCK_DATA` bytes each, or the spans ``block_off``, ``block_size`` (at most
    :data:`BLOCK_DATA` bytes each).  A block that DEFLATE does not shrink is stored.  With
    ``return_offsets``, also returns where each block starts in the output.
    """
    data = _as_bytes(data)
    n = int(data.numel())
    dev = data.device
    if block_off is None:
        off = torch.arange(0, n, BLOCK_DATA, dtype=torch.int64, device=dev)
        isize = torch.clamp(off + BLOCK_DATA, max=n) - off
    else:
        off, isize = _as_index(block_off, dev), _as_index(block_size, dev)
    if off.numel() == 0:
        empty = torch.empty(0, dtype=torch.uint8, device=dev)
        return (empty, torch.empty(0, dtype=torch.int64, device=dev)) if return_offsets else empty
    out, out_off, _, _ = _deflate_many(data, off, isize, level, True, None)
    return (out, out_off) if return_offsets else out


class BgzfWriter:
    """A BGZF file written from data on the GPU (the API of cubam's ``BgzfWriter``,
    ``src/cubam/bgzf.py:425-539``: ``write``, ``flush``, ``close``, a context manager; the same
    blocks for the same calls).

    Bytes given to :meth:`write` (a device uint8 tensor, or bytes) are appended to one staging
    buffer on the device.  Once ``flush_bytes`` are staged, every whole ``BLOCK_DATA`` block of them
    is compressed (:func:`_bgzf_compress`) and the remainder moves to the front of the buffer;
    :meth:`flush` and :meth:`close` compress everything staged.  Each compressed batch is copied to
    a pinned host buffer on a CUDA stream of its own, and a writer thread waits for that copy's event
    and writes the batch at its offset in the file (``n_threads`` parallel ``pwrite`` of ``piece``
    bytes), so compression and disk writes overlap; two batches at most are in flight.  A failed
    write is raised by the next call.  :meth:`close` writes the EOF block after the last batch.
    """

    _IN_FLIGHT = 2

    def __init__(self, path: str | Path, level: int = 2, flush_bytes: int = 1024 * BLOCK_DATA, *, n_threads: int = 8,
                 piece: int = 16 << 20):
        import queue
        import threading
        from concurrent.futures import ThreadPoolExecutor

        self.path = Path(path)
        self.level = level
        self.flush_bytes = int(flush_bytes)
        self._fd = os.open(self.path, os.O_WRONLY | os.O_CREAT | os.O_TRUNC, 0o666)
        self._open = True
        self._stage = torch.empty(max(self.flush_bytes + BLOCK_DATA, BLOCK_DATA), dtype=torch.uint8, device="cuda")
        self._staged = 0
        self._end = 0  # file offset after the batches handed to the writer thread
        self._piece = max(int(piece), 1)
        self._copy_stream = torch.cuda.Stream()
        self._room = threading.Semaphore(self._IN_FLIGHT)
        self._spare: list[torch.Tensor] = []  # pinned buffers back from the writer thread
        self._batches: queue.SimpleQueue = queue.SimpleQueue()
        self._failure: BaseException | None = None
        self._pool = ThreadPoolExecutor(max(int(n_threads), 1))
        self._writer = threading.Thread(target=self._write_batches, name="cubam-bgzf-writer", daemon=True)
        self._writer.start()

    # ---------------------------------------------------------------- the writer thread
    def _pwrite_all(self, mv: memoryview, offset: int) -> None:
        while len(mv):
            k = os.pwrite(self._fd, mv, offset)
            mv, offset = mv[k:], offset + k

    def _write_batches(self) -> None:
        while True:
            item = self._batches.get()
            if item is None:
                return
            host, n, offset, done = item
            try:
                if self._failure is None:
                    if done is not None:
                        done.synchronize()  # the device-to-host copy of this batch
                    mv = memoryview(host.numpy())[:n]
                    parts = [self._pool.submit(self._pwrite_all, mv[a : a + self._piece], offset + a)
                             for a in range(0, n, self._piece)]
                    for f in parts:
                        f.result()
            except BaseException as e:  # noqa: BLE001  (raised by the next call of the owner)
                self._failure = e
            finally:
                self._spare.append(host)
                self._room.release()

    # ---------------------------------------------------------------- the caller's side
    def _raise_failure(self) -> None:
        if self._failure is not None:
            raise self._failure

    def _emit(self, blocks: torch.Tensor) -> None:
        """Hand one batch of BGZF blocks (device) to the writer thread, at the next file offset."""
        n = int(blocks.numel())
        if n == 0:
            return
        self._room.acquire()
        if self._failure is not None:
            self._room.release()
            raise self._failure
        host = next((b for b in self._spare if b.numel() >= n), None)
        if host is not None:
            self._spare.remove(host)
        else:
            host = torch.empty(max(n, 2 * self.flush_bytes), dtype=torch.uint8, pin_memory=True)
        cs = self._copy_stream
        cs.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(cs):
            host[:n].copy_(blocks, non_blocking=True)
            done = torch.cuda.Event()
            done.record(cs)
        blocks.record_stream(cs)
        self._batches.put((host, n, self._end, done))
        self._end += n

    def _compress_staged(self, everything: bool) -> None:
        cut = self._staged if everything else self._staged // BLOCK_DATA * BLOCK_DATA
        if cut:
            self._emit(_bgzf_compress(self._stage[:cut], self.level))
            rest = self._staged - cut
            if rest:  # less than one block: moved to the front
                self._stage[:rest].copy_(self._stage[cut : cut + rest].clone())
            self._staged = rest

    def write(self, data) -> None:
        self._raise_failure()
        data = _as_bytes(data)
        n = int(data.numel())
        if n:
            need = self._staged + n
            if need > self._stage.numel():
                grown = torch.empty(max(need, 2 * self._stage.numel()), dtype=torch.uint8, device="cuda")
                grown[: self._staged].copy_(self._stage[: self._staged])
                self._stage = grown
            self._stage[self._staged : need].copy_(data)
            self._staged = need
        if self._staged >= self.flush_bytes:
            self._compress_staged(everything=False)

    def flush(self) -> None:
        """Compress and write what is buffered, so that the next bytes start a new block."""
        self._compress_staged(everything=True)

    def close(self) -> None:
        if not self._open:
            return
        self._open = False
        try:
            self._compress_staged(everything=True)
            self._room.acquire()
            eof = torch.frombuffer(bytearray(EOF_BLOCK), dtype=torch.uint8)
            self._batches.put((eof, len(EOF_BLOCK), self._end, None))
            self._end += len(EOF_BLOCK)
        finally:
            self._batches.put(None)
            self._writer.join()
            self._pool.shutdown()
            os.close(self._fd)
        self._raise_failure()

    def __enter__(self) -> BgzfWriter:
        return self

    def __exit__(self, *exc) -> None:
        self.close()
