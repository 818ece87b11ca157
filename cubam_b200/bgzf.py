"""BGZF files read and inflated on the B200.

Same API and chunk semantics as cubam's ``src/cubam/bgzf.py`` read side
(``inflate_chunks`` ``:615``, ``_inflate`` ``:625-652``, ``_inflate_blocks``
``:542-612``, ``_ChunkReader`` ``:38-125``), on this package's kernels:

1. **Read.** A background thread reads the next chunks into pinned host
   buffers with parallel ``pread`` calls (``_ChunkReader``).
2. **Find members.** ``cb_scan_members``: 128-bit loads and byte matching find
   every BGZF header, the chain from offset 0 is kept and checked, and one
   inflate job per non-empty member is written with its output offset.  The
   compressed bytes of the incomplete last member stay on the GPU.
3. **Inflate.** ``cb_inflate``: one warp per member, persistent grid, with the
   CRC32 and ISIZE checks.

Errors are the reference's ``ValueError`` messages; a CRC32 mismatch (which
cubam does not check) is a ``ValueError`` too, unless ``check_crc=False``.
"""

from __future__ import annotations

import os
import queue
import threading
from collections.abc import Iterator
from pathlib import Path

import torch

from cubam_b200 import _lib

#: The empty BGZF block that ends a file
EOF_BLOCK = bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")
#: Data per BGZF block, as samtools and htslib write
BLOCK_DATA = 0xFF00
#: Check the CRC32 of every member (cubam's reader does not)
CHECK_CRC = True

_HEADER, _TRAILER = 18, 8

_MESSAGES = {
    _lib.TRUNCATED: "Truncated BGZF file: the last block is incomplete",
    _lib.NO_CHAIN: "No valid block or record where one was expected: the data is corrupt",
    _lib.CORRUPT_BLOCK: "Corrupt BGZF block",
    _lib.INFLATE: "Corrupt BGZF block: it does not inflate to the size in its trailer",
    _lib.CRC: "Corrupt BGZF block: CRC32 mismatch",
    _lib.TOO_MANY: "Too many candidates: the data is corrupt",
}


def raise_status(status: int, what: str) -> None:
    """The reference's exception for a device status code."""
    if status == _lib.OK:
        return
    if status in _MESSAGES:
        raise ValueError(_MESSAGES[status])
    raise RuntimeError(f"{what} failed (status {status})")


def stream_ptr() -> int:
    return torch.cuda.current_stream().cuda_stream


def _device_struct(cls) -> torch.Tensor:
    return torch.zeros(ctypes_sizeof(cls), dtype=torch.uint8, device="cuda")


def ctypes_sizeof(cls) -> int:
    import ctypes

    return ctypes.sizeof(cls)


def read_struct(t: torch.Tensor, cls):
    """A summary struct copied from the device (synchronises the stream)."""
    return cls.from_buffer_copy(t.cpu().numpy().tobytes())


class _ChunkReader:
    """Chunks of a file read ahead into pinned buffers by a background thread.

    Each chunk is read by ``n_threads`` parallel ``pread`` calls of ``piece``
    bytes.  Iterating yields ``(slot, nbytes, eof)``; the consumer copies
    :meth:`host` ``(slot)[:nbytes]`` to the GPU and then calls :meth:`release`.
    """

    def __init__(self, path, chunk_bytes: int, *, n_buffers: int = 3, n_threads: int = 8, piece: int = 16 << 20):
        self.path, self.chunk, self.n_threads, self.piece = Path(path), chunk_bytes, n_threads, max(int(piece), 1)
        pin = torch.cuda.is_available()  # page-locked for the H2D copies; plain memory on a host without CUDA
        self._mem = [torch.empty(chunk_bytes, dtype=torch.uint8, pin_memory=pin) for _ in range(n_buffers)]
        self._free: queue.Queue = queue.Queue()
        for i in range(n_buffers):
            self._free.put(i)
        self._full: queue.Queue = queue.Queue()
        self._error: BaseException | None = None
        self._stop = False
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    def host(self, slot: int) -> torch.Tensor:
        return self._mem[slot]

    def release(self, slot: int) -> None:
        self._free.put(slot)

    def close(self) -> None:
        self._stop = True
        self._free.put(-1)

    @staticmethod
    def _pread(fd: int, mv: memoryview, offset: int) -> None:
        while len(mv):
            got = os.preadv(fd, [mv], offset)
            if not got:
                raise ValueError("The file is shorter than its size")
            mv, offset = mv[got:], offset + got

    def _run(self) -> None:
        from concurrent.futures import ThreadPoolExecutor

        try:
            fd = os.open(self.path, os.O_RDONLY)
            try:
                size = os.fstat(fd).st_size
                off = 0
                with ThreadPoolExecutor(self.n_threads) as ex:
                    while True:
                        slot = self._free.get()
                        if self._stop:
                            return
                        n = min(self.chunk, size - off)
                        mv = memoryview(self._mem[slot].numpy())
                        futures = [
                            ex.submit(self._pread, fd, mv[p : min(p + self.piece, n)], off + p)
                            for p in range(0, n, self.piece)
                        ]
                        for f in futures:
                            f.result()
                        off += n
                        eof = off >= size
                        self._full.put((slot, n, eof))
                        if eof:
                            return
            finally:
                os.close(fd)
        except BaseException as e:  # noqa: BLE001  (re-raised in the consumer)
            self._error = e
            self._full.put(None)

    def __iter__(self) -> Iterator[tuple[int, int, bool]]:
        while True:
            item = self._full.get()
            if item is None:
                raise self._error  # type: ignore[misc]
            yield item
            if item[2]:
                return


def _workspace(nbytes: int) -> torch.Tensor:
    return torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device="cuda")


def scan_members(buf: torch.Tensor, eof: bool, out_base: int = 0, jobs_cap: int | None = None):
    """Run ``cb_scan_members`` on ``buf`` (device uint8); returns ``(jobs, summary)`` after one sync."""
    n = int(buf.numel())
    ws = _workspace(_lib.lib.cb_scan_workspace_bytes(n))
    summ = torch.zeros(ctypes_sizeof(_lib.ScanSummary), dtype=torch.uint8, device="cuda")
    cap = jobs_cap if jobs_cap is not None else n // 8192 + 1024
    while True:
        jobs = torch.empty(max(cap, 1) * _lib.JOB_BYTES, dtype=torch.uint8, device="cuda")
        rc = _lib.lib.cb_scan_members(
            buf.data_ptr() if n else None, n, int(eof), out_base, jobs.data_ptr(), cap, summ.data_ptr(),
            ws.data_ptr(), ws.numel(), stream_ptr(),
        )
        _lib.check(rc, "cb_scan_members")
        s = read_struct(summ, _lib.ScanSummary)
        if s.status == _lib.CAPACITY and s.n_jobs > cap:
            cap = int(s.n_jobs)
            continue
        return jobs, s


def inflate_jobs(jobs: torch.Tensor, n_jobs: int, out: torch.Tensor, check_crc: bool = True, form: int = 0,
                 job_status: torch.Tensor | None = None) -> torch.Tensor:
    """Launch ``cb_inflate_form`` of ``n_jobs`` jobs into ``out``; returns the device summary (no sync).

    ``form`` 0 lets the library choose (as ``cb_inflate``), 1 is one member per warp, 2 one per lane.
    ``job_status`` (device uint32/int32 of ``n_jobs``) receives a status code per job when given.
    """
    summ = torch.zeros(ctypes_sizeof(_lib.InflateSummary), dtype=torch.uint8, device="cuda")
    ws = _workspace(_lib.lib.cb_inflate_workspace_bytes())
    rc = _lib.lib.cb_inflate_form(
        jobs.data_ptr(), n_jobs, None, out.data_ptr() if out.numel() else None, int(check_crc),
        job_status.data_ptr() if job_status is not None else None,
        summ.data_ptr(), ws.data_ptr(), ws.numel(), int(form), stream_ptr(),
    )
    _lib.check(rc, "cb_inflate_form")
    return summ


def check_inflate(summ: torch.Tensor) -> None:
    s = read_struct(summ, _lib.InflateSummary)
    raise_status(s.status, "inflate")


def _inflate_blocks(buf: torch.Tensor, eof: bool, prefix: torch.Tensor | None = None, check_crc: bool | None = None,
                    defer_check: bool = False):
    """Inflate the complete BGZF members of ``buf`` (device uint8, starting at a member).

    Returns ``(data, used)`` as ``src/cubam/bgzf.py:542-612`` does: the data
    starts with ``prefix``.  With ``defer_check`` it returns
    ``(data, used, summary)`` and the caller checks the inflate summary later.
    """
    check_crc = CHECK_CRC if check_crc is None else check_crc
    if prefix is None:
        prefix = torch.empty(0, dtype=torch.uint8, device="cuda")
    jobs, s = scan_members(buf, eof)
    raise_status(s.status, "BGZF member scan")
    p = int(prefix.numel())
    out = torch.empty(p + int(s.total_out), dtype=torch.uint8, device="cuda")
    if p:
        out[:p].copy_(prefix)
    summ = None
    if s.n_jobs:
        summ = inflate_jobs(jobs, int(s.n_jobs), out[p:], check_crc)
        if not defer_check:
            check_inflate(summ)
            summ = None
    if defer_check:
        return out, int(s.used), summ
    return out, int(s.used)


def inflate_chunks(path: str | Path, chunk_bytes: int | None = None, **reader_kw) -> Iterator[torch.Tensor]:
    """Inflated data of a BGZF file on the GPU, chunk by chunk (device uint8 tensors).

    Each chunk holds the data of the complete members read so far
    (``src/cubam/bgzf.py:615-622``).  ``check_crc`` (default :data:`CHECK_CRC`)
    may be passed with the reader options.
    """
    return _inflate(path, chunk_bytes, None, **reader_kw)


def _inflate(path: str | Path, chunk_bytes: int | None, prefix, check_crc: bool | None = None,
             defer_check: bool = False, **reader_kw) -> Iterator:
    """:func:`inflate_chunks`, each chunk after the bytes returned by ``prefix()`` (when not None).

    With ``defer_check`` it yields ``(data, summary)``: the inflate summary is
    checked by the caller (:func:`check_inflate`) after its own work on the chunk.
    """
    from cubam_b200._memory import auto_chunk_bytes

    chunk_bytes = chunk_bytes or auto_chunk_bytes()
    reader = _ChunkReader(path, chunk_bytes, **reader_kw)
    carry = torch.empty(0, dtype=torch.uint8, device="cuda")
    copies = torch.cuda.Stream()  # host-to-device copies of the next chunk overlap the work on this one

    def upload(item):
        slot, nbytes, eof = item
        dev = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
        copies.wait_stream(torch.cuda.current_stream())  # dev's memory may have been in use there
        with torch.cuda.stream(copies):
            dev.copy_(reader.host(slot)[:nbytes], non_blocking=True)
        ev = torch.cuda.Event()
        ev.record(copies)
        return slot, eof, dev, ev

    try:
        chunks = iter(reader)
        first = next(chunks, None)
        cur = upload(first) if first is not None else None
        while cur is not None:
            slot, eof, dev, ev = cur
            ev.synchronize()
            reader.release(slot)  # the host slot is copied: the reader may fill it again
            nxt = next(chunks, None)
            cur = upload(nxt) if nxt is not None else None
            torch.cuda.current_stream().wait_event(ev)
            c = int(carry.numel())
            buf = torch.cat([carry, dev]) if c else dev
            del dev
            res = _inflate_blocks(buf, eof, prefix and prefix(), check_crc, defer_check)
            data, used = res[0], res[1]
            carry = buf[used:].clone()
            del buf
            yield (data, res[2]) if defer_check else data
            del data, res
    finally:
        reader.close()


# The write side (it imports this module's names, so it comes last).
from cubam_b200.bgzf_writer import (  # noqa: E402
    BgzfWriter,
    _adler32_spans,
    _bgzf_compress,
    _crc32_spans,
    _deflate_spans,
)
