"""BGZF files read and inflated on the B200.

Same API and chunk semantics as cubam's ``src/cubam/bgzf.py`` read side
(``inflate_chunks`` ``:615``, ``_inflate`` ``:625-652``, ``_inflate_blocks``
``:542-612``, ``_ChunkReader`` ``:38-125``), on this package's kernels:

1. **Read.** A background thread reads the next chunks into pinned host
   slots with parallel ``preadv`` calls and copies each to the device on a
   stream of its own; the consumer waits on the copy's event
   (``_ChunkReader``).
2. **Find members.** ``cb_scan_members``: 128-bit loads and byte matching find
   every BGZF header, the chain from offset 0 is kept and checked, and one
   inflate job per non-empty member is written with its output offset.  The
   compressed bytes of the incomplete last member stay on the GPU.
3. **Inflate.** ``cb_inflate_form`` in the library's default form (form 3:
   the Huffman decode with one member per lane into a token arena, then the
   copy with one member per warp), with the CRC32 and ISIZE checks.

Errors are the reference's ``ValueError`` messages; a CRC32 mismatch (which
cubam does not check) is a ``ValueError`` too, unless ``check_crc=False``.
"""

from __future__ import annotations

import os
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
    if status == _lib.TIMEOUT:
        raise TimeoutError(f"{what}: deadline passed before it was served")
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
    """The chunks of a file on the device, read ahead on the host by one background thread.

    The thread fills pinned host slots (``n_buffers`` of ``chunk_bytes``) in turn: a chunk is read
    by ``n_threads`` workers with ``os.preadv`` of ``piece`` bytes each, straight into its slot.
    Iterating yields ``(chunk, eof)`` with the chunk on the device; the copy of the NEXT chunk is
    issued (on a stream of its own, into memory of the consumer's stream) before the current one is
    yielded, so it runs under the kernels the consumer launches for the current one; the consumer's
    stream waits on the copy's event, never the host.  A slot is refilled once the copy out of it
    has completed, and the thread reads at most ``n_buffers`` chunks ahead.

    An exception in the thread (an unreadable file, a short read) reaches the consumer at the first
    chunk it has not delivered.  Without CUDA the chunks are host tensors (no pinned memory, no
    stream), which is how the reading logic is tested on a host without a GPU.
    """

    def __init__(self, path, chunk_bytes: int, *, n_buffers: int = 3, n_threads: int = 16, piece: int = 16 << 20):
        self.path, self.chunk = Path(path), int(chunk_bytes)
        self.n_buffers, self.n_threads, self.piece = max(int(n_buffers), 1), max(int(n_threads), 1), max(int(piece), 1)
        self._cuda = torch.cuda.is_available()
        self._slots = [torch.empty(self.chunk, dtype=torch.uint8, pin_memory=self._cuda) for _ in range(self.n_buffers)]
        self._cv = threading.Condition()
        self._ready: dict[int, tuple] = {}         # chunk index -> (slot, nbytes, eof), read by the thread
        self._copied: list = [None] * self.n_buffers  # event of the last copy out of each slot
        self._taken = 0                              # chunks the consumer has taken from the thread
        self._failure: BaseException | None = None
        self._closed = False
        self._thread = threading.Thread(target=self._produce, name="cubam-reader", daemon=True)
        self._thread.start()

    def close(self) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()

    @staticmethod
    def _read_piece(fd: int, dst: memoryview, offset: int) -> None:
        """Fill ``dst`` from ``offset`` of the file (pread until it is full)."""
        while len(dst):
            got = os.preadv(fd, [dst], offset)
            if got <= 0:
                raise ValueError("The file is shorter than its size")
            dst, offset = dst[got:], offset + got

    def _produce(self) -> None:
        from concurrent.futures import ThreadPoolExecutor

        try:
            fd = os.open(self.path, os.O_RDONLY)
            try:
                size = os.fstat(fd).st_size
                with ThreadPoolExecutor(self.n_threads) as workers:
                    k = off = 0
                    while True:
                        slot = k % self.n_buffers
                        with self._cv:
                            while not self._closed and k - self._taken >= self.n_buffers:
                                self._cv.wait()
                            if self._closed:
                                return
                            ev = self._copied[slot]
                        if ev is not None:
                            ev.synchronize()  # the copy out of this slot has completed
                        n = min(self.chunk, size - off)
                        view = memoryview(self._slots[slot].numpy())[:n]
                        reads = [workers.submit(self._read_piece, fd, view[p : p + self.piece], off + p)
                                 for p in range(0, n, self.piece)]
                        for r in reads:
                            r.result()
                        off += n
                        eof = off >= size
                        with self._cv:
                            self._ready[k] = (slot, n, eof)
                            self._cv.notify_all()
                        if eof:
                            return
                        k += 1
            finally:
                os.close(fd)
        except BaseException as e:  # noqa: BLE001  (raised in the consumer)
            with self._cv:
                self._failure = e
                self._cv.notify_all()

    def _take(self, k: int) -> tuple:
        with self._cv:
            while k not in self._ready and self._failure is None:
                self._cv.wait()
            if k not in self._ready:
                raise self._failure  # type: ignore[misc]
            return self._ready.pop(k)

    def _upload(self, k: int, stream) -> tuple:
        """Chunk k on the device: its copy issued on ``stream``; (tensor, eof, event)."""
        slot, n, eof = self._take(k)
        if not self._cuda:
            chunk = self._slots[slot][:n].clone()
            with self._cv:
                self._taken = k + 1
                self._cv.notify_all()
            return chunk, eof, None
        chunk = torch.empty(n, dtype=torch.uint8, device="cuda")  # memory of the consumer's stream
        stream.wait_stream(torch.cuda.current_stream())  # the memory may have been in use there
        with torch.cuda.stream(stream):
            chunk.copy_(self._slots[slot][:n], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        with self._cv:
            self._copied[slot] = ev
            self._taken = k + 1
            self._cv.notify_all()
        return chunk, eof, ev

    def __iter__(self) -> Iterator[tuple[torch.Tensor, bool]]:
        stream = torch.cuda.Stream() if self._cuda else None
        k = 0
        cur = self._upload(0, stream)
        while cur is not None:
            chunk, eof, ev = cur
            failure = None
            try:
                cur = None if eof else self._upload(k + 1, stream)  # the next copy runs under this chunk's work
            except BaseException as e:  # noqa: BLE001  (raised after the chunk read before it)
                cur, failure = None, e
            if ev is not None:
                torch.cuda.current_stream().wait_event(ev)
            yield chunk, eof
            del chunk
            if failure is not None:
                raise failure
            k += 1


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


def inflate_form(form: int = 0, n_jobs: int | None = None) -> int:
    """The inflate form a call of ``n_jobs`` jobs with ``form`` runs, as ``cb_inflate_form`` chooses it:
    0 is the library's default (``CB_PARAM_INFLATE_FORM``; form 1 in place of form 3 below
    ``CB_PARAM_SPLIT_MIN_JOBS`` jobs)."""
    if form:
        return int(form)
    f = int(_lib.lib.cb_get_param(_lib.PARAM_INFLATE_FORM))
    if f == 3 and n_jobs is not None and n_jobs < int(_lib.lib.cb_get_param(_lib.PARAM_SPLIT_MIN_JOBS)):
        return 1
    return f


def inflate_workspace_bytes(n_jobs: int, out_bytes: int, form: int = 0) -> int:
    """Workspace bytes of an inflate of ``n_jobs`` jobs writing ``out_bytes`` bytes in total, in ``form``."""
    if inflate_form(form, n_jobs) == 3:
        return max(int(_lib.lib.cb_inflate_split_workspace_bytes(n_jobs, out_bytes)), 512)
    return int(_lib.lib.cb_inflate_workspace_bytes())


def launch_inflate(jobs_ptr: int, n_jobs: int, out_ptr, out_bytes: int, check_crc: bool, summary_ptr: int,
                   workspace: torch.Tensor, form: int = 0, job_status_ptr=None, d_n_jobs_ptr=None) -> None:
    """``cb_inflate_form`` on the current stream with a workspace from :func:`inflate_workspace_bytes`
    (a workspace larger than the forms-1/2 size selects form 3 when the form asks for it)."""
    rc = _lib.lib.cb_inflate_form(jobs_ptr, n_jobs, d_n_jobs_ptr, out_ptr, int(check_crc), job_status_ptr, summary_ptr,
                                  workspace.data_ptr(), workspace.numel(), int(form), stream_ptr())
    _lib.check(rc, "cb_inflate_form")


def inflate_jobs(jobs: torch.Tensor, n_jobs: int, out: torch.Tensor, check_crc: bool = True, form: int = 0,
                 job_status: torch.Tensor | None = None) -> torch.Tensor:
    """Launch ``cb_inflate_form`` of ``n_jobs`` jobs into ``out``; returns the device summary (no sync).

    ``form`` 0 lets the library choose (``CB_PARAM_INFLATE_FORM``), 1 is one member per warp, 2 one per
    lane, 3 the two-kernel form (``cb_inflate_split``: decode one member per lane, copy one per warp).
    ``job_status`` (device uint32/int32 of ``n_jobs``) receives a status code per job when given.
    """
    summ = torch.zeros(ctypes_sizeof(_lib.InflateSummary), dtype=torch.uint8, device="cuda")
    out_bytes = int(out.numel())
    ws = _workspace(inflate_workspace_bytes(n_jobs, out_bytes, form))
    launch_inflate(jobs.data_ptr(), n_jobs, out.data_ptr() if out_bytes else None, out_bytes, check_crc,
                   summ.data_ptr(), ws, form, job_status.data_ptr() if job_status is not None else None)
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
    carry = torch.empty(0, dtype=torch.uint8, device="cuda")  # the incomplete last member, compressed
    try:
        for chunk, eof in reader:
            buf = torch.cat([carry, chunk]) if carry.numel() else chunk
            del chunk
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
