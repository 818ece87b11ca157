"""One BAM file decoded by several GPUs: shards at member boundaries, each rank's records found
speculatively, and only a boundary check passed from rank to rank.

cubam reads a file on one GPU; this splits it (the multi-GPU row of the path: members are
independent, records span members).  Rank k of N:

1. finds its shard, from the first BGZF member at or after k/N of the file to the first member at
   or after (k+1)/N (:func:`member_boundaries`), reading only small windows of the file around those
   points -- a member header followed by member headers BSIZE later, for a few members.  No shard
   but rank 0's starts before the end of the member where the BAM header ends, so rank 0 holds and
   skips the whole header however many members it takes;
2. reads and inflates its members (one inflate launch), leaving room in front of its bytes for the
   previous rank's incomplete-record tail;
3. speculates where its first record starts (``cb_first_record``: the first offset where the record
   predicate holds for a few linked records) and chains its records from there -- all ranks at once;
4. receives the previous rank's tail (:func:`recv_tail`), places it in front of its bytes, and
   checks that the records of tail + bytes before the speculative start end exactly there.  When
   they do, the speculation stands; when they do not (a false start), the rank chains its bytes
   again from the tail.  Then it sends its own tail on (:func:`send_tail`);
5. decodes the columns and tags of its records, after the send.

Only step 4 waits for the previous rank, and it chains a few records.  The exchange is a
send/recv of a length and the tail bytes (``torch.distributed``: NCCL for device tensors, gloo for
host tensors); there is no collective and no multicast.

:class:`ShardProtocol` holds steps 3-4 over abstract primitives, so that the rank logic is tested
on the host with a restatement of the record predicate; :class:`Shard` is the GPU form.
"""

from __future__ import annotations

import os
import struct
from pathlib import Path

import torch

from cubam_b200 import _lib
from cubam_b200.bam import BamHeader, record_chain
from cubam_b200.batch import DecodedFile, _View
from cubam_b200.bgzf import _inflate_blocks, check_inflate, raise_status, read_struct, stream_ptr

MAGIC = b"\x1f\x8b\x08\x04"
#: room in front of a rank's inflated bytes for the previous rank's tail: an incomplete record is
#: shorter than 4 + 2^22 bytes (block_size is at most 2^22)
TAIL_ROOM = (4 << 20) + 64
#: records a speculative start must chain through (or reach the end of the data)
SPECULATION_HOPS = 4
_WINDOW = 1 << 17


class _Source:
    """Random access to a file's bytes: an in-memory copy, or a path read by windows."""

    def __init__(self, src):
        if isinstance(src, (bytes, bytearray, memoryview)):
            self._mem = memoryview(src)
            self.size = len(src)
            self._fd = None
        else:
            self._mem = None
            self._fd = os.open(src, os.O_RDONLY)
            self.size = os.fstat(self._fd).st_size

    def read(self, off: int, n: int) -> bytes:
        if off >= self.size or n <= 0:
            return b""
        n = min(n, self.size - off)
        if self._mem is not None:
            return bytes(self._mem[off : off + n])
        return os.pread(self._fd, n, off)

    def close(self) -> None:
        if self._fd is not None:
            os.close(self._fd)
            self._fd = None


def _bsize_at(src: _Source, o: int) -> int:
    """BSIZE + 1 of a BGZF member header at ``o`` (the reference's test, ``_kernels.py:69-80``), else 0."""
    h = src.read(o, 18)
    if len(h) < 18 or h[:4] != MAGIC:
        return 0
    if struct.unpack_from("<H", h, 10)[0] != 6 or h[12:16] != b"BC\x02\x00":
        return 0
    return struct.unpack_from("<H", h, 16)[0] + 1


def first_member_at_or_after(src, start: int, hops: int = 4) -> int:
    """The first offset >= start where a member header begins and the chain of the next ``hops``
    members holds (or reaches the end of the file); the file size when there is none."""
    s = src if isinstance(src, _Source) else _Source(src)
    n = s.size
    o = start
    while o < n:
        win = s.read(o, _WINDOW)
        k = win.find(MAGIC)
        if k < 0:
            if o + len(win) >= n:
                return n
            o += len(win) - 3
            continue
        c = o + k
        p, ok = c, True
        for _ in range(hops):
            bs = _bsize_at(s, p)
            if bs == 0:
                ok = False
                break
            p += bs
            if p >= n:
                break
        if ok and (p >= n or _bsize_at(s, p) or p > n - 18):
            return c
        o = c + 1
    return n


def records_start_member(src, header_size: int) -> int:
    """The end of the member in which the BAM header (``header_size`` inflated bytes) ends: the first
    offset at which a shard other than rank 0's may start."""
    s = src if isinstance(src, _Source) else _Source(src)
    o, inflated = 0, 0
    while o < s.size:
        bs = _bsize_at(s, o)
        if bs == 0:
            return o
        isize = struct.unpack("<I", s.read(o + bs - 4, 4).ljust(4, b"\0"))[0]
        inflated += isize
        o += bs
        if inflated >= header_size:
            return o
    return o


def member_boundaries(src, world: int, header_size: int = 0) -> list[int]:
    """Shard starts of ranks 0..world-1 and the end of the file (world + 1 offsets, non-decreasing).
    ``src``: the file's bytes or its path (then only windows around the cut points are read).  With
    ``header_size``, no shard after rank 0's starts before the member where the header ends."""
    s = src if isinstance(src, _Source) else _Source(src)
    try:
        n = s.size
        lo = records_start_member(s, header_size) if header_size else 0
        out = [0]
        for k in range(1, world):
            out.append(max(out[-1], first_member_at_or_after(s, max((n * k) // world, lo))))
        out.append(n)
        return out
    finally:
        if s is not src:
            s.close()


def recv_tail(rank: int, group=None, device: str = "cuda") -> torch.Tensor:
    """The incomplete-record tail that rank - 1 sends (empty on rank 0): a length, then the bytes."""
    import torch.distributed as td

    got = torch.empty(0, dtype=torch.uint8, device=device)
    if rank > 0:
        n = torch.zeros(1, dtype=torch.int64, device=device)
        td.recv(n, src=rank - 1, group=group)
        got = torch.empty(int(n.item()), dtype=torch.uint8, device=device)
        if got.numel():
            td.recv(got, src=rank - 1, group=group)
    return got


def send_tail(tail: torch.Tensor, rank: int, world: int, group=None) -> None:
    """This rank's incomplete-record tail to rank + 1 (nothing on the last rank)."""
    import torch.distributed as td

    if rank + 1 < world:
        n = torch.tensor([int(tail.numel())], dtype=torch.int64, device=tail.device)
        td.send(n, dst=rank + 1, group=group)
        if tail.numel():
            td.send(tail.contiguous(), dst=rank + 1, group=group)


class ShardProtocol:
    """Steps 3 and 4 of a rank (see the module docstring) over four primitives of a subclass:

    - ``_first_record(limit) -> int``: the speculative first record start in the rank's bytes, or -1;
    - ``_chain(start, stop) -> (offsets, tail, ok)``: the record chain of the combined bytes (tail in
      front, then the rank's bytes) from ``start`` up to ``stop``: record offsets, where the record
      after the last complete one starts, and whether every record on the way passed;
    - ``_place_tail(prev)``: put the previous rank's tail in front of the rank's bytes;
    - ``_cat(a, b)``: offsets ``a`` then ``b``.

    Positions are in the combined bytes (``t`` = the tail's length, the rank's own bytes after it)."""

    rank: int
    n_data: int

    def speculate(self, limit: int | None = None) -> None:
        """Step 3: the speculative first record and the chain from it (no previous tail needed)."""
        if self.rank == 0 or self.n_data == 0:
            self.start = 0
        else:
            # a record starts within 4 + 2^22 bytes of any position (block_size is at most 2^22)
            s = self._first_record(min(self.n_data, TAIL_ROOM) if limit is None else limit)
            self.start = self.n_data if s < 0 else s
        self._spec = self._chain(self.start, self.n_data, tail_len=0)

    def confirm(self, prev) -> tuple:
        """Step 4: the records of the combined bytes once the previous tail ``prev`` is known:
        ``(offsets, tail position, speculation held)`` in the combined bytes."""
        t = self._place_tail(prev)
        offs, tail, ok = self._spec
        if self.start == 0 and t == 0:
            return offs, tail, True
        b_offs, b_tail, b_ok = self._chain(0, t + self.start, tail_len=t)  # the records across the boundary
        if b_ok and b_tail == t + self.start and ok:
            return self._cat(b_offs, self._shift(offs, t)), tail + t, True
        offs, tail, ok = self._chain(0, t + self.n_data, tail_len=t)  # a false start: chain everything again
        if not ok:
            raise ValueError("No valid block or record where one was expected: the data is corrupt")
        return offs, tail, False


class Shard(ShardProtocol):
    """Rank ``rank``'s part of a file on the GPU: its members inflated (with room for the previous
    rank's tail in front), its records found speculatively, waiting for the previous rank's tail."""

    def __init__(self, path: str | Path, rank: int, world: int, raw: bytes | None = None):
        self.path = Path(path)
        self.rank, self.world = rank, world
        self.header = BamHeader.read(path)
        self.n_ref = len(self.header.names)
        src = _Source(raw if raw is not None else self.path)
        try:
            self.bounds = member_boundaries(src, world, self.header.size)
            a, b = self.bounds[rank], self.bounds[rank + 1]
            comp_host = src.read(a, b - a)
        finally:
            src.close()
        room = torch.zeros(TAIL_ROOM, dtype=torch.uint8, device="cuda")
        self.summary = None
        skip = 0
        if comp_host:  # a rank of a file smaller than the ranks has no members
            comp = torch.frombuffer(bytearray(comp_host), dtype=torch.uint8).cuda()
            out, used, self.summary = _inflate_blocks(comp, rank + 1 == world, room, True, True)
            if used != b - a:
                raise ValueError("a shard does not end at a member boundary")
            if rank == 0:
                skip = min(self.header.size, int(out.numel()) - TAIL_ROOM)  # all of the header is in rank 0's shard
        else:
            out = room
        self._out = out
        self._base = TAIL_ROOM + skip          # where the rank's own bytes start in _out
        self.n_data = int(out.numel()) - self._base
        self._t = 0

    # ---- the primitives
    def _first_record(self, limit: int) -> int:
        first = torch.empty(1, dtype=torch.int64, device="cuda")
        data = self._out[self._base :]
        rc = _lib.lib.cb_first_record(data.data_ptr(), self.n_data, self.n_ref, limit, SPECULATION_HOPS,
                                      first.data_ptr(), stream_ptr())
        _lib.check(rc, "cb_first_record")
        return int(first.item())

    def _chain(self, start: int, stop: int, tail_len: int):
        base = self._base - tail_len
        buf = self._out[base + start : base + stop]
        n = int(buf.numel())
        if n == 0:
            return torch.empty(0, dtype=torch.int64, device="cuda"), start, True
        offsets, cs = record_chain(buf, self.n_ref)
        s = read_struct(cs, _lib.ChainSummary)
        ok = s.status == _lib.OK
        if s.status not in (_lib.OK, _lib.NO_CHAIN):
            raise_status(s.status, "record chain")
        nrec = int(s.n_records) if ok else 0
        return offsets[:nrec] + start, start + (int(s.tail) if ok else 0), ok

    def _place_tail(self, prev: torch.Tensor) -> int:
        t = int(prev.numel())
        if t > TAIL_ROOM:
            raise ValueError("an incomplete record longer than a BAM record can be")
        if t:
            self._out[self._base - t : self._base].copy_(prev)
        self._t = t
        return t

    @staticmethod
    def _shift(offs: torch.Tensor, t: int) -> torch.Tensor:
        return offs + t

    @staticmethod
    def _cat(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
        return torch.cat([a, b]) if a.numel() else b

    # ---- the rank's steps
    def finish(self, prev_tail: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
        """Step 4 with the previous rank's tail: (record offsets in :attr:`data`, this rank's tail)."""
        if self.summary is not None:
            check_inflate(self.summary)
        offs, tail, _ = self.confirm(prev_tail)
        self.data = self._out[self._base - self._t :]
        self.offsets = offs
        own_tail = self.data[tail:].clone()
        if self.rank + 1 == self.world and int(own_tail.numel()):
            raise ValueError("truncated BAM file (incomplete record at the end)")
        return offs, own_tail

    def decode(self, tags=("CB", "UB", "GN")) -> DecodedFile:
        """Step 5: the columns and tags of the rank's records."""
        from cubam_b200.bam import RecordBatch, Tag

        data, off = self.data, self.offsets
        b = RecordBatch.decode(data, off, self.header)
        if tags and len(b):
            tag_cols = {t: T for t, T in zip(tags, b.tags(*tags))}
        else:
            view = _View(data, off)
            z8 = torch.empty(0, dtype=torch.uint8, device="cuda")
            z64 = torch.empty(0, dtype=torch.int64, device="cuda")
            z32 = torch.empty(0, dtype=torch.int32, device="cuda")
            tag_cols = {t: Tag._from_columns(view, t, z8, z64, z32, z64) for t in tags}
        return DecodedFile(self.header, data, off, b.columns, tag_cols, 0, self.n_data)


def decode_sharded(path: str | Path, rank: int, world: int, group=None, tags=("CB", "UB", "GN")) -> DecodedFile:
    """This rank's records of ``path`` decoded by ``world`` ranks (each process one GPU), the tails
    passed along over ``torch.distributed`` (initialised by the caller; NCCL with device tensors)."""
    sh = Shard(path, rank, world)
    sh.speculate()
    prev = recv_tail(rank, group)
    _, tail = sh.finish(prev)
    send_tail(tail, rank, world, group)
    return sh.decode(tags)


def decode_shards_in_turn(path: str | Path, world: int, tags=("CB", "UB", "GN")) -> list[DecodedFile]:
    """All ranks' results computed in this process (one GPU), the tails handed on directly: the sharded
    decode without a process group (every rank speculates before any tail is handed on)."""
    raw = Path(path).read_bytes()
    shards = [Shard(path, k, world, raw) for k in range(world)]
    for sh in shards:
        sh.speculate()
    prev = torch.empty(0, dtype=torch.uint8, device="cuda")
    for sh in shards:
        _, prev = sh.finish(prev)
    return [sh.decode(tags) for sh in shards]
