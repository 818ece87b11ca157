"""One BAM file decoded by several GPUs: shards at member boundaries, record tails passed along.

cubam reads a file on one GPU; this splits it (the multi-GPU row of the path: members are
independent, records span members).  Rank k of N:

1. takes the compressed bytes from the first BGZF member at or after k/N of the file to the first
   member at or after (k+1)/N (:func:`member_boundaries`: every rank finds all boundaries itself,
   from the file, with the chain rule -- a member header followed by a member header BSIZE later,
   for a few members -- so no exchange is needed for them);
2. scans and inflates its members (one inflate launch);
3. receives from rank k-1 the bytes of the record that rank k-1's last member left incomplete
   (:func:`recv_tail` / :func:`send_tail`; a record is at most 4 + 2^31 bytes in the format, in practice a few
   hundred), puts them in front of its own bytes, chains its records from there, and sends its own
   incomplete tail to rank k+1;
4. decodes the columns and tags of its records.

Rank 0's shard starts with the BAM header, which it skips.  The exchange is the only step that
crosses ranks: a send/recv of a length and of the tail bytes, NCCL for device tensors or gloo for
host tensors (``torch.distributed``).  Chaining waits for the previous rank's tail; scans and
inflates of all ranks run at once.
"""

from __future__ import annotations

from pathlib import Path

import torch

from cubam_b200 import _lib
from cubam_b200.bam import BamHeader, record_chain
from cubam_b200.batch import DecodedFile, _View
from cubam_b200.bgzf import _inflate_blocks, check_inflate, raise_status, read_struct

MAGIC = b"\x1f\x8b\x08\x04"


def _is_member(buf: memoryview, o: int, n: int) -> int:
    """BSIZE + 1 of a BGZF member header at ``o`` (the reference's test, ``_kernels.py:69-80``), else 0."""
    if o + 18 > n or bytes(buf[o : o + 4]) != MAGIC:
        return 0
    xlen = buf[o + 10] | (buf[o + 11] << 8)
    if xlen != 6 or buf[o + 12] != 66 or buf[o + 13] != 67 or buf[o + 14] != 2 or buf[o + 15] != 0:
        return 0
    return (buf[o + 16] | (buf[o + 17] << 8)) + 1


def first_member_at_or_after(buf, start: int, hops: int = 4) -> int:
    """The first offset >= start where a member header begins and the chain of the next ``hops``
    members holds (or reaches the end of the file); len(buf) when there is none."""
    mv = memoryview(buf)
    n = len(buf)
    o = start
    while o < n:
        k = bytes(mv[o : min(n, o + (1 << 17))]).find(MAGIC)
        if k < 0:
            o = min(n, o + (1 << 17) - 3)
            if o >= n - 3:
                return n
            continue
        c = o + k
        p, ok = c, True
        for _ in range(hops):
            bs = _is_member(mv, p, n)
            if bs == 0:
                ok = False
                break
            p += bs
            if p == n:
                break
        if ok and (p == n or _is_member(mv, p, n) or p > n - 18):
            return c
        o = c + 1
    return n


def member_boundaries(buf, world: int) -> list[int]:
    """Shard starts of ranks 0..world-1 and the end of the file (world + 1 offsets, non-decreasing)."""
    n = len(buf)
    out = [0]
    for k in range(1, world):
        out.append(max(out[-1], first_member_at_or_after(buf, (n * k) // world)))
    out.append(n)
    return out


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


class Shard:
    """Rank ``rank``'s part of a file: its members inflated, waiting for the previous rank's tail."""

    def __init__(self, path: str | Path, rank: int, world: int, raw: bytes | None = None):
        self.path = Path(path)
        self.rank, self.world = rank, world
        self.header = BamHeader.read(path)
        raw = raw if raw is not None else self.path.read_bytes()
        self.bounds = member_boundaries(raw, world)
        a, b = self.bounds[rank], self.bounds[rank + 1]
        empty = torch.empty(0, dtype=torch.uint8, device="cuda")
        self.summary, self.data = None, empty
        if b > a:  # a rank of a file smaller than the ranks has no members
            comp = torch.frombuffer(bytearray(raw[a:b]), dtype=torch.uint8).cuda()
            data, used, self.summary = _inflate_blocks(comp, rank + 1 == world, empty, True, True)
            if used != b - a:
                raise ValueError("a shard does not end at a member boundary")
            self.data = data
        if rank == 0:
            self.data = data[min(self.header.size, int(data.numel())) :]

    def decode(self, prev_tail: torch.Tensor, tags=("CB", "UB", "GN")) -> tuple[DecodedFile, torch.Tensor]:
        """The records of this shard (after the previous rank's tail) and this shard's own tail."""
        from cubam_b200.bam import RecordBatch

        data = torch.cat([prev_tail, self.data]) if prev_tail.numel() else self.data
        if self.summary is not None:
            check_inflate(self.summary)
        n = int(data.numel())
        if n == 0:
            off = torch.empty(0, dtype=torch.int64, device="cuda")
            tail = data
        else:
            offsets, cs = record_chain(data, len(self.header.names))
            s = read_struct(cs, _lib.ChainSummary)
            raise_status(s.status, "record chain")
            off = offsets[: s.n_records]
            tail = data[s.tail :].clone()
            if self.rank + 1 == self.world and int(tail.numel()):
                raise ValueError("truncated BAM file (incomplete record at the end)")
        b = RecordBatch.decode(data, off, self.header)
        tag_cols = {t: T for t, T in zip(tags, b.tags(*tags))} if tags and len(b) else {}
        if tags and not len(b):
            from cubam_b200.bam import Tag

            view = _View(data, off)
            z8 = torch.empty(0, dtype=torch.uint8, device="cuda")
            z64 = torch.empty(0, dtype=torch.int64, device="cuda")
            z32 = torch.empty(0, dtype=torch.int32, device="cuda")
            tag_cols = {t: Tag._from_columns(view, t, z8, z64, z32, z64) for t in tags}
        return DecodedFile(self.header, data, off, b.columns, tag_cols, 0, int(self.data.numel())), tail


def decode_sharded(path: str | Path, rank: int, world: int, group=None, tags=("CB", "UB", "GN")) -> DecodedFile:
    """This rank's records of ``path`` decoded by ``world`` ranks (each process one GPU), the tails
    passed along over ``torch.distributed`` (initialised by the caller; NCCL with device tensors)."""
    sh = Shard(path, rank, world)
    prev = recv_tail(rank, group)
    res, tail = sh.decode(prev, tags)
    send_tail(tail, rank, world, group)
    return res


def decode_shards_in_turn(path: str | Path, world: int, tags=("CB", "UB", "GN")) -> list[DecodedFile]:
    """All ranks' results computed one after another in this process (one GPU), the tails handed on
    directly: the sharded decode without a process group."""
    raw = Path(path).read_bytes()
    prev = torch.empty(0, dtype=torch.uint8, device="cuda")
    out = []
    for k in range(world):
        res, prev = Shard(path, k, world, raw).decode(prev, tags)
        out.append(res)
    return out
