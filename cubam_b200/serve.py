"""Serving decode requests over resident BAM files: continuous batching on one GPU.

A request names a file and a range of BGZF virtual offsets (compressed member offset << 16 |
offset in the member's inflated bytes), and gets back the records that start in that range with
their fixed columns and tags, as a :class:`~cubam_b200.batch.DecodedFile`.  cubam reads files from
the start only and has no BAI or virtual-offset access (docs/reading.md:52-53); the member index
here is this project's own.

- :class:`ResidentFile`: a file's compressed bytes on the device plus its member index, built by
  one decode of the file: per member its compressed offset, inflated offset, the offset of the
  first record that starts in it, and the records that start before it.  Request boundaries are
  the virtual offsets of those first records (:meth:`ResidentFile.voff`), so every request's
  record count, inflated size and output layout are known on the host before it runs.
- :class:`Server`: requests arrive at any time (:meth:`Server.submit`); the loop admits them in
  arrival order while their bytes fit the HBM budget (inflated bytes in one pool tensor, plus
  offsets, columns and tags), splits each into slices of at most ``slice_bytes`` compressed
  bytes at member boundaries, and runs steps.  A step takes slices of many requests (the
  shortest remaining first, and always one of the oldest request's) up to ``step_bytes``: ONE
  inflate launch for all their members, a record chain per slice, and the columns and tags of
  the requests whose last slice ran.  While a step runs the host admits arrivals and plans the
  next step, so requests that arrive while others are on the GPU join at the next step.
- :func:`decode_alone`: one request decoded by itself (one inflate launch for its members, one
  chain, columns, tags, then a sync): the plain sequential form.

The bytes of a request's records are the same in every form: a slice starts and ends at a
record boundary that the index gives, and its members land at their offsets in the request's
output region.
"""

from __future__ import annotations

import bisect
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from cubam_b200 import _lib
from cubam_b200.bam import _TYPES, FIELDS, BamHeader, Tag
from cubam_b200.batch import DecodedFile, _View, decode_many
from cubam_b200.bgzf import (
    ctypes_sizeof,
    inflate_workspace_bytes,
    launch_inflate,
    raise_status,
    read_struct,
    scan_members,
    stream_ptr,
)

#: device bytes per record besides the inflated bytes: offset, 11 columns, 21 bytes per tag
RECORD_BYTES = 8 + 43


def record_bytes(n_tags: int) -> int:
    return RECORD_BYTES + 21 * n_tags


# ---------------------------------------------------------------------------------------------- index


@dataclass
class MemberIndex:
    """Per member m of the members with data (M of them; entry M stands for the end of the file)."""

    coff: np.ndarray  # compressed offset of member m in the file, int64 (M + 1)
    ucum: np.ndarray  # offset of member m's first byte in the file's inflated bytes (M + 1)
    first_rec: np.ndarray  # offset in member m of the first record starting in it, -1 if none (M + 1)
    cum_rec: np.ndarray  # records starting before member m (M + 1)
    jobs: np.ndarray  # the scan's job rows (M, 4) int64: in pointer, out_off, in_len | isize << 32, crc

    @property
    def n_members(self) -> int:
        return len(self.coff) - 1


class ResidentFile:
    """A BAM file's compressed bytes on the device and its member index."""

    def __init__(self, comp: torch.Tensor, header: BamHeader):
        self.comp = comp
        self.header = header
        self.index = self._build_index()

    @classmethod
    def load(cls, path) -> ResidentFile:
        from cubam_b200.batch import load_compressed

        return cls(load_compressed(path), BamHeader.read(path))

    def _build_index(self) -> MemberIndex:
        comp = self.comp
        jobs, s = scan_members(comp, True)
        raise_status(s.status, "BGZF member scan")
        M = int(s.n_jobs)
        rows = jobs[: M * _lib.JOB_BYTES].view(torch.int64).view(M, 4).cpu().numpy().copy()
        base = comp.data_ptr()
        coff = np.empty(M + 1, np.int64)
        coff[:M] = rows[:, 0] - base - 18
        coff[M] = coff[M - 1] + (rows[M - 1, 2] & 0xFFFFFFFF) + 26 if M else 0  # just past the last member
        ucum = np.empty(M + 1, np.int64)
        ucum[:M] = rows[:, 1]
        ucum[M] = int(s.total_out)
        d = decode_many([(comp, self.header)], tags=())[0]
        starts = d.offset + self.header.size  # record starts in the file's inflated bytes
        uc = torch.from_numpy(ucum).to(comp.device)
        m = torch.searchsorted(uc, starts, right=True) - 1
        first = torch.full((M + 1,), -1, dtype=torch.int64, device=comp.device)
        first.scatter_reduce_(0, m, starts - uc[m], reduce="amin", include_self=False)
        counts = torch.bincount(m, minlength=M + 1)
        first = first.cpu().numpy()
        first[M] = 0
        cum = np.zeros(M + 1, np.int64)
        cum[1:] = np.cumsum(counts.cpu().numpy()[:M])
        del d
        return MemberIndex(coff, ucum, first, cum, rows)

    @property
    def n_members(self) -> int:
        return self.index.n_members

    def boundaries(self) -> np.ndarray:
        """Members where a request may start or end (a record starts in them, or the end)."""
        return np.flatnonzero(self.index.first_rec >= 0)

    def voff(self, m: int) -> int:
        """Virtual offset of the first record that starts in member m (m = n_members: the end)."""
        fr = int(self.index.first_rec[m])
        if fr < 0:
            raise ValueError(f"no record starts in member {m}")
        return (int(self.index.coff[m]) << 16) | fr

    def member_of(self, voff: int) -> int:
        """The member of a virtual offset that :meth:`voff` gives; ValueError for any other."""
        c, u = voff >> 16, voff & 0xFFFF
        m = int(np.searchsorted(self.index.coff, c))
        if m > self.n_members or int(self.index.coff[m]) != c or int(self.index.first_rec[m]) != u:
            raise ValueError(f"virtual offset {voff:#x} is not the start of a member's first record")
        return m


# ---------------------------------------------------------------------------------------------- requests


@dataclass
class Request:
    file: int
    voff_begin: int
    voff_end: int
    arrival: float = 0.0  # host seconds (time.perf_counter) when it arrives
    rid: int = 0
    # set by the server
    m0: int = 0
    m1: int = 0
    done: float | None = None
    result: DecodedFile | None = None
    status: int = 0  # CB_OK, or CB_ERR_TIMEOUT when its deadline passed before it was served
    error: Exception | None = None
    compressed_bytes: int = 0
    inflated_bytes: int = 0
    n_records: int = 0
    _region: int = -1
    _region_size: int = 0
    _slices: list = field(default_factory=list)
    _next: int = 0
    _last_launched: bool = False
    _off: torch.Tensor | None = None
    _inflight: int = 0  # queued steps holding slices of it
    _cancelled: bool = False


def plan_request(rf: ResidentFile, req: Request) -> None:
    """Members, sizes and records of a request from the index (host only)."""
    ix = rf.index
    req.m0 = rf.member_of(req.voff_begin)
    req.m1 = rf.member_of(req.voff_end)
    if req.m1 < req.m0:
        raise ValueError("request range ends before it begins")
    req.compressed_bytes = int(ix.coff[req.m1] - ix.coff[req.m0])
    req.n_records = int(ix.cum_rec[req.m1] - ix.cum_rec[req.m0])
    req.inflated_bytes = int(ix.ucum[req.m1] - ix.ucum[req.m0]) + int(ix.first_rec[req.m1]) - int(ix.first_rec[req.m0])
    # region: members m0 .. m1 (m1 only when the last record runs into it)
    last = req.m1 if (req.m1 < rf.n_members and int(ix.first_rec[req.m1]) > 0) else req.m1 - 1
    req._region_size = int(ix.ucum[last + 1] - ix.ucum[req.m0]) if last >= req.m0 else 0


def slice_request(rf: ResidentFile, req: Request, slice_bytes: int) -> list[tuple[int, int]]:
    """Member ranges [ma, mb) covering [m0, m1), cut where a record starts: each the longest of at most
    ``slice_bytes`` compressed bytes, or the shortest possible when none is that short."""
    ix = rf.index
    ok = rf.boundaries()
    out = []
    ma = req.m0
    while ma < req.m1:
        lo = int(np.searchsorted(ok, ma, side="right"))
        hi = int(np.searchsorted(ok, req.m1, side="right"))
        cands = ok[lo:hi]  # boundaries in (ma, m1]; m1 is one
        k = int(np.searchsorted(ix.coff[cands], int(ix.coff[ma]) + slice_bytes, side="right")) - 1
        mb = int(cands[max(k, 0)])
        out.append((ma, mb))
        ma = mb
    return out


class PoolAllocator:
    """First-fit ranges of one device pool (offsets aligned to 256 bytes)."""

    def __init__(self, size: int):
        self.size = int(size)
        self.free = [(0, self.size)]  # sorted, coalesced (start, end)

    def alloc(self, n: int) -> int | None:
        n = max((int(n) + 255) & ~255, 256)
        for i, (a, b) in enumerate(self.free):
            if b - a >= n:
                if b - a == n:
                    self.free.pop(i)
                else:
                    self.free[i] = (a + n, b)
                return a
        return None

    def release(self, off: int, n: int) -> None:
        n = max((int(n) + 255) & ~255, 256)
        a, b = off, off + n
        i = bisect.bisect_left(self.free, (a, b))
        self.free.insert(i, (a, b))
        merged = []
        for x, y in self.free:
            if merged and merged[-1][1] >= x:
                merged[-1] = (merged[-1][0], max(merged[-1][1], y))
            else:
                merged.append((x, y))
        self.free = merged

    def available(self) -> int:
        return sum(b - a for a, b in self.free)


# ---------------------------------------------------------------------------------------------- device work


def _job_rows(rf: ResidentFile, ma: int, mb_incl: int, dst: int, m0: int) -> np.ndarray:
    """Job rows of members [ma, mb_incl] writing at dst + (their inflated offset - member m0's)."""
    rows = rf.index.jobs[ma : mb_incl + 1].copy()
    rows[:, 1] = dst + (rf.index.ucum[ma : mb_incl + 1] - rf.index.ucum[m0])
    return rows


class _Scratch:
    """Growing device buffers reused from step to step (one stream: steps never overlap)."""

    def __init__(self):
        self.bufs = {}

    def get(self, name: str, nbytes: int) -> torch.Tensor:
        b = self.bufs.get(name)
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(int(nbytes * 1.25), 256), dtype=torch.uint8, device="cuda")
            self.bufs[name] = b
        return b

    def host(self, name: str, nbytes: int) -> torch.Tensor:
        """A pinned host buffer (the step that last used it has completed before it is reused)."""
        b = self.bufs.get(name)
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(int(nbytes * 1.25), 256), dtype=torch.uint8, pin_memory=True)
            self.bufs[name] = b
        return b


def _finish_request(req: Request, rf: ResidentFile, data: torch.Tensor, off: torch.Tensor, tags, s) -> DecodedFile:
    """Columns and tags of a request whose records are all chained (launches only)."""
    n = req.n_records
    cols = {k: torch.empty(n, dtype=t, device="cuda") for k, t in _TYPES.items()}
    tag_cols = {}
    if n:
        rc = _lib.lib.cb_decode_fixed(data.data_ptr(), off.data_ptr(), n, *(cols[f].data_ptr() for f in FIELDS), s)
        _lib.check(rc, "cb_decode_fixed")
    if tags:  # tag columns exist (empty) for a request without records too
        k = len(tags)
        ty = torch.empty((k, n), dtype=torch.uint8, device="cuda")
        vo = torch.empty((k, n), dtype=torch.int64, device="cuda")
        vl = torch.empty((k, n), dtype=torch.int32, device="cuda")
        iv = torch.empty((k, n), dtype=torch.int64, device="cuda")
        if n:
            rc = _lib.lib.cb_find_tags(data.data_ptr(), off.data_ptr(), n, "".join(tags).encode(), k, ty.data_ptr(),
                                       vo.data_ptr(), vl.data_ptr(), iv.data_ptr(), s)
            _lib.check(rc, "cb_find_tags")
        view = _View(data, off)
        for q, t in enumerate(tags):
            tag_cols[t] = Tag._from_columns(view, t, ty[q], vo[q], vl[q], iv[q])
    return DecodedFile(rf.header, data, off, cols, tag_cols, req.m1 - req.m0, req.inflated_bytes)


def decode_alone(rf: ResidentFile, req: Request, tags=("CB", "UB", "GN"), check_crc: bool = True) -> DecodedFile:
    """One request by itself: one inflate launch for its members, one record chain, columns and tags,
    then one synchronisation (the plain sequential form)."""
    plan_request(rf, req)
    ix = rf.index
    region = torch.empty(max(req._region_size, 1), dtype=torch.uint8, device="cuda")
    last = req.m1 if (req.m1 < rf.n_members and int(ix.first_rec[req.m1]) > 0) else req.m1 - 1
    s = stream_ptr()
    summ = torch.zeros(ctypes_sizeof(_lib.InflateSummary), dtype=torch.uint8, device="cuda")
    if req._region_size:
        rows = _job_rows(rf, req.m0, last, 0, req.m0)
        jobs = torch.from_numpy(rows).cuda()
        qws = torch.empty(inflate_workspace_bytes(len(rows), req._region_size), dtype=torch.uint8, device="cuda")
        launch_inflate(jobs.data_ptr(), len(rows), region.data_ptr(), req._region_size, check_crc, summ.data_ptr(),
                       qws)
    start = int(ix.first_rec[req.m0])
    data = region[start : start + req.inflated_bytes]
    off = torch.empty(max(req.n_records, 1), dtype=torch.int64, device="cuda")
    csumm = torch.zeros(ctypes_sizeof(_lib.ChainSummary), dtype=torch.uint8, device="cuda")
    n = req.inflated_bytes
    if n:
        ws = torch.empty(max(int(_lib.lib.cb_record_chain_workspace_bytes(n)), 256), dtype=torch.uint8,
                         device="cuda")
        rc = _lib.lib.cb_record_chain(data.data_ptr(), n, len(rf.header.names), off.data_ptr(), max(req.n_records, 1),
                                      csumm.data_ptr(), ws.data_ptr(), ws.numel(), s)
        _lib.check(rc, "cb_record_chain")
    res = _finish_request(req, rf, data, off[: req.n_records], tags, s)
    if req._region_size:
        raise_status(read_struct(summ, _lib.InflateSummary).status, "inflate")
    if n:
        cs = read_struct(csumm, _lib.ChainSummary)
        raise_status(cs.status, "record chain")
        if int(cs.n_records) != req.n_records or int(cs.tail) != n:
            raise RuntimeError("the record chain of the request differs from the index")
    return res


@dataclass
class _Slice:
    req: Request
    ma: int
    mb: int
    last: bool  # the request's last slice


class Server:
    """Continuous batching of decode requests (see the module docstring).

    ``budget_bytes`` is the HBM the in-flight requests may hold: the pool for their inflated bytes
    is ``pool_frac`` of it, the rest bounds their offsets, columns and tags.  A step holds up to
    ``step_bytes`` compressed bytes, or ``short_step_bytes`` while a request of at most
    ``small_bytes`` waits to start: shorter steps for a small request's latency, longer ones for
    throughput.

    ``request_timeout`` (seconds after arrival, None for none) bounds how long a request may wait: when
    it passes, a request not yet admitted or not yet started is dropped at once, and a started one gets
    no further slices and gives its memory back once the steps already queued with it are done.  Either
    way it finishes with ``status`` CB_ERR_TIMEOUT, ``error`` a TimeoutError and no result.
    """

    def __init__(self, files: list[ResidentFile], budget_bytes: int = 40 << 30, step_bytes: int = 1 << 30,
                 slice_bytes: int = 48 << 20, tags=("CB", "UB", "GN"), check_crc: bool = True,
                 pool_frac: float = 0.7, short_step_bytes: int = 128 << 20, small_bytes: int = 8 << 20,
                 request_timeout: float | None = None):
        self.files = files
        self.request_timeout = request_timeout
        self.timed_out = 0
        self.tags = tuple(tags)
        self.check_crc = check_crc
        self.long_step_bytes = int(step_bytes)
        self.short_step_bytes = min(int(short_step_bytes), int(step_bytes))
        self.small_bytes = int(small_bytes)
        self.step_bytes = int(step_bytes)
        self.slice_bytes = int(slice_bytes)
        self.pool_bytes = int(budget_bytes * pool_frac) & ~255
        self.side_budget = int(budget_bytes) - self.pool_bytes
        self.pool = torch.empty(self.pool_bytes, dtype=torch.uint8, device="cuda")
        self.alloc = PoolAllocator(self.pool_bytes)
        self.side_used = 0
        self.pending: list[Request] = []  # arrived, not admitted (arrival order)
        self.active: list[Request] = []  # admitted, slices left
        self.finished: list[Request] = []
        self.scratch = (_Scratch(), _Scratch())
        self.steps = 0
        self.step_log = []
        self.host_s = {"plan": 0.0, "launch": 0.0, "wait": 0.0, "complete": 0.0}  # host seconds per loop phase
        self.gpu_ms = 0.0  # device time of the steps (first to last kernel of each)

    # -------------------------------------------------------------- admission and planning
    def submit(self, req: Request) -> None:
        plan_request(self.files[req.file], req)
        side = req.n_records * record_bytes(len(self.tags))
        if max(req._region_size, 1) > self.pool_bytes or side > self.side_budget:
            raise ValueError("request larger than the HBM budget")
        self.pending.append(req)

    def _admit(self) -> None:
        while self.pending:
            req = self.pending[0]
            side = req.n_records * record_bytes(len(self.tags))
            if self.side_used + side > self.side_budget:
                return
            off = self.alloc.alloc(max(req._region_size, 1))
            if off is None:
                return
            self.pending.pop(0)
            req._region = off
            self.side_used += side
            req._slices = slice_request(self.files[req.file], req, self.slice_bytes)
            req._next = 0
            req._off = torch.empty(max(req.n_records, 1), dtype=torch.int64, device="cuda")
            self.active.append(req)

    def _pick(self) -> list[_Slice]:
        """The slices of the next step: one of the oldest request's, then the shortest remaining first."""
        if not self.active:
            return []

        def remaining(r):
            ix = self.files[r.file].index
            return int(ix.coff[r.m1]) - (int(ix.coff[r._slices[r._next][0]]) if r._next < len(r._slices) else 0)

        ready = [r for r in self.active if not r._last_launched and not r._cancelled]
        if not ready:
            return []
        small_waiting = any(r.compressed_bytes <= self.small_bytes and r._next == 0 for r in ready) or any(
            r.compressed_bytes <= self.small_bytes for r in self.pending)
        self.step_bytes = self.short_step_bytes if small_waiting else self.long_step_bytes
        order = [ready[0]] + sorted(ready[1:], key=remaining)
        out, total = [], 0
        for r in order:
            if not r._slices:  # an empty range: finishes in this step
                out.append(_Slice(r, r.m0, r.m0, True))
                r._last_launched = True
                continue
            # consecutive slices of the request while the step has room, as one member range
            coff = self.files[r.file].index.coff
            ma, mb = r._slices[r._next]
            b = int(coff[mb] - coff[ma])
            if out and total + b > self.step_bytes:
                continue
            k = r._next + 1
            while k < len(r._slices):
                nb = int(coff[r._slices[k][1]] - coff[ma])
                if total + nb > self.step_bytes:
                    break
                mb, b = r._slices[k][1], nb
                k += 1
            last = k == len(r._slices)
            out.append(_Slice(r, ma, mb, last))
            r._next = k
            r._last_launched = last
            total += b
        return out

    # -------------------------------------------------------------- one step
    def _launch(self, slices: list[_Slice]):
        ev0 = torch.cuda.Event(enable_timing=True)
        ev0.record()
        s = stream_ptr()
        scratch = self.scratch[self.steps % 2]  # the step before may still be read back by the host
        rows = []
        for sl in slices:
            sl.req._inflight += 1
        for sl in slices:
            r, rf = sl.req, self.files[sl.req.file]
            ix = rf.index
            if sl.mb > sl.ma:
                last = sl.mb if (sl.mb < rf.n_members and int(ix.first_rec[sl.mb]) > 0) else sl.mb - 1
                rows.append(_job_rows(rf, sl.ma, last, r._region, r.m0))
        n_jobs = sum(len(x) for x in rows)
        summ = scratch.get("isumm", ctypes_sizeof(_lib.InflateSummary))
        if n_jobs:
            table = np.concatenate(rows)
            nb = table.nbytes
            host = scratch.host("jobs_host", nb)  # pinned, reused: the step that last used it is done
            host[:nb].numpy()[:] = table.view(np.uint8).reshape(-1)
            jobs = scratch.get("jobs", nb)
            jobs[:nb].copy_(host[:nb], non_blocking=True)
            out_bytes = int(sum(int((x[:, 2] >> 32).sum()) for x in rows))  # sum of ISIZE (high half of word 2)
            qws = scratch.get("queue", inflate_workspace_bytes(n_jobs, out_bytes))
            launch_inflate(jobs.data_ptr(), n_jobs, self.pool.data_ptr(), out_bytes, self.check_crc, summ.data_ptr(),
                           qws)
        csz = ctypes_sizeof(_lib.ChainSummary)
        csumm = scratch.get("csumm", csz * max(len(slices), 1))
        csumm[: csz * max(len(slices), 1)].zero_()
        checks = []
        done = []
        for k, sl in enumerate(slices):
            r, rf = sl.req, self.files[sl.req.file]
            ix = rf.index
            r_start = r._region + int(ix.first_rec[r.m0])  # the request's records in the pool
            if sl.mb > sl.ma:
                a = r._region + int(ix.ucum[sl.ma] - ix.ucum[r.m0]) + int(ix.first_rec[sl.ma])
                n = int(ix.ucum[sl.mb] - ix.ucum[sl.ma]) + int(ix.first_rec[sl.mb]) - int(ix.first_rec[sl.ma])
                nrec = int(ix.cum_rec[sl.mb] - ix.cum_rec[sl.ma])
                rec0 = int(ix.cum_rec[sl.ma] - ix.cum_rec[r.m0])
                if n:
                    ws = scratch.get("chain_ws", int(_lib.lib.cb_record_chain_workspace_bytes(n)))
                    off = r._off[rec0 : rec0 + max(nrec, 1)]
                    rc = _lib.lib.cb_record_chain(self.pool.data_ptr() + a, n, len(rf.header.names), off.data_ptr(),
                                                  max(nrec, 1), csumm.data_ptr() + k * csz, ws.data_ptr(), ws.numel(),
                                                  s)
                    _lib.check(rc, "cb_record_chain")
                    if nrec and a != r_start:
                        r._off[rec0 : rec0 + nrec].add_(a - r_start)
                    checks.append((k, nrec, n))
            if sl.last:
                data = self.pool[r_start : r_start + r.inflated_bytes]
                r.result = _finish_request(r, rf, data, r._off[: r.n_records], self.tags, s)
                done.append(r)
        # the step's summaries go to pinned host memory behind its kernels: reading them needs only the
        # step's event, not a copy that would also wait for the step queued after it
        isz = ctypes_sizeof(_lib.InflateSummary)
        ncs = csz * max(len(slices), 1)
        host = scratch.host("summaries", isz + ncs)
        host[:isz].copy_(summ[:isz], non_blocking=True)
        host[isz : isz + ncs].copy_(csumm[:ncs], non_blocking=True)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record()
        return ev, n_jobs, checks, done, host[:isz], host[isz : isz + ncs], ev0, [sl.req for sl in slices]

    def _check(self, n_jobs, checks, summ, csumm) -> None:
        """Statuses of a completed step from its summaries in pinned host memory."""
        if n_jobs:
            raise_status(_lib.InflateSummary.from_buffer_copy(summ.numpy().tobytes()).status, "inflate")
        if checks:
            csz = ctypes_sizeof(_lib.ChainSummary)
            raw = csumm[: csz * (max(k for k, _, _ in checks) + 1)].numpy()
            for k, nrec, n in checks:
                cs = _lib.ChainSummary.from_buffer_copy(raw[k * csz : (k + 1) * csz].tobytes())
                raise_status(cs.status, "record chain")
                if int(cs.n_records) != nrec or int(cs.tail) != n:
                    raise RuntimeError("a slice's record chain differs from the index")

    def release(self, req: Request) -> None:
        """Give a finished request's device memory back (its result must no longer be used)."""
        if req._region >= 0:
            self._free(req)
            req.result = None

    def _expire(self, now: float, finish) -> None:
        """Apply ``request_timeout`` at host time ``now`` (seconds since the loop's t0)."""
        if self.request_timeout is None:
            return
        late = [r for r in self.pending if now - r.arrival > self.request_timeout]
        for r in late:
            self.pending.remove(r)
            finish(r)
        for r in [r for r in self.active if not r._cancelled and now - r.arrival > self.request_timeout]:
            if r._last_launched:  # its last slice is queued: it is served
                continue
            r._cancelled = True
            if r._inflight == 0:
                self.active.remove(r)
                self._free(r)
                finish(r)

    def _time_out(self, r: Request, now: float) -> None:
        r.done = now
        r.status = _lib.TIMEOUT
        r.error = TimeoutError(f"request {r.rid} not served within {self.request_timeout} s of its arrival")
        r.result = None
        self.timed_out += 1

    def _free(self, r: Request) -> None:
        if r._region >= 0:
            self.alloc.release(r._region, max(r._region_size, 1))
            r._region = -1
            self.side_used -= r.n_records * record_bytes(len(self.tags))
            r._off = None

    # -------------------------------------------------------------- the loop
    def run(self, requests: list[Request], on_done=None, t0: float | None = None) -> list[Request]:
        """Serve ``requests``, each arriving at ``t0 + arrival`` (host seconds).  ``on_done(req)`` is called
        when a request's result is ready; the request is then released unless ``on_done`` returns False.

        At most two steps are queued on the stream: while one runs, the next is already launched and
        the host admits arrivals and plans the one after."""
        incoming = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter() if t0 is None else t0
        i = 0
        inflight = []
        finished = []

        def arrivals():
            nonlocal i
            now = time.perf_counter() - t0
            while i < len(incoming) and incoming[i].arrival <= now:
                self.submit(incoming[i])
                i += 1

        def timed_out(r):
            self._time_out(r, time.perf_counter() - t0)
            finished.append(r)
            if on_done:
                on_done(r)

        def complete(step):
            ev, n_jobs, checks, done, summ, csumm, _, touched = step
            now = time.perf_counter() - t0
            self._check(n_jobs, checks, summ, csumm)
            for r in touched:
                r._inflight -= 1
            for r in done:
                r.done = now
                self.active.remove(r)
                finished.append(r)
                keep = on_done(r) if on_done else None
                if keep is not False:
                    self.release(r)
            for r in {id(r): r for r in touched}.values():  # cancelled: free once no queued step holds it
                if r._cancelled and r._inflight == 0 and r in self.active:
                    self.active.remove(r)
                    self._free(r)
                    timed_out(r)

        clock = time.perf_counter
        while i < len(incoming) or self.pending or self.active or inflight:
            ta = clock()
            arrivals()
            self._expire(clock() - t0, timed_out)
            self._admit()
            launched = False
            if len(inflight) < 2:
                nxt = self._pick()
                tb = clock()
                self.host_s["plan"] += tb - ta
                if nxt:
                    inflight.append(self._launch(nxt))
                    self.steps += 1
                    self.step_log.append((len(nxt), inflight[-1][1]))
                    launched = True
                self.host_s["launch"] += clock() - tb
            if inflight and (len(inflight) == 2 or not launched):
                if len(inflight) == 2 or inflight[0][0].query():
                    tc = clock()
                    inflight[0][0].synchronize()
                    td = clock()
                    self.host_s["wait"] += td - tc
                    step = inflight.pop(0)
                    self.gpu_ms += step[6].elapsed_time(step[0])
                    complete(step)
                    self.host_s["complete"] += clock() - td
                else:
                    time.sleep(0.0002)
            elif not inflight and not launched and i < len(incoming):
                time.sleep(max(0.0, min(0.0005, incoming[i].arrival - (time.perf_counter() - t0))))
        return finished


def poisson_requests(files: list[ResidentFile], n: int, rate: float, seed: int = 4, min_bytes: int = 64 << 10,
                     max_bytes: int = 512 << 20) -> list[Request]:
    """Requests with sizes log-uniform in [min_bytes, max_bytes] of compressed data (capped by the file),
    over files at random, arriving as a Poisson stream of ``rate`` per second."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for k in range(n):
        t += float(rng.exponential(1.0 / rate))
        f = int(rng.integers(len(files)))
        rf = files[f]
        ok = rf.boundaries()
        size = float(np.exp(rng.uniform(np.log(min_bytes), np.log(max_bytes))))
        a = int(ok[int(rng.integers(len(ok)))])
        target = int(rf.index.coff[a]) + size
        j = int(np.searchsorted(rf.index.coff[ok], target))
        b = int(ok[min(max(j, 0), len(ok) - 1)])
        if b <= a:
            b = int(ok[min(int(np.searchsorted(ok, a, side="right")), len(ok) - 1)])
        if b <= a:  # a at the end: take the range that ends there
            a, b = int(ok[max(0, len(ok) - 2)]), int(ok[-1])
        out.append(Request(f, rf.voff(a), rf.voff(b), arrival=t, rid=k))
    return out


def latency_summary(reqs: list[Request], small_bytes: int = 8 << 20) -> dict:
    lat = np.array([(r.done - r.arrival) * 1e3 for r in reqs if r.done is not None])
    small = np.array([(r.done - r.arrival) * 1e3 for r in reqs if r.done is not None and r.compressed_bytes <= small_bytes])

    def pct(a):
        if not len(a):
            return None
        return {"p50": float(np.percentile(a, 50)), "p95": float(np.percentile(a, 95)),
                "p99": float(np.percentile(a, 99)), "n": int(len(a))}

    return {"all_ms": pct(lat), "small_ms": pct(small)}
