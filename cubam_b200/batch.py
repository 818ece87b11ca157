"""Batched decoding of whole BAM files resident in GPU memory.

The plain reader (:func:`cubam_b200.read_bam`, as cubam's) works chunk by
chunk: scan, inflate, record chain and decode for each compressed chunk, with
host synchronisations in between.  This module is the batched form of the
same kernels for files whose compressed bytes are already on the device:

1. ``cb_scan_members`` runs on every file (launched back to back, one
   synchronisation for all of them) and gives each file's inflate jobs, with
   output offsets placed one file after another in one output arena;
2. ONE ``cb_inflate`` launch inflates the members of all files: a persistent
   grid whose warps take members from a work queue, so files of very uneven
   sizes share the GPU without a tail per file;
3. per file, ``cb_record_chain`` over the records area (header skipped), then
   the fixed columns and the requested tags in one aux walk.

The records and columns of a file equal the concatenation of the batches of
``read_bam`` over the same file (records never depend on the chunking; only
their split into batches does).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import torch

from cubam_b200 import _lib
from cubam_b200.bam import _TYPES, FIELDS, BamHeader, Tag
from cubam_b200.bgzf import ctypes_sizeof, raise_status, read_struct, stream_ptr

#: kernels launched by each entry point (for the launch count of a step)
KERNELS = {"scan": 4, "inflate": 3, "chain": 5, "decode": 1, "tags": 1}


@dataclass
class DecodedFile:
    """All records of one file: the records area of the inflated bytes, offsets, columns, tags."""

    header: BamHeader
    data: torch.Tensor
    offset: torch.Tensor
    columns: dict
    tags: dict = field(default_factory=dict)
    n_members: int = 0
    inflated_bytes: int = 0

    def __len__(self) -> int:
        return int(self.offset.numel())

    def __getattr__(self, name: str):
        cols = self.__dict__.get("columns")
        if cols is not None and name in cols:
            return cols[name]
        raise AttributeError(name)


@dataclass
class StageEvents:
    """CUDA events around the stages of one batched decode (recorded on the current stream)."""

    names: tuple = ("scan", "inflate", "chain", "decode")
    ev: dict = field(default_factory=dict)

    def mark(self, name: str) -> None:
        e = torch.cuda.Event(enable_timing=True)
        e.record()
        self.ev[name] = e

    def ms(self) -> dict:
        keys = [k for k in ("start", "scanned", "inflated", "chained", "decoded") if k in self.ev]
        out = {}
        for a, b in zip(keys, keys[1:]):
            out[b] = self.ev[a].elapsed_time(self.ev[b])
        return out


class _View:
    """Minimal batch view for :class:`~cubam_b200.bam.Tag` construction."""

    def __init__(self, data, offset):
        self.data, self.offset = data, offset

    def __len__(self):
        return int(self.offset.numel())


def decode_many(files: list[tuple[torch.Tensor, BamHeader]], tags=("CB", "UB", "GN"), check_crc: bool = True,
                events: StageEvents | None = None, counter: dict | None = None) -> list[DecodedFile]:
    """Decode whole files (compressed bytes on the device) with one inflate launch for all of them."""
    if events:
        events.mark("start")
    scans = []
    for comp, _ in files:
        n = int(comp.numel())
        ws = torch.empty(max(int(_lib.lib.cb_scan_workspace_bytes(n)), 256), dtype=torch.uint8, device="cuda")
        summ = torch.zeros(ctypes_sizeof(_lib.ScanSummary), dtype=torch.uint8, device="cuda")
        cap = n // 8192 + 1024
        jobs = torch.empty(cap * _lib.JOB_BYTES, dtype=torch.uint8, device="cuda")
        scans.append([comp, n, ws, summ, cap, jobs])
    # scans place their outputs one after another: the output base of file k is known only after
    # the sizes of files < k; launch with base 0 and shift the job offsets afterwards (one sync)
    for s in scans:
        comp, n, ws, summ, cap, jobs = s
        rc = _lib.lib.cb_scan_members(comp.data_ptr() if n else None, n, 1, 0, jobs.data_ptr(), cap,
                                      summ.data_ptr(), ws.data_ptr(), ws.numel(), stream_ptr())
        _lib.check(rc, "cb_scan_members")
        if counter is not None:
            counter["launches"] = counter.get("launches", 0) + KERNELS["scan"]
    summaries = torch.stack([s[3] for s in scans]).cpu().numpy()  # one sync for all files
    infos = [_lib.ScanSummary.from_buffer_copy(row.tobytes()) for row in summaries]
    for k, (s, info) in enumerate(zip(scans, infos)):
        if info.status == _lib.CAPACITY and info.n_jobs > s[4]:  # more members than the first guess: rescan
            comp, n, ws, summ, _, _ = s
            cap = int(info.n_jobs)
            jobs = torch.empty(cap * _lib.JOB_BYTES, dtype=torch.uint8, device="cuda")
            rc = _lib.lib.cb_scan_members(comp.data_ptr(), n, 1, 0, jobs.data_ptr(), cap, summ.data_ptr(),
                                          ws.data_ptr(), ws.numel(), stream_ptr())
            _lib.check(rc, "cb_scan_members")
            s[4], s[5] = cap, jobs
            infos[k] = read_struct(summ, _lib.ScanSummary)
        raise_status(infos[k].status, "BGZF member scan")
    total = sum(int(i.total_out) for i in infos)
    n_jobs = sum(int(i.n_jobs) for i in infos)
    out = torch.empty(max(total, 1), dtype=torch.uint8, device="cuda")
    job_lists, base = [], 0
    for s, info in zip(scans, infos):
        j = s[5][: int(info.n_jobs) * _lib.JOB_BYTES].view(torch.int64).view(-1, 4)
        if base:
            j = j.clone()
            j[:, 1] += base
        job_lists.append(j)
        base += int(info.total_out)
    all_jobs = torch.cat(job_lists) if len(job_lists) > 1 else job_lists[0]
    if events:
        events.mark("scanned")
    inflate_summ = torch.zeros(ctypes_sizeof(_lib.InflateSummary), dtype=torch.uint8, device="cuda")
    qws = torch.empty(256, dtype=torch.uint8, device="cuda")
    if n_jobs:
        rc = _lib.lib.cb_inflate(all_jobs.data_ptr(), n_jobs, None, out.data_ptr(), int(check_crc), None,
                                 inflate_summ.data_ptr(), qws.data_ptr(), qws.numel(), stream_ptr())
        _lib.check(rc, "cb_inflate")
        if counter is not None:
            counter["launches"] = counter.get("launches", 0) + KERNELS["inflate"]
    if events:
        events.mark("inflated")
    chains = []
    base = 0
    for (comp, header), info in zip(files, infos):
        data = out[base + header.size : base + int(info.total_out)]
        base += int(info.total_out)
        n = int(data.numel())
        cap = n // 37 + 2  # records are at least 37 bytes
        offsets = torch.empty(cap, dtype=torch.int64, device="cuda")
        csumm = torch.zeros(ctypes_sizeof(_lib.ChainSummary), dtype=torch.uint8, device="cuda")
        ws = torch.empty(max(int(_lib.lib.cb_record_chain_workspace_bytes(n)), 256), dtype=torch.uint8,
                         device="cuda")
        if n:
            rc = _lib.lib.cb_record_chain(data.data_ptr(), n, len(header.names), offsets.data_ptr(), cap,
                                          csumm.data_ptr(), ws.data_ptr(), ws.numel(), stream_ptr())
            _lib.check(rc, "cb_record_chain")
            if counter is not None:
                counter["launches"] = counter.get("launches", 0) + KERNELS["chain"]
        chains.append((data, offsets, csumm))
    if events:
        events.mark("chained")
    sums = torch.stack([c[2] for c in chains]).cpu().numpy()  # one sync for all files
    raise_status(read_struct(inflate_summ, _lib.InflateSummary).status, "inflate")
    results = []
    for (comp, header), info, (data, offsets, _), row in zip(files, infos, chains, sums):
        cs = _lib.ChainSummary.from_buffer_copy(row.tobytes())
        if int(data.numel()):
            raise_status(cs.status, "record chain")
            if cs.tail != int(data.numel()):
                raise ValueError("truncated BAM file (incomplete record at the end)")
        nrec = int(cs.n_records) if int(data.numel()) else 0
        off = offsets[:nrec]
        cols = {k: torch.empty(nrec, dtype=t, device="cuda") for k, t in _TYPES.items()}
        tag_cols = {}
        if nrec:
            rc = _lib.lib.cb_decode_fixed(data.data_ptr(), off.data_ptr(), nrec, *(cols[k].data_ptr() for k in FIELDS),
                                          stream_ptr())
            _lib.check(rc, "cb_decode_fixed")
            if tags:
                k = len(tags)
                ty = torch.empty((k, nrec), dtype=torch.uint8, device="cuda")
                vo = torch.empty((k, nrec), dtype=torch.int64, device="cuda")
                vl = torch.empty((k, nrec), dtype=torch.int32, device="cuda")
                iv = torch.empty((k, nrec), dtype=torch.int64, device="cuda")
                rc = _lib.lib.cb_find_tags(data.data_ptr(), off.data_ptr(), nrec, "".join(tags).encode(), k,
                                           ty.data_ptr(), vo.data_ptr(), vl.data_ptr(), iv.data_ptr(), stream_ptr())
                _lib.check(rc, "cb_find_tags")
                view = _View(data, off)
                for q, t in enumerate(tags):
                    tag_cols[t] = Tag._from_columns(view, t, ty[q], vo[q], vl[q], iv[q])
            if counter is not None:
                counter["launches"] = counter.get("launches", 0) + KERNELS["decode"] + (KERNELS["tags"] if tags else 0)
        results.append(DecodedFile(header, data, off, cols, tag_cols, int(info.n_members), int(info.total_out)))
    if events:
        events.mark("decoded")
    return results


def decode_resident(comp: torch.Tensor, header: BamHeader, **kw) -> DecodedFile:
    """One whole file (compressed bytes on the device): :func:`decode_many` of one."""
    return decode_many([(comp, header)], **kw)[0]


def load_compressed(path, device="cuda") -> torch.Tensor:
    """The bytes of a file, copied to the device through a pinned buffer."""
    import numpy as np

    raw = np.fromfile(path, dtype=np.uint8)
    host = torch.from_numpy(raw).pin_memory()
    return host.to(device, non_blocking=True)
