"""Batched decoding of whole BAM files resident in GPU memory.

The plain reader (:func:`cubam_b200.read_bam`, as cubam's) works chunk by
chunk: scan, inflate, record chain and decode for each compressed chunk, with
host synchronisations in between.  This module is the batched form of the
same kernels for files whose compressed bytes are already on the device:

1. ``cb_scan_members`` runs on every file (launched back to back, one
   synchronisation for all of them) and gives each file's inflate jobs, with
   output offsets placed one file after another in one output arena;
2. ONE ``cb_inflate`` call inflates the members of all files: persistent
   grids whose lanes (decode) and warps (copy) take members from work queues,
   so files of very uneven sizes share the GPU without a tail per file;
3. per file, ``cb_record_chain`` over the records area (header skipped), then
   one record pass (``cb_decode_columns``) for the fixed columns and the
   requested tags.

The records and columns of a file equal the concatenation of the batches of
``read_bam`` over the same file (records never depend on the chunking; only
their split into batches does).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import torch

from cubam_b200 import _lib, _trace
from cubam_b200.bam import _TYPES, FIELDS, BamHeader, Tag
from cubam_b200.bgzf import (
    ctypes_sizeof,
    inflate_form,
    inflate_workspace_bytes,
    launch_inflate,
    raise_status,
    read_struct,
    stream_ptr,
)

#: kernels launched by each entry point (for the launch count of a step)
KERNELS = {"scan": 4, "inflate": 3, "chain": 9, "records": 1}


def _tag_arrays(k: int, nrec: int):
    """Tag-major type, value offset, value length and integer value arrays of k tags (device)."""
    if not k:
        return ()
    return (torch.empty((k, nrec), dtype=torch.uint8, device="cuda"),
            torch.empty((k, nrec), dtype=torch.int64, device="cuda"),
            torch.empty((k, nrec), dtype=torch.int32, device="cuda"),
            torch.empty((k, nrec), dtype=torch.int64, device="cuda"))


def inflate_launches(form: int = 0, n_jobs: int | None = None) -> int:
    """Kernels of one inflate call: init, the persistent grid, finish; form 3 adds the slot scan and
    splits the grid into decode and copy."""
    return 5 if inflate_form(form, n_jobs) == 3 else KERNELS["inflate"]


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
                events: StageEvents | None = None, counter: dict | None = None,
                derived: bool = False) -> list[DecodedFile]:
    """Decode whole files (compressed bytes on the device) with one inflate launch for all of them.

    With ``derived`` the columns also hold ``aligned_length`` and ``name_hash``, computed in the
    same pass over the records as the fixed fields."""
    _trace.mark(events, "start")
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
    _trace.mark(events, "scanned")
    inflate_summ = torch.zeros(ctypes_sizeof(_lib.InflateSummary), dtype=torch.uint8, device="cuda")
    if n_jobs:
        qws = torch.empty(inflate_workspace_bytes(n_jobs, total), dtype=torch.uint8, device="cuda")
        launch_inflate(all_jobs.data_ptr(), n_jobs, out.data_ptr(), total, check_crc, inflate_summ.data_ptr(), qws)
        del qws
        if counter is not None:
            counter["launches"] = counter.get("launches", 0) + inflate_launches(0, n_jobs)
    _trace.mark(events, "inflated")
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
    _trace.mark(events, "chained")
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
        if derived:
            cols["aligned_length"] = torch.empty(nrec, dtype=torch.int32, device="cuda")
            cols["name_hash"] = torch.empty(nrec, dtype=torch.uint64, device="cuda")
        tag_cols = {}
        if nrec:
            # columns, derived columns and tags in one record pass
            k = len(tags)
            arrs = _tag_arrays(k, nrec)
            rc = _lib.lib.cb_decode_columns(
                data.data_ptr(), off.data_ptr(), nrec, *(cols[f].data_ptr() for f in FIELDS),
                cols["aligned_length"].data_ptr() if derived else None, cols["name_hash"].data_ptr() if derived else None,
                None, None, "".join(tags).encode(), k, *((a.data_ptr() for a in arrs) if k else (None,) * 4), stream_ptr())
            _lib.check(rc, "cb_decode_columns")
            if k:
                view = _View(data, off)
                for q, t in enumerate(tags):
                    tag_cols[t] = Tag._from_columns(view, t, *(a[q] for a in arrs))
            if counter is not None:
                counter["launches"] = counter.get("launches", 0) + KERNELS["records"]
        results.append(DecodedFile(header, data, off, cols, tag_cols, int(info.n_members), int(info.total_out)))
    _trace.mark(events, "decoded")
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


class BatchPlan:
    """A fixed set of resident files decoded by one launch sequence with no host synchronisation.

    The first decode (:func:`decode_many`) sizes everything: each file's jobs, inflated bytes and
    records.  The plan then owns every buffer (one job table and one output arena for all files,
    per-file offsets, columns and tag columns, shared scan and chain workspaces) and
    :meth:`launch` issues, on the current stream, the scans (each writing its jobs straight into
    its slice of the job table, with its output base), ONE inflate launch for the members of all
    files, the record chains, and the columns and tags.  Because nothing in it waits for the
    host, :meth:`capture` records it as a CUDA graph and :meth:`replay` re-runs the whole batch
    with one launch; :meth:`check` reads every device summary with one copy and raises on a
    status or on counts that differ from the plan.

    ``form`` is the inflate form (1: a member per warp, 2: a member per lane, 3: decode per lane and
    copy per warp); None lets :meth:`autotune` choose it, with the other launch parameters, by timing
    this batch (or from the tuning cache for a batch of the same shape on the same device).
    """

    def __init__(self, files: list[tuple[torch.Tensor, BamHeader]], tags=("CB", "UB", "GN"), check_crc: bool = True,
                 form: int | None = None):
        self.files = files
        self.tags = tuple(tags)
        self.check_crc = check_crc
        first = decode_many(files, tags=tags, check_crc=check_crc)
        self.n_files = len(files)
        self.n_members = [d.n_members for d in first]
        self.inflated = [d.inflated_bytes for d in first]
        self.n_records = [len(d) for d in first]
        del first  # its buffers go back to the allocator before the plan takes its own
        # jobs per file (members with ISIZE > 0): from a scan summary of the first pass
        self.n_jobs = []
        self.out_base = []
        base = 0
        for (comp, _), total in zip(files, self.inflated):
            self.out_base.append(base)
            base += total
        self.total_out = base
        dev = "cuda"
        sizes = [int(c.numel()) for c, _ in files]
        self.scan_ws = torch.empty(max([int(_lib.lib.cb_scan_workspace_bytes(n)) for n in sizes] + [256]),
                                   dtype=torch.uint8, device=dev)
        ssz = ctypes_sizeof(_lib.ScanSummary)
        self.scan_summ = torch.zeros((self.n_files, ssz), dtype=torch.uint8, device=dev)
        # count the jobs of each file with one scan pass (a cap-0 scan reports n_jobs)
        probe = torch.empty(_lib.JOB_BYTES, dtype=torch.uint8, device=dev)
        for k, ((comp, _), n) in enumerate(zip(files, sizes)):
            rc = _lib.lib.cb_scan_members(comp.data_ptr() if n else None, n, 1, 0, probe.data_ptr(), 0,
                                          self.scan_summ[k].data_ptr(), self.scan_ws.data_ptr(),
                                          self.scan_ws.numel(), stream_ptr())
            _lib.check(rc, "cb_scan_members")
        infos = [_lib.ScanSummary.from_buffer_copy(r.tobytes()) for r in self.scan_summ.cpu().numpy()]
        self.n_jobs = [int(i.n_jobs) for i in infos]
        self.job_base = [0]
        for nj in self.n_jobs:
            self.job_base.append(self.job_base[-1] + nj)
        self.jobs = torch.empty(max(self.job_base[-1], 1) * _lib.JOB_BYTES, dtype=torch.uint8, device=dev)
        self.out = torch.empty(max(self.total_out, 1), dtype=torch.uint8, device=dev)
        self.inflate_summ = torch.zeros(ctypes_sizeof(_lib.InflateSummary), dtype=torch.uint8, device=dev)
        self.queue_ws = None  # sized for the form (autotune or launch)
        self.data = []
        for (comp, header), b, total in zip(files, self.out_base, self.inflated):
            self.data.append(self.out[b + header.size : b + total])
        self.chain_ws = torch.empty(
            max([int(_lib.lib.cb_record_chain_workspace_bytes(int(d.numel()))) for d in self.data] + [256]),
            dtype=torch.uint8, device=dev)
        self.chain_summ = torch.zeros((self.n_files, ctypes_sizeof(_lib.ChainSummary)), dtype=torch.uint8,
                                      device=dev)
        self.offsets = [torch.empty(max(n, 1), dtype=torch.int64, device=dev) for n in self.n_records]
        self.results = []
        k = len(self.tags)
        self._tag_arrays = []
        for (comp, header), data, off, nrec, nm, total in zip(files, self.data, self.offsets, self.n_records,
                                                               self.n_members, self.inflated):
            o = off[:nrec]
            cols = {name: torch.empty(nrec, dtype=t, device=dev) for name, t in _TYPES.items()}
            arrs = None
            tag_cols = {}
            if k:
                arrs = _tag_arrays(k, nrec)
                view = _View(data, o)
                for q, t in enumerate(self.tags):
                    tag_cols[t] = Tag._from_columns(view, t, arrs[0][q], arrs[1][q], arrs[2][q], arrs[3][q])
            self._tag_arrays.append(arrs)
            self.results.append(DecodedFile(header, data, o, cols, tag_cols, nm, total))
        self.form = form
        self.graph = None
        if self.form is None:
            self.autotune()

    # ------------------------------------------------------------------ launches
    def launch(self, form: int | None = None, events: StageEvents | None = None) -> None:
        """Issue the whole batch on the current stream (no host synchronisation)."""
        form = form or self.form or 0
        s = stream_ptr()
        _trace.mark(events, "start")
        for k, ((comp, _), n) in enumerate(zip(self.files, [int(c.numel()) for c, _ in self.files])):
            jp = self.jobs.data_ptr() + self.job_base[k] * _lib.JOB_BYTES
            rc = _lib.lib.cb_scan_members(comp.data_ptr() if n else None, n, 1, self.out_base[k], jp,
                                          self.n_jobs[k], self.scan_summ[k].data_ptr(), self.scan_ws.data_ptr(),
                                          self.scan_ws.numel(), s)
            _lib.check(rc, "cb_scan_members")
        _trace.mark(events, "scanned")
        need = inflate_workspace_bytes(self.job_base[-1], self.total_out, form)
        if self.queue_ws is None or self.queue_ws.numel() < need:
            if self.graph is not None:
                raise RuntimeError("the captured plan's inflate workspace is too small for this form")
            self.queue_ws = torch.empty(max(need, 512), dtype=torch.uint8, device="cuda")
        ws = (self.queue_ws if inflate_form(form, self.job_base[-1]) == 3
              else self.queue_ws[: int(_lib.lib.cb_inflate_workspace_bytes())])
        launch_inflate(self.jobs.data_ptr(), self.job_base[-1], self.out.data_ptr(), self.total_out, self.check_crc,
                       self.inflate_summ.data_ptr(), ws, form)
        _trace.mark(events, "inflated")
        for k, ((comp, header), data, off, nrec) in enumerate(zip(self.files, self.data, self.offsets,
                                                                   self.n_records)):
            n = int(data.numel())
            if n:
                rc = _lib.lib.cb_record_chain(data.data_ptr(), n, len(header.names), off.data_ptr(), max(nrec, 1),
                                              self.chain_summ[k].data_ptr(), self.chain_ws.data_ptr(),
                                              self.chain_ws.numel(), s)
                _lib.check(rc, "cb_record_chain")
        _trace.mark(events, "chained")
        for k, (res, arrs, nrec) in enumerate(zip(self.results, self._tag_arrays, self.n_records)):
            if not nrec:
                continue
            cols = res.columns
            k = len(self.tags) if arrs is not None else 0
            rc = _lib.lib.cb_decode_columns(res.data.data_ptr(), res.offset.data_ptr(), nrec,
                                            *(cols[f].data_ptr() for f in FIELDS), None, None, None, None,
                                            "".join(self.tags).encode(), k,
                                            *((a.data_ptr() for a in arrs) if k else (None,) * 4), s)
            _lib.check(rc, "cb_decode_columns")
        _trace.mark(events, "decoded")

    def launches_per_run(self) -> int:
        """Kernels of this library in one :meth:`launch` (the graph holds the same)."""
        chains = sum(1 for d in self.data if int(d.numel()))
        decodes = sum(1 for n in self.n_records if n)
        return (KERNELS["scan"] * self.n_files + inflate_launches(self.form or 0, self.job_base[-1]) + KERNELS["chain"] * chains
                + KERNELS["records"] * decodes)

    def check(self) -> None:
        """Raise on any device status of the last run, or counts that differ from the plan (one sync)."""
        scan = self.scan_summ.cpu().numpy()
        chain = self.chain_summ.cpu().numpy()
        raise_status(read_struct(self.inflate_summ, _lib.InflateSummary).status, "inflate")
        for k in range(self.n_files):
            si = _lib.ScanSummary.from_buffer_copy(scan[k].tobytes())
            raise_status(si.status, "BGZF member scan")
            if int(si.n_jobs) != self.n_jobs[k] or int(si.total_out) != self.inflated[k]:
                raise RuntimeError(f"file {k}: the scan differs from the plan")
            if int(self.data[k].numel()):
                ci = _lib.ChainSummary.from_buffer_copy(chain[k].tobytes())
                raise_status(ci.status, "record chain")
                if int(ci.n_records) != self.n_records[k] or int(ci.tail) != int(self.data[k].numel()):
                    raise RuntimeError(f"file {k}: the record chain differs from the plan")

    # ------------------------------------------------------------------ tuning and graphs
    def autotune(self, reps: int = 2, cache_path=None, use_cache: bool = True) -> dict:
        """Choose the launch parameters for this batch by timing it (:func:`cubam_b200.tune.tune`: the
        inflate form 1-3, form 3's decoder roots, copy warps, decode steps and prefetch, the chain tile),
        apply them to the process and cache them by device and batch shape; returns the tuner's entry
        (``params`` and the milliseconds of every candidate)."""
        from cubam_b200 import tune

        entry = tune.tune(self, reps=reps, path=cache_path, use_cache=use_cache)
        self.form = entry["params"]["inflate_form"]
        self.tuning = entry
        return entry

    def capture(self) -> None:
        """Record :meth:`launch` as a CUDA graph (after one eager run has set every kernel up)."""
        self.launch()
        torch.cuda.synchronize()
        self.check()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch()
        torch.cuda.synchronize()
        self.graph = g

    def replay(self) -> list[DecodedFile]:
        """Re-run the whole batch (the graph when captured, else the launches); no synchronisation."""
        if self.graph is not None:
            self.graph.replay()
        else:
            self.launch()
        return self.results


class _DeviceArray:
    """Device memory owned by a native batch, seen by torch through ``__cuda_array_interface__``."""

    def __init__(self, ptr, shape, typestr: str, owner):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr or 0), False),
                                         "version": 3, "strides": None}
        self.owner = owner  # the batch stays alive while a tensor views its memory


_TYPESTR = {torch.int32: "<i4", torch.uint8: "|u1", torch.uint16: "<u2", torch.int64: "<i8"}


class NativeBatch:
    """The batched decode run by the library itself (``cb_batch_*`` in ``include/cubam_b200.h``): the
    same launch sequence as :class:`BatchPlan` -- every file's member scan, ONE inflate for the members
    of all files, every file's record chain and one record pass per file -- planned, owned and run in
    C++, so that a host that is not Python reaches it through the C ABI.

    ``files`` holds (compressed bytes on the device, header) pairs; :meth:`run` decodes them again
    (the results are rewritten in place), :meth:`capture` records a run as a CUDA graph that later runs
    replay, :meth:`check` synchronises and raises on any status or count that differs from the plan.
    """

    def __init__(self, files: list[tuple[torch.Tensor, BamHeader]], tags=("CB", "UB", "GN"), check_crc: bool = True):
        import ctypes

        self.files = files
        self.tags = tuple(tags)
        n = len(files)
        ptrs = (ctypes.c_void_p * n)(*[c.data_ptr() if c.numel() else None for c, _ in files])
        sizes = (ctypes.c_int64 * n)(*[int(c.numel()) for c, _ in files])
        handle = ctypes.c_void_p()
        rc = _lib.lib.cb_batch_create(ptrs, sizes, n, "".join(self.tags).encode(), len(self.tags), int(check_crc),
                                      stream_ptr(), ctypes.byref(handle))
        _raise(rc, "cb_batch_create")
        self._h = handle
        self.results = [self._file(k) for k in range(n)]

    def _file(self, k: int) -> DecodedFile:
        info = _lib.BatchFile()
        _raise(_lib.lib.cb_batch_file_info(self._h, k, info), "cb_batch_file_info")
        n, kt = int(info.n_records), int(info.k_tags)

        def view(ptr, dtype, shape):
            if not all(shape):
                return torch.empty(shape, dtype=dtype, device="cuda")
            return torch.as_tensor(_DeviceArray(ptr, shape, _TYPESTR[dtype], self), device="cuda")

        data = view(info.data, torch.uint8, (int(info.data_bytes),))
        off = view(info.offsets, torch.int64, (n,))
        cols = {f: view(getattr(info, f), t, (n,)) for f, t in _TYPES.items()}
        tag_cols = {}
        if kt:
            arrs = (view(info.tag_type, torch.uint8, (kt, n)), view(info.tag_voff, torch.int64, (kt, n)),
                    view(info.tag_vlen, torch.int32, (kt, n)), view(info.tag_value, torch.int64, (kt, n)))
            v = _View(data, off)
            for q, t in enumerate(self.tags):
                tag_cols[t] = Tag._from_columns(v, t, *(a[q] for a in arrs))
        return DecodedFile(self.files[k][1], data, off, cols, tag_cols, int(info.n_members), int(info.inflated_bytes))

    @property
    def form(self) -> int:
        return int(_lib.lib.cb_batch_form(self._h))

    def run(self) -> None:
        _raise(_lib.lib.cb_batch_run(self._h, stream_ptr()), "cb_batch_run")

    def capture(self) -> None:
        _raise(_lib.lib.cb_batch_capture(self._h, stream_ptr()), "cb_batch_capture")

    def check(self) -> None:
        _raise(_lib.lib.cb_batch_check(self._h, stream_ptr()), "cb_batch_check")

    def close(self) -> None:
        if getattr(self, "_h", None):
            torch.cuda.synchronize()
            _lib.lib.cb_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass


def _raise(rc: int, what: str) -> None:
    """The reference's exception for a status code, NativeError for CUDA and argument errors."""
    if rc in (_lib.OK, _lib.CUDA, _lib.ARG):
        if rc == _lib.ARG:
            raise _lib.NativeError(f"{what}: {_lib.lib.cb_last_error().decode()}")
        _lib.check(rc, what)
        return
    raise_status(rc, what)
