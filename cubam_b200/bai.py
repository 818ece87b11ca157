"""BAI index of a resident BAM file, and region queries.

cubam has no region access (docs/reading.md:52-53 lists the BAI index as not done,
docs/development.md:52 as next); this adds it on top of the resident files of
:mod:`cubam_b200.serve`.  The index is the standard one of the SAM/BAM specification (SAMv1
section 5.2): per reference, the records' bins (reg2bin over [pos, alignment end)) with their
chunks of virtual offsets, and the linear index of the smallest virtual offset per 16 kb window.

- :func:`build` computes it on the device from one decode of the file (bins, chunk runs and the
  linear index are torch operations over the records' columns and virtual offsets);
  :meth:`BaiIndex.to_bytes` writes the ``.bai`` bytes and :meth:`BaiIndex.from_bytes` reads any
  ``.bai`` of that format.
- :meth:`BaiIndex.query` gives the chunks to read for a region; :func:`fetch` decodes the members
  that hold them and keeps the records that overlap the region.

Chunks are runs of consecutive records with the same bin, and two chunks of a bin are merged when
the first ends in the BGZF block where the second starts (as htslib does, to keep the index small).
"""

from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np
import torch

from cubam_b200.bam import FIELDS, Tag, _index
from cubam_b200.batch import DecodedFile, _View, decode_many
from cubam_b200.serve import Request, ResidentFile, decode_alone

PSEUDO_BIN = 37450
WINDOW_SHIFT = 14


def reg2bin(beg: torch.Tensor, end: torch.Tensor) -> torch.Tensor:
    """Bins of [beg, end) (SAMv1 5.3), element-wise on int64 tensors."""
    e = end - 1
    b = torch.zeros_like(beg)
    done = torch.zeros_like(beg, dtype=torch.bool)
    for first, shift in ((4681, 14), (585, 17), (73, 20), (9, 23), (1, 26)):
        same = (~done) & ((beg >> shift) == (e >> shift))
        b = torch.where(same, first + (beg >> shift), b)
        done |= same
    return b


def reg2bins(beg: int, end: int) -> list[int]:
    """Bins that may hold records overlapping [beg, end) (SAMv1 5.3)."""
    end -= 1
    out = [0]
    for first, shift in ((1, 26), (9, 23), (73, 20), (585, 17), (4681, 14)):
        out.extend(range(first + (beg >> shift), first + (end >> shift) + 1))
    return out


@dataclass
class RefIndex:
    bins: dict = field(default_factory=dict)  # bin -> uint64 array (k, 2) of [begin, end) virtual offsets
    lin: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint64))
    meta: tuple | None = None  # (first record's voff, end of the last, mapped, unmapped)


@dataclass
class BaiIndex:
    refs: list
    n_no_coor: int = 0

    def to_bytes(self) -> bytes:
        out = [b"BAI\x01", struct.pack("<i", len(self.refs))]
        for R in self.refs:
            out.append(struct.pack("<i", len(R.bins) + (R.meta is not None)))
            for b in sorted(R.bins):
                ch = R.bins[b]
                out.append(struct.pack("<Ii", b, len(ch)))
                out.append(np.ascontiguousarray(ch, dtype="<u8").tobytes())
            if R.meta is not None:
                out.append(struct.pack("<Ii", PSEUDO_BIN, 2))
                out.append(struct.pack("<QQQQ", *R.meta))
            out.append(struct.pack("<i", len(R.lin)))
            out.append(np.ascontiguousarray(R.lin, dtype="<u8").tobytes())
        out.append(struct.pack("<Q", self.n_no_coor))
        return b"".join(out)

    @classmethod
    def from_bytes(cls, b: bytes) -> BaiIndex:
        if b[:4] != b"BAI\x01":
            raise ValueError("not a BAI index")
        o = 4
        (n_ref,) = struct.unpack_from("<i", b, o)
        o += 4
        refs = []
        for _ in range(n_ref):
            R = RefIndex()
            (n_bin,) = struct.unpack_from("<i", b, o)
            o += 4
            for _ in range(n_bin):
                bn, nc = struct.unpack_from("<Ii", b, o)
                o += 8
                ch = np.frombuffer(b, dtype="<u8", count=2 * nc, offset=o).reshape(nc, 2).copy()
                o += 16 * nc
                if bn == PSEUDO_BIN:
                    R.meta = (int(ch[0, 0]), int(ch[0, 1]), int(ch[1, 0]), int(ch[1, 1]))
                else:
                    R.bins[bn] = ch
            (n_intv,) = struct.unpack_from("<i", b, o)
            o += 4
            R.lin = np.frombuffer(b, dtype="<u8", count=n_intv, offset=o).copy()
            o += 8 * n_intv
            refs.append(R)
        n_no_coor = struct.unpack_from("<Q", b, o)[0] if o + 8 <= len(b) else 0
        return cls(refs, int(n_no_coor))

    def query(self, ref: int, beg: int, end: int) -> list[tuple[int, int]]:
        """Merged chunks [begin, end) of virtual offsets that hold every record overlapping
        [beg, end) of reference ``ref`` (and possibly others: the caller filters)."""
        if ref < 0 or ref >= len(self.refs) or end <= beg:
            return []
        R = self.refs[ref]
        w = beg >> WINDOW_SHIFT
        min_off = int(R.lin[min(w, len(R.lin) - 1)]) if len(R.lin) else 0
        chunks = []
        for b in reg2bins(max(beg, 0), end):
            ch = R.bins.get(b)
            if ch is not None:
                chunks.extend((int(u), int(v)) for u, v in ch if int(v) > min_off)
        chunks.sort()
        merged = []
        for u, v in chunks:
            if merged and u <= merged[-1][1]:
                merged[-1] = (merged[-1][0], max(merged[-1][1], v))
            else:
                merged.append((u, v))
        return merged


def record_voffs(rf: ResidentFile, offset: torch.Tensor) -> tuple[torch.Tensor, torch.Tensor]:
    """Virtual offsets of records (offsets into the records area) and of the end of each."""
    ix = rf.index
    dev = offset.device
    starts = offset + rf.header.size
    uc = torch.from_numpy(ix.ucum).to(dev)
    co = torch.from_numpy(ix.coff).to(dev)
    m = torch.searchsorted(uc, starts, right=True) - 1
    voff = (co[m] << 16) | (starts - uc[m])
    nxt = torch.empty_like(voff)
    if len(voff):
        nxt[:-1] = voff[1:]
        nxt[-1] = int(ix.coff[-1]) << 16  # the end of the last member with data
    return voff, nxt


def build(rf: ResidentFile, decoded: DecodedFile | None = None) -> BaiIndex:
    """The BAI index of a resident file, computed on the device."""
    d = decoded if decoded is not None else decode_many([(rf.comp, rf.header)], tags=())[0]
    n_ref = len(rf.header.names)
    ref = d.columns["ref"].to(torch.int64)
    pos = d.columns["pos"].to(torch.int64)
    end = torch.maximum(d.columns["end"].to(torch.int64), pos + 1)
    flag = d.columns["flag"].to(torch.int64)
    voff, nxt = record_voffs(rf, d.offset)
    n = int(ref.numel())
    coor = ref >= 0
    n_no_coor = int((~coor).sum().item())
    b = reg2bin(pos, end)
    # chunks: runs of consecutive records with the same (ref, bin), records without a reference
    # breaking runs
    key = torch.where(coor, ref * 65536 + b, torch.full_like(ref, -1))
    starts = torch.ones(n, dtype=torch.bool, device=ref.device)
    if n > 1:
        starts[1:] = key[1:] != key[:-1]
    starts &= coor
    first = torch.nonzero(starts).flatten()
    # last record of each run: the record before the next run start (or the end of its coordinate run)
    run_id = torch.cumsum(starts.to(torch.int64), 0) - 1
    in_run = coor & (run_id >= 0)
    last = torch.zeros(len(first), dtype=torch.int64, device=ref.device)
    if len(first):
        idx = torch.arange(n, device=ref.device)
        last.scatter_reduce_(0, run_id[in_run], idx[in_run], reduce="amax", include_self=False)
    run_key = key[first]
    run_u = voff[first]
    run_v = nxt[last]
    order = torch.argsort(run_key, stable=True)
    run_key, run_u, run_v = run_key[order].cpu().numpy(), run_u[order].cpu().numpy(), run_v[order].cpu().numpy()
    # linear index: the smallest voff of the records overlapping each 16 kb window
    w0 = pos >> WINDOW_SHIFT
    w1 = (end - 1) >> WINDOW_SHIFT
    cnt = torch.where(coor, w1 - w0 + 1, torch.zeros_like(w0))
    rep = torch.repeat_interleave(torch.arange(n, device=ref.device), cnt)
    if len(rep):
        within = torch.arange(len(rep), device=ref.device) - torch.repeat_interleave(torch.cumsum(cnt, 0) - cnt, cnt)
        wref, wwin, wvoff = ref[rep], w0[rep] + within, voff[rep]
        maxw = int(wwin.max().item()) + 1
        flat = torch.full((n_ref * maxw,), -1, dtype=torch.int64, device=ref.device)
        flat.scatter_reduce_(0, wref * maxw + wwin, wvoff, reduce="amin", include_self=False)
        flat = flat.view(n_ref, maxw).cpu().numpy()
    else:
        maxw, flat = 0, np.full((n_ref, 0), -1, np.int64)
    mapped = torch.zeros(n_ref, dtype=torch.int64, device=ref.device)
    unmapped = torch.zeros(n_ref, dtype=torch.int64, device=ref.device)
    if n:
        mapped.index_add_(0, ref[coor], ((flag[coor] & 4) == 0).to(torch.int64))
        unmapped.index_add_(0, ref[coor], ((flag[coor] & 4) != 0).to(torch.int64))
    rbeg = torch.full((n_ref,), -1, dtype=torch.int64, device=ref.device)
    rend = torch.full((n_ref,), -1, dtype=torch.int64, device=ref.device)
    if n and bool(coor.any()):
        idx = torch.arange(n, device=ref.device)
        fi = torch.full((n_ref,), n, dtype=torch.int64, device=ref.device)
        la = torch.full((n_ref,), -1, dtype=torch.int64, device=ref.device)
        fi.scatter_reduce_(0, ref[coor], idx[coor], reduce="amin", include_self=True)
        la.scatter_reduce_(0, ref[coor], idx[coor], reduce="amax", include_self=True)
        has = la >= 0
        rbeg = torch.where(has, voff[fi.clamp(max=max(n - 1, 0))], rbeg)
        rend = torch.where(has, nxt[la.clamp(min=0)], rend)
    mapped, unmapped, rbeg, rend = (x.cpu().numpy() for x in (mapped, unmapped, rbeg, rend))
    refs = [RefIndex() for _ in range(n_ref)]
    rk = run_key // 65536
    bk = run_key % 65536
    bounds = np.flatnonzero(np.diff(run_key)) + 1
    for s, e in zip(np.concatenate([[0], bounds]), np.concatenate([bounds, [len(run_key)]])):
        if s == e:
            continue
        u, v = run_u[s:e], run_v[s:e]
        # merge a chunk into the one before when that one ends in the block where it starts
        new = np.ones(len(u), dtype=bool)
        new[1:] = (v[:-1] >> 16) < (u[1:] >> 16)
        mu = u[new]
        mv = np.maximum.reduceat(v, np.flatnonzero(new))
        refs[int(rk[s])].bins[int(bk[s])] = np.stack([mu, mv], axis=1).astype(np.uint64)
    for r in range(n_ref):
        R = refs[r]
        if rbeg[r] >= 0:
            R.meta = (int(rbeg[r]), int(rend[r]), int(mapped[r]), int(unmapped[r]))
        row = flat[r] if maxw else np.zeros(0, np.int64)
        set_ = np.flatnonzero(row >= 0)
        if len(set_):
            n_intv = int(set_[-1]) + 1
            vals = row[:n_intv].copy()
            # empty windows take the value of the window before; those before the first record's
            # window take the reference's first record offset (the pseudo-bin's start), as htslib does
            fill = np.maximum.accumulate(np.where(vals >= 0, np.arange(n_intv), -1))
            lead = int(rbeg[r]) if rbeg[r] >= 0 else 0
            R.lin = np.where(fill >= 0, vals[np.maximum(fill, 0)], lead).astype(np.uint64)
    return BaiIndex(refs, n_no_coor)


def _boundary_at_or_after(rf: ResidentFile, v: int) -> int:
    """The first member whose first record starts at or after virtual offset v."""
    ix = rf.index
    ok = rf.boundaries()
    c, u = v >> 16, v & 0xFFFF
    m = int(np.searchsorted(ix.coff, c))
    if m < len(ix.coff) and int(ix.coff[m]) == c and int(ix.first_rec[m]) >= u:
        start = m
    else:
        start = m + 1 if m < len(ix.coff) and int(ix.coff[m]) == c else m
    k = int(np.searchsorted(ok, start))
    return int(ok[min(k, len(ok) - 1)])


def fetch(rf: ResidentFile, index: BaiIndex, ref: int | str, beg: int, end: int,
          tags=("CB", "UB", "GN")) -> DecodedFile:
    """Records of reference ``ref`` (index or name) overlapping [beg, end), with their columns and
    tags: the members holding the index's chunks are decoded, the overlapping records kept."""
    if isinstance(ref, str):
        ref = rf.header.names.index(ref)
    chunks = index.query(ref, beg, end)
    ix = rf.index
    if chunks:
        u, v = chunks[0][0], max(c[1] for c in chunks)
        m0 = int(np.searchsorted(ix.coff, u >> 16))
        m1 = _boundary_at_or_after(rf, v)
        req = Request(0, rf.voff(m0), rf.voff(max(m1, m0)))
    else:
        b = int(rf.boundaries()[0])
        req = Request(0, rf.voff(b), rf.voff(b))
    res = decode_alone(rf, req, tags=tags)
    c = res.columns
    pos = c["pos"].to(torch.int64)
    e = torch.maximum(c["end"].to(torch.int64), pos + 1)
    keep = (c["ref"].to(torch.int64) == ref) & (pos < end) & (e > beg)
    sel = torch.nonzero(keep).flatten()
    off = res.offset[sel]
    cols = {k: _index(c[k], sel) for k in FIELDS}
    view = _View(res.data, off)
    tag_cols = {t: Tag._from_columns(view, t, _index(T.type, sel), _index(T.offset, sel), _index(T.length, sel),
                                     _index(T.value, sel))
                for t, T in res.tags.items()}
    return DecodedFile(rf.header, res.data, off, cols, tag_cols, res.n_members, res.inflated_bytes)
