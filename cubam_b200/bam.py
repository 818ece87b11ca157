"""BAM records on the B200, as columns.

The API of cubam's ``src/cubam/bam.py``: :func:`read_bam` (``:421``) yields
one :class:`RecordBatch` (``:251``) per chunk of the file, with the chunk's
inflated bytes on the GPU, the offset of each record and the fixed fields
decoded into columns; :meth:`RecordBatch.tag` (``Tag``, ``:176``) and the
other decoders work on request.  Columns are PyTorch CUDA tensors (DLPack:
``cupy.from_dlpack(t)`` gives CuPy arrays without a copy); string columns are
:class:`~cubam_b200.strings.StringColumn`.

Records are found with the reference's record predicate
(``src/cubam/_kernels.py:250-278``) at every byte offset, and the chain from
offset 0 is kept (``cb_record_chain``), so batches hold exactly the records
cubam's batches hold for the same ``chunk_bytes``.
"""

from __future__ import annotations

import gzip
import struct
import zlib
from collections.abc import Iterator
from dataclasses import dataclass
from pathlib import Path

import numpy as np
import torch

from cubam_b200 import _lib
from cubam_b200.bgzf import _inflate, check_inflate, ctypes_sizeof, raise_status, read_struct, stream_ptr
from cubam_b200.strings import StringColumn

#: SAM flags
PAIRED, PROPER_PAIR, UNMAPPED, MATE_UNMAPPED = 0x1, 0x2, 0x4, 0x8
REVERSE, MATE_REVERSE, READ1, READ2 = 0x10, 0x20, 0x40, 0x80
SECONDARY, QC_FAIL, DUPLICATE, SUPPLEMENTARY = 0x100, 0x200, 0x400, 0x800

FIELDS = ("ref", "pos", "end", "mapq", "flag", "nref", "npos", "tlen", "l_seq", "clip_left", "clip_right")
_TYPES = {
    "ref": torch.int32,
    "pos": torch.int32,
    "end": torch.int32,
    "mapq": torch.uint8,
    "flag": torch.uint16,
    "nref": torch.int32,
    "npos": torch.int32,
    "tlen": torch.int32,
    "l_seq": torch.int32,
    "clip_left": torch.uint16,
    "clip_right": torch.uint16,
}


_SIGNED_VIEW = {torch.uint16: torch.int16, torch.uint32: torch.int32, torch.uint64: torch.int64}


def _index(t: torch.Tensor, idx: torch.Tensor) -> torch.Tensor:
    """``t[idx]`` for every dtype (unsigned 16/32/64-bit tensors go through same-width signed views)."""
    s = _SIGNED_VIEW.get(t.dtype)
    return t[idx] if s is None else t.view(s)[idx].view(t.dtype)


def _ptr(t: torch.Tensor | None):
    return None if t is None or t.numel() == 0 else t.data_ptr()


class _MemberStream:
    """The inflated bytes of a gzip/BGZF file, produced member by member as a reader asks for them.

    Only as many members are read and inflated as the bytes asked for need: a BAM header takes the
    first member or few of a file of any size.  A file that is not gzip raises
    :class:`gzip.BadGzipFile`, as reading it with :mod:`gzip` would.
    """

    _READ = 1 << 16

    def __init__(self, path: str | Path):
        self._fh = open(path, "rb")  # noqa: SIM115  (closed by close())
        self._inflater = zlib.decompressobj(31)  # a gzip member: header, raw DEFLATE, trailer
        self._have = bytearray()
        self._raw = b""  # file bytes read but not yet given to the inflater
        self._started = False
        self._spent = False  # the file has no more bytes

    def close(self) -> None:
        self._fh.close()

    def _more(self) -> bool:
        """Inflate some more of the file into the buffer; False once nothing is left."""
        while True:
            raw, self._raw = self._raw, b""
            if not raw:
                if self._spent:
                    return False
                raw = self._fh.read(self._READ)
                if not raw:
                    self._spent = True
                    return False
            try:
                got = self._inflater.decompress(raw)
            except zlib.error as e:
                if not self._started:
                    raise gzip.BadGzipFile(f"Not a gzipped file ({raw[:2]!r})") from e
                raise
            self._started = True
            self._have += got
            if self._inflater.eof:  # the member ended: what is left of raw starts the next one
                self._raw = self._inflater.unused_data
                self._inflater = zlib.decompressobj(31)
            if got:
                return True

    def take(self, n: int) -> bytes | None:
        """The next ``n`` inflated bytes, or None when the file ends first (or ``n`` is negative)."""
        if n < 0:
            return None
        while len(self._have) < n:
            if not self._more():
                return None
        out = bytes(self._have[:n])
        del self._have[:n]
        return out


@dataclass(frozen=True)
class BamHeader:
    """The header of a BAM file: SAM text, reference names and lengths, and ``size``, the inflated
    bytes before the first record (the API of cubam's ``BamHeader``, ``src/cubam/bam.py:40-100``,
    with its error messages)."""

    text: str
    names: list[str]
    lengths: list[int]
    size: int  # bytes of the uncompressed header

    @classmethod
    def read(cls, path: str | Path) -> BamHeader:
        """Parse the header at the start of a BAM file; only the members that hold it are inflated."""
        src = _MemberStream(path)
        try:
            return cls._parse(src, str(path))
        finally:
            src.close()

    @classmethod
    def _parse(cls, src: _MemberStream, where: str) -> BamHeader:
        def need(n: int) -> bytes:
            got = src.take(n)
            if got is None:
                raise ValueError(f"{where}: truncated BAM header")
            return got

        def i32() -> int:
            return struct.unpack("<i", need(4))[0]

        if need(4) != b"BAM\1":
            raise ValueError(f"{where}: not a BAM file")
        l_text = i32()
        sam = need(l_text)
        nul = sam.find(b"\0")
        text = (sam if nul < 0 else sam[:nul]).decode()
        n_ref = i32()
        names, lengths, size = [], [], 12 + l_text
        for _ in range(max(n_ref, 0)):
            l_name = i32()
            names.append(need(l_name)[:-1].decode())  # the name without its terminating byte
            lengths.append(i32())
            size += 8 + l_name
        return cls(text, names, lengths, size)

    def _hd_fields(self) -> list[str]:
        hd = self.text.partition("\n")[0]
        return hd.split("\t")[1:] if hd.startswith("@HD") else []

    @property
    def sort_order(self) -> str:
        """``SO`` of the ``@HD`` line (``unknown`` without one)."""
        return next((f[3:] for f in self._hd_fields() if f.startswith("SO:")), "unknown")

    def to_bytes(self, text: str | None = None) -> bytes:
        """The uncompressed BAM header, with ``text`` in place of the SAM text."""
        sam = (self.text if text is None else text).encode()
        refs = bytearray()
        for name, length in zip(self.names, self.lengths, strict=True):
            nb = name.encode()
            refs += struct.pack("<i", len(nb) + 1) + nb + b"\0" + struct.pack("<i", length)
        return b"BAM\1" + struct.pack("<i", len(sam)) + sam + struct.pack("<i", len(self.names)) + bytes(refs)

    def require_coordinate_sorted(self, path: str | Path = "BAM") -> None:
        """ValueError unless ``@HD SO`` is ``coordinate``."""
        order = self.sort_order
        if order != "coordinate":
            raise ValueError(f"{path}: not coordinate-sorted (@HD SO:{order})")

    def lines(self, kind: str) -> list[str]:
        """The header lines of one record type (``"@SQ"``, ``"@PG"`` ...)."""
        prefix = kind + "\t"
        return [ln for ln in self.text.split("\n") if ln.startswith(prefix)]


def _strings_at(data: torch.Tensor, offset: torch.Tensor, length: torch.Tensor) -> StringColumn:
    """``data[offset[i] : offset[i] + length[i]]`` as a string column (``bam.py:103-112``)."""
    n = int(offset.numel())
    offsets = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    if n:
        torch.cumsum(length.to(torch.int64), 0, out=offsets[1:])
    total = int(offsets[-1])
    chars = torch.empty(max(total, 1), dtype=torch.uint8, device="cuda")
    if n:
        rc = _lib.lib.cb_copy_spans(
            _ptr(data), chars.data_ptr(), offset.to(torch.int64).contiguous().data_ptr(), offsets.data_ptr(),
            length.to(torch.int64).contiguous().data_ptr(), n, stream_ptr(),
        )
        _lib.check(rc, "cb_copy_spans")
    return _string_series(chars, offsets)


def _string_series(chars: torch.Tensor, offsets: torch.Tensor) -> StringColumn:
    """A string column of ``chars[offsets[i] : offsets[i + 1]]`` (``bam.py:115-134``): int32 offsets below 2^31 - 1."""
    total = int(offsets[-1])
    if total < 2**31 - 1:
        offsets = offsets.to(torch.int32)
    return StringColumn(chars, offsets)


def unpack_acgt(codes) -> StringColumn:
    """Strings of codes made by :meth:`Tag.packed` (``bam.py:137-161``)."""
    codes = torch.as_tensor(codes, device="cuda").to(torch.uint64)
    n = int(codes.numel())
    c = codes.view(torch.int64)
    nb = (c >> 48) & 31
    suffix = ((c >> 53) & 0x7FF) - 1
    length = nb + torch.where(suffix >= 0, 2 + (suffix >= 10).to(torch.int64) + (suffix >= 100).to(torch.int64), 0)
    offsets = torch.zeros(n + 1, dtype=torch.int64, device="cuda")
    if n:
        torch.cumsum(length, 0, out=offsets[1:])
    chars = torch.empty(max(int(offsets[-1]), 1), dtype=torch.uint8, device="cuda")
    if n:
        rc = _lib.lib.cb_unpack_acgt(codes.contiguous().data_ptr(), offsets.data_ptr(), n, chars.data_ptr(),
                                     stream_ptr())
        _lib.check(rc, "cb_unpack_acgt")
    return StringColumn(chars, offsets.to(torch.int32))


def _fnv1a(values) -> np.ndarray:
    """64-bit FNV-1a hashes of strings on the host, as :meth:`Tag.hash` computes them (``bam.py:164-173``)."""
    out = np.empty(len(values), np.uint64)
    mask = (1 << 64) - 1
    for i, v in enumerate(values):
        x = 1469598103934665603
        for c in v.encode():
            x = ((x ^ c) * 1099511628211) & mask
        out[i] = x
    return out


def find_tags(batch: RecordBatch, names: list[str]) -> list[Tag]:
    """Several tags of a batch in one walk over the aux data of each record."""
    for name in names:
        if len(name) != 2:
            raise ValueError(f"A tag name has two characters, not {name!r}")
    n = len(batch)
    out = []
    for k0 in range(0, len(names), 16):
        part = names[k0 : k0 + 16]
        k = len(part)
        ty = torch.empty((k, n), dtype=torch.uint8, device="cuda")
        vo = torch.empty((k, n), dtype=torch.int64, device="cuda")
        vl = torch.empty((k, n), dtype=torch.int32, device="cuda")
        iv = torch.empty((k, n), dtype=torch.int64, device="cuda")
        if n:
            rc = _lib.lib.cb_find_tags(
                batch.data.data_ptr(), batch.offset.data_ptr(), n, "".join(part).encode(), k, ty.data_ptr(),
                vo.data_ptr(), vl.data_ptr(), iv.data_ptr(), stream_ptr(),
            )
            _lib.check(rc, "cb_find_tags")
        for t, name in enumerate(part):
            out.append(Tag._from_columns(batch, name, ty[t], vo[t], vl[t], iv[t]))
    return out


class Tag:
    """An auxiliary tag of the records of a batch (``bam.py:176-248``).

    ``type`` is the SAM type character of each record (0 when the tag is
    missing, 255 when the aux data is malformed).  ``value`` holds integer
    values.  String values (``Z``, ``H``) are at ``offset`` with ``length``.
    """

    def __init__(self, batch: RecordBatch, name: str):
        if len(name) != 2:
            raise ValueError(f"A tag name has two characters, not {name!r}")
        (t,) = find_tags(batch, [name])
        self.__dict__.update(t.__dict__)

    @classmethod
    def _from_columns(cls, batch, name, ty, vo, vl, iv) -> Tag:
        t = cls.__new__(cls)
        t.batch, t.name, t.type, t.offset, t.length, t.value = batch, name, ty, vo, vl, iv
        return t

    @property
    def present(self) -> torch.Tensor:
        return (self.type != 0) & (self.type != 255)

    def _is_str(self) -> torch.Tensor:
        return (self.type == ord("Z")) | (self.type == ord("H"))

    def strings(self) -> StringColumn:
        """String values (empty strings where the tag is missing or not a string)."""
        length = torch.where(self._is_str(), self.length, 0).to(torch.int64)
        return _strings_at(self.batch.data, self.offset, length)

    def hash(self) -> torch.Tensor:
        """64-bit FNV-1a hash of string values, 0 where missing."""
        n = len(self.batch)
        out = torch.empty(n, dtype=torch.uint64, device="cuda")
        length = torch.where(self._is_str(), self.length, -1).to(torch.int32).contiguous()
        if n:
            rc = _lib.lib.cb_hash_spans(self.batch.data.data_ptr(), self.offset.contiguous().data_ptr(),
                                        length.data_ptr(), n, out.data_ptr(), stream_ptr())
            _lib.check(rc, "cb_hash_spans")
        return out

    def packed(self):
        """String values packed into uint64 codes, and whether each value fits (``[ACGT]{1,24}`` + ``-N``)."""
        n = len(self.batch)
        out = torch.empty(n, dtype=torch.uint64, device="cuda")
        ok = torch.empty(n, dtype=torch.uint8, device="cuda")
        length = torch.where(self.type == ord("Z"), self.length, 0).to(torch.int32).contiguous()
        if n:
            rc = _lib.lib.cb_pack_acgt(self.batch.data.data_ptr(), self.offset.contiguous().data_ptr(),
                                       length.data_ptr(), n, out.data_ptr(), ok.data_ptr(), stream_ptr())
            _lib.check(rc, "cb_pack_acgt")
        return out, ok.to(torch.bool)


class RecordBatch:
    """BAM records of one chunk, as columns (``bam.py:251-400``).

    Fixed fields are attributes (CUDA tensors): ``ref``, ``pos`` (0-based),
    ``end`` (alignment end, exclusive), ``mapq``, ``flag``, ``nref``,
    ``npos``, ``tlen``, ``l_seq``, and the soft clips ``clip_left`` and
    ``clip_right``.  ``data`` is the chunk's inflated bytes (a writable
    contiguous uint8 tensor) and ``offset`` (int64) where each record starts.
    """

    FIELDS = FIELDS

    def __init__(self, data: torch.Tensor, offset: torch.Tensor, header: BamHeader, columns: dict):
        self.data = data
        self.offset = offset
        self.header = header
        self.columns = columns

    @classmethod
    def decode(cls, data: torch.Tensor, offset: torch.Tensor, header: BamHeader, derived: bool = False) -> RecordBatch:
        """Fixed columns of the records; with ``derived`` also their aligned lengths, read-name hashes
        and aligned-block counts (both modes of :meth:`blocks`), in the same pass over the record bytes
        (then :meth:`aligned_length` and :meth:`name_hash` return them without reading the records
        again, and :meth:`blocks` runs only its writing pass)."""
        n = int(offset.numel())
        cols = {k: torch.empty(n, dtype=t, device="cuda") for k, t in _TYPES.items()}
        extra = {}
        if derived:
            extra = {"aligned_length": torch.empty(n, dtype=torch.int32, device="cuda"),
                     "name_hash": torch.empty(n, dtype=torch.uint64, device="cuda"),
                     "n_blocks": torch.empty(n, dtype=torch.int32, device="cuda"),
                     "n_blocks_split": torch.empty(n, dtype=torch.int32, device="cuda")}
        if n:
            if derived:
                rc = _lib.lib.cb_decode_columns(data.data_ptr(), offset.data_ptr(), n,
                                                *(cols[k].data_ptr() for k in FIELDS),
                                                *(extra[k].data_ptr() for k in ("aligned_length", "name_hash",
                                                                                "n_blocks", "n_blocks_split")),
                                                b"", 0, None, None, None, None, stream_ptr())
                _lib.check(rc, "cb_decode_columns")
            else:
                rc = _lib.lib.cb_decode_fixed(data.data_ptr(), offset.data_ptr(), n,
                                              *(cols[k].data_ptr() for k in FIELDS), stream_ptr())
                _lib.check(rc, "cb_decode_fixed")
        b = cls(data, offset, header, cols)
        b.__dict__["_derived"] = extra
        return b

    def __len__(self) -> int:
        return int(self.offset.numel())

    def __getattr__(self, name: str):
        cols = self.__dict__.get("columns")
        if cols is not None and name in cols:
            return cols[name]
        raise AttributeError(name)

    def take(self, idx) -> RecordBatch:
        """The records at ``idx`` (indices or a boolean mask), sharing the bytes of this batch."""
        idx = torch.as_tensor(idx, device="cuda")
        if idx.dtype == torch.bool:
            idx = torch.nonzero(idx).flatten()
        b = RecordBatch(self.data, self.offset[idx], self.header, {k: _index(v, idx) for k, v in self.columns.items()})
        d = self.__dict__.get("_derived")
        if d:
            b.__dict__["_derived"] = {k: _index(v, idx) for k, v in d.items()}
        return b

    def record_sizes(self) -> torch.Tensor:
        """Bytes of each record, its length field included (int64)."""
        n = len(self)
        out = torch.empty(n, dtype=torch.int64, device="cuda")
        if n:
            _lib.check(_lib.lib.cb_record_sizes(self.data.data_ptr(), self.offset.contiguous().data_ptr(), n,
                                                out.data_ptr(), stream_ptr()), "cb_record_sizes")
        return out

    def has_flags(self, all_of: int = 0, none_of: int = 0) -> torch.Tensor:
        f = self.flag.to(torch.int32)
        return ((f & all_of) == all_of) & ((f & none_of) == 0)

    def tag(self, name: str) -> Tag:
        return Tag(self, name)

    def tags(self, *names: str) -> list[Tag]:
        """Several tags in one walk of the aux data (one launch instead of one per tag)."""
        return find_tags(self, list(names))

    def name_hash(self) -> torch.Tensor:
        """64-bit FNV-1a hash of the read names (mates share it)."""
        d = self.__dict__.get("_derived")
        if d and "name_hash" in d:
            return d["name_hash"]
        n = len(self)
        out = torch.empty(n, dtype=torch.uint64, device="cuda")
        if n:
            _lib.check(_lib.lib.cb_name_hash(self.data.data_ptr(), self.offset.contiguous().data_ptr(), n,
                                             out.data_ptr(), stream_ptr()), "cb_name_hash")
        return out

    def names(self) -> StringColumn:
        """Read names as a string column."""
        off = self.offset.to(torch.int64)
        lrn = self.data[off + 12].to(torch.int64)
        return _strings_at(self.data, off + 36, lrn - 1)

    def aligned_length(self) -> torch.Tensor:
        """Number of aligned bases (CIGAR M, = and X) of each read."""
        d = self.__dict__.get("_derived")
        if d and "aligned_length" in d:
            return d["aligned_length"]
        n = len(self)
        out = torch.empty(n, dtype=torch.int32, device="cuda")
        if n:
            _lib.check(_lib.lib.cb_aligned_length(self.data.data_ptr(), self.offset.contiguous().data_ptr(), n,
                                                  out.data_ptr(), stream_ptr()), "cb_aligned_length")
        return out

    def blocks(self, split_deletions: bool = False):
        """Aligned blocks of the reads: ``(rec, start, end)``, one row per block, in read order."""
        n = len(self)
        off = self.offset.contiguous()
        d = self.__dict__.get("_derived")
        key = "n_blocks_split" if split_deletions else "n_blocks"
        if d and key in d:  # counted by the record pass
            cnt = d[key].contiguous()
        else:
            cnt = torch.zeros(n, dtype=torch.int32, device="cuda")
            if n:
                _lib.check(_lib.lib.cb_blocks(self.data.data_ptr(), off.data_ptr(), n, int(split_deletions), 0,
                                              None, cnt.data_ptr(), None, None, None, stream_ptr()), "cb_blocks")
        first = torch.zeros(n, dtype=torch.int64, device="cuda")
        if n > 1:
            first[1:] = torch.cumsum(cnt[:-1], 0, dtype=torch.int64)
        total = int(first[-1] + cnt[-1]) if n else 0
        rec = torch.empty(total, dtype=torch.int64, device="cuda")
        start = torch.empty(total, dtype=torch.int32, device="cuda")
        end = torch.empty(total, dtype=torch.int32, device="cuda")
        if total:
            _lib.check(_lib.lib.cb_blocks(self.data.data_ptr(), off.data_ptr(), n, int(split_deletions), 1,
                                          first.data_ptr(), cnt.data_ptr(), rec.data_ptr(), start.data_ptr(),
                                          end.data_ptr(), stream_ptr()), "cb_blocks")
        return rec, start, end

    def base_at(self, rec, refpos) -> torch.Tensor:
        """The base of read ``rec[j]`` at reference position ``refpos[j]`` (0-3 ACGT, 4 other, -1 D, -2 N, -3 none)."""
        rec = torch.as_tensor(rec, device="cuda").to(torch.int64).contiguous()
        refpos = torch.as_tensor(refpos, device="cuda").to(torch.int32).contiguous()
        m = int(rec.numel())
        out = torch.empty(m, dtype=torch.int8, device="cuda")
        if m:
            _lib.check(_lib.lib.cb_base_at(self.data.data_ptr(), self.offset.contiguous().data_ptr(), rec.data_ptr(),
                                           refpos.data_ptr(), m, out.data_ptr(), stream_ptr()), "cb_base_at")
        return out

    def five_prime(self) -> torch.Tensor:
        """The 5' end of each read, soft clips included."""
        rev = (self.flag.to(torch.int32) & REVERSE) != 0
        return torch.where(rev, self.end + self.clip_right.to(torch.int32), self.pos - self.clip_left.to(torch.int32))


def record_chain(data: torch.Tensor, n_ref: int):
    """Launch ``cb_record_chain``; returns ``(offsets capacity buffer, device summary)`` without a sync."""
    n = int(data.numel())
    cap = n // 37 + 2  # records are at least 37 bytes
    offsets = torch.empty(cap, dtype=torch.int64, device="cuda")
    summ = torch.zeros(ctypes_sizeof(_lib.ChainSummary), dtype=torch.uint8, device="cuda")
    ws = torch.empty(max(int(_lib.lib.cb_record_chain_workspace_bytes(n)), 256), dtype=torch.uint8, device="cuda")
    rc = _lib.lib.cb_record_chain(_ptr(data), n, n_ref, offsets.data_ptr(), cap, summ.data_ptr(), ws.data_ptr(),
                                  ws.numel(), stream_ptr())
    _lib.check(rc, "cb_record_chain")
    return offsets, summ


def _record_chain(data: torch.Tensor, n_ref: int):
    """Offsets of the complete records of ``data`` and where the next one starts (``bam.py:403-418``)."""
    if int(data.numel()) == 0:
        return torch.empty(0, dtype=torch.int64, device="cuda"), 0
    offsets, summ = record_chain(data, n_ref)
    s = read_struct(summ, _lib.ChainSummary)
    raise_status(s.status, "record chain")
    return offsets[: s.n_records].clone(), int(s.tail)


def read_bam(path: str | Path, chunk_bytes: int | None = None, **reader_kw) -> Iterator[RecordBatch]:
    """Records of a BAM file on the GPU, one :class:`RecordBatch` per chunk (``bam.py:421-446``).

    ``chunk_bytes`` is the size of the compressed chunks (default
    :func:`cubam_b200.auto_chunk_bytes`).  ``reader_kw``: ``n_buffers``,
    ``n_threads``, ``piece`` of the read-ahead thread, and ``check_crc``.
    """
    header = BamHeader.read(path)
    n_ref = len(header.names)
    skip = header.size
    carry = torch.empty(0, dtype=torch.uint8, device="cuda")  # bytes of the incomplete last record
    for data, inflate_summary in _inflate(path, chunk_bytes, lambda: carry, defer_check=True, **reader_kw):  # noqa: B023
        if skip:  # header bytes: no record started yet, so nothing was put in front
            k = min(skip, int(data.numel()))
            data = data[k:]
            skip -= k
        n = int(data.numel())
        if n:
            offsets, summ = record_chain(data, n_ref)
        if inflate_summary is not None:
            check_inflate(inflate_summary)
        if n:
            s = read_struct(summ, _lib.ChainSummary)
            raise_status(s.status, "record chain")
            offset, tail = offsets[: s.n_records].clone(), int(s.tail)
            del offsets
        else:
            offset, tail = torch.empty(0, dtype=torch.int64, device="cuda"), 0
        carry = data[tail:].clone()
        if offset.numel():
            yield RecordBatch.decode(data, offset, header)
        del data, offset
    if carry.numel():
        raise ValueError(f"{path}: truncated BAM file (incomplete record at the end)")
