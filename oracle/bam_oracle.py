"""CPU oracle of the BAM reader hot path: TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this module, and only to check or time against it.
The product path (``cubam_b200``) never calls it.

It restates, in plain Python + numpy + ``zlib``, what cubam's reader does:

- BGZF member scan, chain and checks: ``src/cubam/_kernels.py:69-89``
  (``bgzf_candidates``, ``bgzf_sizes``), ``src/cubam/_kernels.py:676-702``
  (``chain``), ``src/cubam/bgzf.py:542-612`` (``_inflate_blocks``);
- inflate: cubam calls nvCOMP's batched Deflate decompressor
  (``src/cubam/bgzf.py:595``), a closed library pinned as
  ``nvidia-libnvcomp-cu12>=5.1``.  Its algorithm is raw DEFLATE (RFC 1951);
  the oracle uses the system zlib (``zlib.decompressobj(-15)``), which is also
  what the reference's own fixture writer (``tests/bamwriter.py:15-29``) uses;
- chunking and carries: ``src/cubam/bgzf.py:625-652``, ``src/cubam/bam.py:421-446``;
- the record predicate and chain: ``src/cubam/_kernels.py:235-289``,
  ``src/cubam/bam.py:403-418``;
- columns and on-request decoders: ``src/cubam/_kernels.py:292-620``,
  ``src/cubam/bam.py:103-400``.

One deliberate difference is opt-in: ``check_crc=True`` also compares each
member's CRC32 with its trailer, which cubam's reader does not do
(``docs/reading.md:48-51``) and the B200 reader does by default.

Pinning: ``tests/test_oracle.py`` checks this module against the golden
vectors under ``tests/golden/`` (made by the reference's own writer and by the
reference's reader code run on the CPU, see ``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import struct
import zlib

import numpy as np

HEADER, TRAILER = 18, 8
MAX_ISIZE = 1 << 16
FNV_OFFSET = 1469598103934665603
FNV_PRIME = 1099511628211
M64 = (1 << 64) - 1
FIELDS = ("ref", "pos", "end", "mapq", "flag", "nref", "npos", "tlen", "l_seq", "clip_left", "clip_right")
DTYPES = {
    "ref": np.int32,
    "pos": np.int32,
    "end": np.int32,
    "mapq": np.uint8,
    "flag": np.uint16,
    "nref": np.int32,
    "npos": np.int32,
    "tlen": np.int32,
    "l_seq": np.int32,
    "clip_left": np.uint16,
    "clip_right": np.uint16,
}


def _wrap32(x: int) -> int:
    """``x`` as a C ``int`` (two's complement wrap)."""
    x &= 0xFFFFFFFF
    return x - (1 << 32) if x & 0x80000000 else x


def _u16(b, o):
    return b[o] | (b[o + 1] << 8)


def _u32(b, o):
    return b[o] | (b[o + 1] << 8) | (b[o + 2] << 16) | (b[o + 3] << 24)


def _i32(b, o):
    return _wrap32(_u32(b, o))


# ---------------------------------------------------------------- BGZF


def bgzf_candidates(buf: bytes) -> np.ndarray:
    """Offsets whose bytes match a complete BGZF member header (``_kernels.py:69-80``), sorted."""
    a = np.frombuffer(buf, np.uint8)
    n = a.size
    if n < 18:
        return np.empty(0, np.int64)
    o = np.arange(n - 17, dtype=np.int64)
    fixed = {0: 31, 1: 139, 2: 8, 3: 4, 10: 6, 11: 0, 12: 66, 13: 67, 14: 2, 15: 0}
    ok = np.ones(o.size, bool)
    for k, v in fixed.items():
        ok &= a[o + k] == v
    o = o[ok]
    bs = a[o + 16].astype(np.int64) + (a[o + 17].astype(np.int64) << 8) + 1
    return o[(bs >= 26) & (o + bs <= n)]


def _chain_walk(cand: np.ndarray, nxt: np.ndarray) -> np.ndarray:
    """Indices on the chain from ``cand[0]`` (``_kernels.py:676-702``): follow ``nxt`` while it is a candidate."""
    if int(cand[0]) != 0:
        raise ValueError("No valid block or record where one was expected: the data is corrupt")
    where = {int(c): i for i, c in enumerate(cand)}
    keep = [0]
    i = 0
    while True:
        j = where.get(int(nxt[i]))
        if j is None:
            break
        keep.append(j)
        i = j
    return np.asarray(keep, np.int64)


def inflate_member(payload: bytes, isize: int) -> bytes:
    """Raw DEFLATE of one member; raises as the reference does when it does not give ``isize`` bytes."""
    d = zlib.decompressobj(-15)
    try:
        out = d.decompress(payload, isize + 1)
    except zlib.error as e:
        raise ValueError("Corrupt BGZF block: it does not inflate to the size in its trailer") from e
    if not d.eof or len(out) != isize:
        raise ValueError("Corrupt BGZF block: it does not inflate to the size in its trailer")
    return out


def scan_members(buf: bytes, eof: bool):
    """Chained BGZF members of ``buf`` and the bytes used (``bgzf.py:542-584``).

    Returns ``(offsets, bsize, isize, used)`` of the chained members
    (empty members included).  Raises ``ValueError`` with the reference's messages.
    """
    n = len(buf)
    cand = bgzf_candidates(buf)
    if cand.size > n // 28 + 1024:
        raise ValueError("Too many candidates: the data is corrupt")
    if cand.size == 0:
        if eof and n:
            raise ValueError("Truncated BGZF file: the last block is incomplete")
        e = np.empty(0, np.int64)
        return e, e, e, 0
    a = np.frombuffer(buf, np.uint8)
    bsize = a[cand + 16].astype(np.int64) + (a[cand + 17].astype(np.int64) << 8) + 1
    end = cand + bsize
    isize = np.array([_u32(buf, int(e) - 4) for e in end], np.int64)
    keep = _chain_walk(cand, end)
    cand, bsize, isize = cand[keep], bsize[keep], isize[keep]
    used = int(cand[-1] + bsize[-1])
    if eof and used != n:
        raise ValueError("Truncated BGZF file: the last block is incomplete")
    empty = isize == 0
    b18 = a[cand + 18] if cand.size else np.empty(0, np.uint8)
    b19 = a[np.minimum(cand + 19, n - 1)]
    bad = (isize > MAX_ISIZE) | (empty & ((bsize != 28) | (b18 != 3) | (b19 != 0)))
    if bad.any():
        raise ValueError("Corrupt BGZF block")
    return cand, bsize, isize, used


def inflate_blocks(buf: bytes, eof: bool, prefix: bytes = b"", check_crc: bool = False):
    """Inflated complete members of ``buf`` after ``prefix``, and the bytes of ``buf`` used (``bgzf.py:542-612``)."""
    cand, bsize, isize, used = scan_members(buf, eof)
    parts = [prefix]
    for c, bs, isz in zip(cand.tolist(), bsize.tolist(), isize.tolist()):
        if isz == 0:
            continue
        out = inflate_member(buf[c + HEADER : c + bs - TRAILER], isz)
        if check_crc and (zlib.crc32(out) & 0xFFFFFFFF) != _u32(buf, c + bs - 8):
            raise ValueError("Corrupt BGZF block: CRC32 mismatch")
        parts.append(out)
    return b"".join(parts), used


def inflate_chunks(file_bytes: bytes, chunk_bytes: int, prefix=None, check_crc: bool = False):
    """Chunks of inflated data as ``_inflate`` yields them (``bgzf.py:625-652``).

    ``prefix`` (callable or None) is called before each chunk and its bytes
    go in front of the chunk's data.
    """
    carry = b""
    size = len(file_bytes)
    off = 0
    while True:
        n = min(chunk_bytes, size - off)
        buf = carry + file_bytes[off : off + n]
        off += n
        eof = off >= size
        data, used = inflate_blocks(buf, eof, prefix() if prefix else b"", check_crc)
        carry = buf[used:]
        yield data
        if eof:
            return


# ---------------------------------------------------------------- BAM header


def read_header(file_bytes: bytes):
    """``(text, names, lengths, size)`` of the BAM header (``bam.py:50-72``), from the whole gzip stream."""
    import gzip
    import io

    with gzip.GzipFile(fileobj=io.BytesIO(file_bytes)) as fh:

        def take(k):
            b = fh.read(k)
            if len(b) != k:
                raise ValueError("truncated BAM header")
            return b

        if take(4) != b"BAM\1":
            raise ValueError("not a BAM file")
        (l_text,) = struct.unpack("<i", take(4))
        text = take(l_text).split(b"\0", 1)[0].decode()
        (n_ref,) = struct.unpack("<i", take(4))
        names, lengths = [], []
        size = 12 + l_text
        for _ in range(n_ref):
            (ln,) = struct.unpack("<i", take(4))
            names.append(take(ln)[:-1].decode())
            (lr,) = struct.unpack("<i", take(4))
            lengths.append(lr)
            size += 8 + ln
    return text, names, lengths, size


# ---------------------------------------------------------------- records


def reg2bin(beg: int, end: int) -> int:
    """``_kernels.py:235-243`` (arithmetic shifts of C ints)."""
    end = _wrap32(end - 1)
    for shift, base in ((14, 4681), (17, 585), (20, 73), (23, 9), (26, 1)):
        if beg >> shift == end >> shift:
            return base + (beg >> shift)
    return 0


_REF_CONSUMING = (True, False, True, True, False, False, False, True, True)  # M I D N S H P = X


def is_record(b, n: int, o: int, n_ref: int) -> bool:
    """The record predicate of ``_kernels.py:250-278``."""
    if o + 36 > n:
        return False
    bs = _i32(b, o)
    if bs < 33 or bs > (1 << 22) or o + 4 + bs > n:
        return False
    ref, pos, nref, npos = _i32(b, o + 4), _i32(b, o + 8), _i32(b, o + 24), _i32(b, o + 28)
    if ref < -1 or ref >= n_ref or pos < -1 or nref < -1 or nref >= n_ref or npos < -1:
        return False
    lrn, ncig, flag, lseq = b[o + 12], _u16(b, o + 16), _u16(b, o + 18), _u32(b, o + 20)
    if lrn < 2 or flag >= 4096 or lseq > (1 << 22):
        return False
    if 32 + lrn + 4 * ncig + (lseq + 1) // 2 + lseq > bs:
        return False
    nm = o + 36
    if b[nm + lrn - 1] != 0:
        return False
    for i in range(lrn - 1):
        c = b[nm + i]
        if c < 33 or c > 126 or c == 64:
            return False
    cg = nm + lrn
    rlen = 0
    for i in range(ncig):
        v = _u32(b, cg + 4 * i)
        op = v & 15
        if op > 8:
            return False
        if _REF_CONSUMING[op]:
            rlen += v >> 4
    if pos >= 0:
        end = _wrap32(pos + _wrap32(rlen if rlen > 0 else 1))
        if _u16(b, o + 14) != reg2bin(pos, end):
            return False
    return True


def record_chain(data: bytes, n_ref: int):
    """Offsets of the complete records of ``data`` and where the next starts (``bam.py:403-418``).

    The reference tests every byte offset and keeps the chain from offset 0;
    the chain only visits offsets reached from 0, so walking from 0 gives the
    same records.  The all-offsets scan is only needed to tell "no record at
    all" (carry everything) from "corrupt" (offset 0 is not a record while
    another offset is).
    """
    n = len(data)
    if n == 0:
        return np.empty(0, np.int64), 0
    if not is_record(data, n, 0, n_ref):
        cap = n // 32 + 1024
        count = 0
        for o in range(1, n):
            if is_record(data, n, o, n_ref):
                count += 1
                if count > cap:
                    raise ValueError("Too many candidates: the data is corrupt")
        if count:
            raise ValueError("No valid block or record where one was expected: the data is corrupt")
        return np.empty(0, np.int64), 0
    out = []
    o = 0
    while is_record(data, n, o, n_ref):
        out.append(o)
        o = o + 4 + _u32(data, o)
    return np.asarray(out, np.int64), o


def decode_fixed(data: bytes, offset) -> dict:
    """Fixed columns of ``_kernels.py:292-319`` (``decode_fixed``)."""
    n = len(offset)
    cols = {k: np.empty(n, t) for k, t in DTYPES.items()}
    for i, o in enumerate(np.asarray(offset).tolist()):
        p = _i32(data, o + 8)
        cols["ref"][i] = _i32(data, o + 4)
        cols["pos"][i] = p
        cols["mapq"][i] = data[o + 13]
        cols["flag"][i] = _u16(data, o + 18)
        cols["nref"][i] = _i32(data, o + 24)
        cols["npos"][i] = _i32(data, o + 28)
        cols["tlen"][i] = _i32(data, o + 32)
        cols["l_seq"][i] = _i32(data, o + 20)
        lrn, ncig = data[o + 12], _u16(data, o + 16)
        cg = o + 36 + lrn
        rlen = cl = cr = 0
        for k in range(ncig):
            v = _u32(data, cg + 4 * k)
            op, ln = v & 15, v >> 4
            if op <= 8 and _REF_CONSUMING[op]:
                rlen += ln
            if op == 4:
                if k == 0:
                    cl = ln
                else:
                    cr = ln
        cols["end"][i] = _wrap32(p + _wrap32(rlen))
        cols["clip_left"][i] = min(cl, 65535)
        cols["clip_right"][i] = min(cr, 65535)
    return cols


def _tag_walk(b, o: int, t0: int, t1: int):
    """One record of ``find_tag`` (``_kernels.py:334-388``): (type, offset, length, value)."""
    rec_end = o + 4 + _u32(b, o)
    lrn, ncig, lseq = b[o + 12], _u16(b, o + 16), _u32(b, o + 20)
    a = o + 36 + lrn + 4 * ncig + (lseq + 1) // 2 + lseq
    while a + 3 <= rec_end:
        ty = b[a + 2]
        v = a + 3
        if ty in b"AcC":
            nx = v + 1
        elif ty in b"sS":
            nx = v + 2
        elif ty in b"iIf":
            nx = v + 4
        elif ty in b"ZH":
            nx = v
            while nx < rec_end and b[nx] != 0:
                nx += 1
            nx += 1
        elif ty == ord("B"):
            if v + 5 > rec_end:
                nx = -1
            else:
                sub = b[v]
                cnt = _u32(b, v + 1)
                sz = 1 if sub in b"cC" else 2 if sub in b"sS" else 4
                nx = v + 5 + cnt * sz
        else:
            nx = -1
        if nx < 0 or nx > rec_end:
            return 255, 0, 0, 0
        if b[a] == t0 and b[a + 1] == t1:
            iv, vl = 0, 0
            if ty == ord("c"):
                iv = b[v] - 256 if b[v] > 127 else b[v]
            elif ty in b"CA":
                iv = b[v]
            elif ty == ord("s"):
                x = _u16(b, v)
                iv = x - 65536 if x > 32767 else x
            elif ty == ord("S"):
                iv = _u16(b, v)
            elif ty == ord("i"):
                iv = _i32(b, v)
            elif ty == ord("I"):
                iv = _u32(b, v)
            elif ty in b"ZH":
                vl = nx - 1 - v
            elif ty == ord("B"):
                vl = _wrap32(nx - v)
            return ty, v, vl, iv
        a = nx
    return 0, 0, 0, 0


def find_tag(data: bytes, offset, name: str):
    """``(type u8, offset i64, length i32, value i64)`` columns of one tag (``_kernels.py:334-388``)."""
    if len(name) != 2:
        raise ValueError(f"A tag name has two characters, not {name!r}")
    t0, t1 = ord(name[0]), ord(name[1])
    rows = [_tag_walk(data, o, t0, t1) for o in np.asarray(offset).tolist()]
    n = len(rows)
    ty = np.fromiter((r[0] for r in rows), np.uint8, n)
    vo = np.fromiter((r[1] for r in rows), np.int64, n)
    vl = np.fromiter((r[2] for r in rows), np.int32, n)
    iv = np.fromiter((r[3] for r in rows), np.int64, n)
    return ty, vo, vl, iv


def fnv1a(bs: bytes) -> int:
    x = FNV_OFFSET
    for c in bs:
        x = ((x ^ c) * FNV_PRIME) & M64
    return x


def hash_spans(data: bytes, voff, vlen) -> np.ndarray:
    """``_kernels.py:532-540``: FNV-1a 64 of each span, 0 where the length is negative."""
    out = np.zeros(len(voff), np.uint64)
    for i, (o, ln) in enumerate(zip(np.asarray(voff).tolist(), np.asarray(vlen).tolist())):
        out[i] = 0 if ln < 0 else fnv1a(data[o : o + ln])
    return out


def name_hash(data: bytes, offset) -> np.ndarray:
    """``_kernels.py:322-330``."""
    out = np.empty(len(offset), np.uint64)
    for i, o in enumerate(np.asarray(offset).tolist()):
        lrn = data[o + 12]
        out[i] = fnv1a(data[o + 36 : o + 36 + max(lrn - 1, 0)])
    return out


def pack_acgt(data: bytes, voff, vlen):
    """``_kernels.py:544-571``: (codes uint64, ok bool)."""
    n = len(voff)
    codes = np.zeros(n, np.uint64)
    ok = np.zeros(n, bool)
    base = {65: 0, 67: 1, 71: 2, 84: 3}
    for i, (o, ln) in enumerate(zip(np.asarray(voff).tolist(), np.asarray(vlen).tolist())):
        k, e = o, o + ln
        code = suffix = nb = 0
        good = ln > 0
        while good and k < e and data[k] != 45:
            x = base.get(data[k], 4)
            if x == 4 or nb == 24:
                good = False
            else:
                code |= x << (2 * nb)
                nb += 1
            k += 1
        if good and k < e:
            k += 1
            nd = 0
            while k < e:
                c = data[k]
                if c < 48 or c > 57 or nd == 3:
                    good = False
                    break
                suffix = suffix * 10 + (c - 48)
                k += 1
                nd += 1
            if nd == 0:
                good = False
            suffix += 1
        if nb == 0:
            good = False
        codes[i] = ((code | (nb << 48) | (suffix << 53)) & M64) if good else 0
        ok[i] = good
    return codes, ok


def unpack_acgt(codes) -> list[str]:
    """``_kernels.py:607-620`` and ``bam.py:137-161``: the strings of packed codes."""
    out = []
    for c in np.asarray(codes, np.uint64).tolist():
        nb = (c >> 48) & 31
        suffix = c >> 53
        s = "".join("ACGT"[(c >> (2 * k)) & 3] for k in range(nb))
        if suffix:
            s += "-" + str(suffix - 1)
        out.append(s)
    return out


def aligned_length(data: bytes, offset) -> np.ndarray:
    """``_kernels.py:391-403``."""
    out = np.empty(len(offset), np.int32)
    for i, o in enumerate(np.asarray(offset).tolist()):
        lrn, ncig = data[o + 12], _u16(data, o + 16)
        cg = o + 36 + lrn
        s = 0
        for k in range(ncig):
            v = _u32(data, cg + 4 * k)
            if v & 15 in (0, 7, 8):
                s += v >> 4
        out[i] = _wrap32(s)
    return out


def blocks(data: bytes, offset, split_deletions: bool = False):
    """``_kernels.py:408-437`` and ``bam.py:350-373``: (rec i64, start i32, end i32)."""
    rec, start, end = [], [], []
    for i, o in enumerate(np.asarray(offset).tolist()):
        lrn, ncig = data[o + 12], _u16(data, o + 16)
        cg = o + 36 + lrn
        x = s = _i32(data, o + 8)
        for c in range(ncig):
            v = _u32(data, cg + 4 * c)
            op, ln = v & 15, v >> 4
            aligned = op in (0, 7, 8) or (op == 2 and not split_deletions)
            gap = op == 3 or (op == 2 and split_deletions)
            if aligned:
                x = _wrap32(x + ln)
            elif gap:
                if x > s:
                    rec.append(i)
                    start.append(s)
                    end.append(x)
                x = _wrap32(x + ln)
                s = x
        if x > s:
            rec.append(i)
            start.append(s)
            end.append(x)
    return np.asarray(rec, np.int64), np.asarray(start, np.int32), np.asarray(end, np.int32)


def base_at(data: bytes, offset, rec, refpos) -> np.ndarray:
    """``_kernels.py:498-529``."""
    off = np.asarray(offset)
    out = np.empty(len(rec), np.int8)
    for j, (r, target) in enumerate(zip(np.asarray(rec).tolist(), np.asarray(refpos).tolist())):
        o = int(off[r])
        lrn, ncig, lseq = data[o + 12], _u16(data, o + 16), _u32(data, o + 20)
        cg = o + 36 + lrn
        sq = cg + 4 * ncig
        x, y, res = _i32(data, o + 8), 0, -3
        for k in range(ncig):
            v = _u32(data, cg + 4 * k)
            op, ln = v & 15, v >> 4
            if op in (0, 7, 8):
                if target < x + ln:
                    q = y + (target - x)
                    if target >= x and q < lseq:
                        c = (data[sq + q // 2] >> (0 if q & 1 else 4)) & 15
                        res = {1: 0, 2: 1, 4: 2, 8: 3}.get(c, 4)
                    break
                x += ln
                y += ln
            elif op in (2, 3):
                if target < x + ln:
                    res = (-1 if op == 2 else -2) if target >= x else -3
                    break
                x += ln
            elif op in (1, 4):
                y += ln
        out[j] = res
    return out


def record_sizes(data: bytes, offset) -> np.ndarray:
    """``bam.py:308-315``."""
    return np.asarray([_u32(data, o) + 4 for o in np.asarray(offset).tolist()], np.int64)


def strings_at(data: bytes, voff, vlen) -> list[bytes]:
    """``bam.py:103-112``: the spans as byte strings."""
    return [bytes(data[o : o + ln]) for o, ln in zip(np.asarray(voff).tolist(), np.asarray(vlen).tolist())]


def tag_strings(data: bytes, ty, voff, vlen) -> list[bytes]:
    """``Tag.strings`` (``bam.py:214-219``): empty where the tag is missing or not Z/H."""
    is_str = (ty == ord("Z")) | (ty == ord("H"))
    return strings_at(data, voff, np.where(is_str, vlen, 0))


def tag_hash(data: bytes, ty, voff, vlen) -> np.ndarray:
    """``Tag.hash`` (``bam.py:221-230``)."""
    is_str = (ty == ord("Z")) | (ty == ord("H"))
    return hash_spans(data, voff, np.where(is_str, vlen, -1))


def tag_packed(data: bytes, ty, voff, vlen):
    """``Tag.packed`` (``bam.py:232-248``)."""
    return pack_acgt(data, voff, np.where(ty == ord("Z"), vlen, 0))


def names(data: bytes, offset) -> list[bytes]:
    """``RecordBatch.names`` (``bam.py:334-339``)."""
    return [bytes(data[o + 36 : o + 36 + data[o + 12] - 1]) for o in np.asarray(offset).tolist()]


def five_prime(cols: dict) -> np.ndarray:
    """``bam.py:391-400``."""
    rev = (cols["flag"] & 0x10) != 0
    return np.where(
        rev,
        cols["end"] + cols["clip_right"].astype(np.int32),
        cols["pos"] - cols["clip_left"].astype(np.int32),
    ).astype(np.int32)


class Batch:
    """One batch of :func:`read_bam`: the chunk's bytes, record offsets and fixed columns."""

    def __init__(self, data: bytes, offset: np.ndarray):
        self.data = data
        self.offset = offset
        self.columns = decode_fixed(data, offset)

    def __len__(self):
        return len(self.offset)

    def tag(self, name: str):
        return find_tag(self.data, self.offset, name)


def read_bam(file_bytes: bytes, chunk_bytes: int, check_crc: bool = False, decode: bool = True):
    """Batches as ``read_bam`` yields them (``bam.py:421-446``)."""
    _, names_, _, skip = read_header(file_bytes)
    n_ref = len(names_)
    carry = [b""]
    for data in inflate_chunks(file_bytes, chunk_bytes, lambda: carry[0], check_crc):
        if skip:
            k = min(skip, len(data))
            data = data[k:]
            skip -= k
        offset, tail = record_chain(data, n_ref)
        carry[0] = data[tail:]
        if offset.size:
            yield Batch(data, offset) if decode else (data, offset)
    if carry[0]:
        raise ValueError("truncated BAM file (incomplete record at the end)")
