"""BGZF writing on the CPU: TEST INFRASTRUCTURE ONLY.

Restates the write side of cubam's ``src/cubam/bgzf.py`` with Python's zlib as the DEFLATE coder
(cubam's coder is nvCOMP, a closed library, so the compressed payload bytes cannot be matched
byte for byte; everything around them can):

- ``_bgzf_compress`` (``:380-422``): blocks of ``BLOCK_DATA`` bytes (or the given spans), each a
  gzip member with the BGZF extra field (``bgzf_frame``, ``src/cubam/_kernels.py:161-191``): the
  16 fixed header bytes, BSIZE = member bytes - 1, the DEFLATE payload, CRC32, ISIZE; a block whose
  compressed payload would make the member longer than 65,536 bytes is a stored block instead
  (``:401``);
- ``BgzfWriter`` (``:425-539``): bytes are buffered; once ``flush_bytes`` are buffered the whole
  blocks are compressed (the cut is a multiple of ``BLOCK_DATA``, ``:505-515``); ``close``
  compresses the rest and appends ``EOF_BLOCK``;
- member parsing, for comparing the framing of two files field by field.

The golden values pinned here come from the reference's own tests (``tests/test_bgzf.py:97-111``):
a file of whole-``BLOCK_DATA`` blocks decompresses with gzip to its input, and an empty writer
leaves exactly ``EOF_BLOCK``.
"""

from __future__ import annotations

import struct
import zlib

EOF_BLOCK = bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")
BLOCK_DATA = 0xFF00
HEADER = bytes([31, 139, 8, 4, 0, 0, 0, 0, 0, 255, 6, 0, 66, 67, 2, 0])


def deflate(raw: bytes, level: int = 6) -> bytes:
    c = zlib.compressobj(level, zlib.DEFLATED, -15)
    return c.compress(raw) + c.flush()


def stored(raw: bytes) -> bytes:
    n = len(raw)
    return bytes([1]) + struct.pack("<HH", n, n ^ 0xFFFF) + raw


def member(raw: bytes, level: int = 6) -> bytes:
    """One BGZF member of ``raw`` (at most BLOCK_DATA bytes)."""
    pay = deflate(raw, level)
    if len(pay) + 26 > 1 << 16:
        pay = stored(raw)
    bsize = 18 + len(pay) + 8
    return HEADER + struct.pack("<H", bsize - 1) + pay + struct.pack("<II", zlib.crc32(raw), len(raw))


def bgzf_compress(data: bytes, level: int = 6, block_off=None, block_size=None) -> tuple[bytes, list[int]]:
    """The members of ``data`` (no EOF block) and where each starts."""
    if block_off is None:
        block_off = list(range(0, len(data), BLOCK_DATA))
        block_size = [min(BLOCK_DATA, len(data) - o) for o in block_off]
    out, offs, pos = [], [], 0
    for o, s in zip(block_off, block_size, strict=True):
        m = member(data[o : o + s], level)
        offs.append(pos)
        out.append(m)
        pos += len(m)
    return b"".join(out), offs


def writer_blocks(writes: list[bytes], flush_bytes: int = 1024 * BLOCK_DATA, flushes: tuple = ()) -> list[int]:
    """ISIZE of every member a BgzfWriter writes for ``writes`` (in order; ``flushes``: indexes of
    writes after which ``flush()`` is called), without the EOF block."""
    sizes, pending = [], 0

    def cut(n):
        for o in range(0, n, BLOCK_DATA):
            sizes.append(min(BLOCK_DATA, n - o))

    for i, w in enumerate(writes):
        pending += len(w)
        if pending >= flush_bytes:
            c = pending // BLOCK_DATA * BLOCK_DATA
            cut(c)
            pending -= c
        if i in flushes:
            cut(pending)
            pending = 0
    cut(pending)
    return sizes


def members(blob: bytes) -> list[dict]:
    """The BGZF members of ``blob``: offset, BSIZE, payload, CRC32, ISIZE."""
    out, o = [], 0
    while o < len(blob):
        if blob[o : o + 16] != HEADER:
            raise ValueError(f"no BGZF header at {o}")
        bs = struct.unpack_from("<H", blob, o + 16)[0] + 1
        crc, isize = struct.unpack_from("<II", blob, o + bs - 8)
        out.append(dict(offset=o, bsize=bs, payload=blob[o + 18 : o + bs - 8], crc=crc, isize=isize))
        o += bs
    if o != len(blob):
        raise ValueError("the last member runs past the end")
    return out


def inflate_payload(payload: bytes) -> bytes:
    """The bytes of one raw DEFLATE stream; ValueError unless it ends exactly at the payload's end."""
    d = zlib.decompressobj(-15)
    raw = d.decompress(payload)
    if not d.eof or d.unused_data:
        raise ValueError("the DEFLATE stream does not end at the end of its payload")
    return raw
