"""The CPU oracle against the golden vectors made by the reference (``tests/golden/``)."""

import zlib
from pathlib import Path

import numpy as np
import pytest

from golden_io import GOLDEN, TAGS, bam_cases, batches, meta
from oracle import bam_oracle as O


@pytest.mark.parametrize(("name", "chunk"), bam_cases())
def test_read_bam_matches_reference(name, chunk):
    raw = (GOLDEN / name).read_bytes()
    got = list(O.read_bam(raw, chunk))
    exp = batches(name, chunk)
    assert len(got) == len(exp)
    for b, e in zip(got, exp):
        assert len(b.data) == e["data_size"]
        assert b.offset.tolist() == e["offset"].tolist()
        for k in O.FIELDS:
            assert b.columns[k].dtype == e[k].dtype, k
            assert b.columns[k].tolist() == e[k].tolist(), k
        d, off = b.data, b.offset
        assert O.name_hash(d, off).tolist() == e["name_hash"].tolist()
        assert O.names(d, off) == e["names"]
        assert O.aligned_length(d, off).tolist() == e["aligned_length"].tolist()
        assert O.five_prime(b.columns).tolist() == e["five_prime"].tolist()
        assert O.record_sizes(d, off).tolist() == e["record_sizes"].tolist()
        for split in (0, 1):
            rec, start, end = O.blocks(d, off, bool(split))
            assert rec.tolist() == e[f"blocks{split}_rec"].tolist()
            assert start.tolist() == e[f"blocks{split}_start"].tolist()
            assert end.tolist() == e[f"blocks{split}_end"].tolist()
        assert O.base_at(d, off, e["base_rec"], e["base_pos"]).tolist() == e["base_at"].tolist()
        for t in TAGS:
            ty, vo, vl, iv = O.find_tag(d, off, t)
            p = f"tag_{t}_"
            assert ty.tolist() == e[p + "type"].tolist(), t
            assert vo.tolist() == e[p + "offset"].tolist(), t
            assert vl.tolist() == e[p + "length"].tolist(), t
            assert iv.tolist() == e[p + "value"].tolist(), t
            assert O.tag_hash(d, ty, vo, vl).tolist() == e[p + "hash"].tolist(), t
            code, ok = O.tag_packed(d, ty, vo, vl)
            assert code.tolist() == e[p + "packed"].tolist(), t
            assert ok.tolist() == e[p + "packed_ok"].astype(bool).tolist(), t
            assert O.tag_strings(d, ty, vo, vl) == e[p + "str"], t


def test_bgzf_chunks_match_reference():
    data = (GOLDEN / "text.raw").read_bytes()
    for key, sizes in meta()["bgzf"].items():
        name, chunk = key.split(":")
        raw = (GOLDEN / name).read_bytes()
        got = list(O.inflate_chunks(raw, int(chunk), check_crc=True))
        assert [len(c) for c in got] == sizes
        assert b"".join(got) == data


@pytest.mark.parametrize(
    ("case", "file", "chunk"),
    [
        ("truncated", "truncated.gz", 8192),
        ("bad_btype", "corrupt_bad_btype.gz", 8192),
        ("bad_isize", "corrupt_bad_isize.gz", 8192),
        ("isize_too_big", "corrupt_isize_too_big.gz", 8192),
        ("bad_empty_member", "corrupt_bad_empty_member.gz", 8192),
    ],
)
def test_bgzf_errors_match_reference(case, file, chunk):
    kind, msg = meta()["errors"][case]
    with pytest.raises(ValueError) as ei:
        list(O.inflate_chunks((GOLDEN / file).read_bytes(), chunk))
    assert kind == "ValueError"
    assert str(ei.value) == msg


def test_not_bgzf_and_empty():
    kind, msg = meta()["errors"]["not_bgzf"]
    with pytest.raises(ValueError, match=msg):
        list(O.inflate_chunks(b"hello world, not compressed" * 100, 4096))
    eof = bytes.fromhex("1f8b08040000000000ff0600424302001b0003000000000000000000")
    assert b"".join(O.inflate_chunks(eof, 4096)) == b""


def test_crc_check_is_a_strictening():
    raw = (GOLDEN / "corrupt_bad_crc.gz").read_bytes()
    assert meta()["errors"]["bad_crc_reference"][0] == "ok"
    assert sum(len(c) for c in O.inflate_chunks(raw, 8192)) == 50_000
    with pytest.raises(ValueError, match="CRC32"):
        list(O.inflate_chunks(raw, 8192, check_crc=True))


def test_hashes_and_codes_match_reference_host_helpers():
    m = meta()
    for v, h in m["fnv1a"].items():
        assert O.fnv1a(v.encode()) == h
    for v, code in m["pack_acgt"].items():
        b = v.encode()
        got, ok = O.pack_acgt(b, [0], [len(b)])
        assert int(got[0]) == code
        if code:
            assert O.unpack_acgt([code]) == [v]


def test_header_matches_reference():
    for name, h in meta()["header"].items():
        text, names, lengths, size = O.read_header((GOLDEN / name).read_bytes())
        assert (text, names, lengths, size) == (h["text"], h["names"], h["lengths"], h["size"])


def test_truncated_bam_raises():
    raw = (GOLDEN / "pairs.bam").read_bytes()
    # drop the EOF member and the last member's tail: the records end in the middle
    import gzip

    data = gzip.decompress(raw)
    import struct

    def member(chunk):
        c = zlib.compressobj(6, zlib.DEFLATED, -15)
        p = c.compress(chunk) + c.flush()
        return (b"\x1f\x8b\x08\x04\x00\x00\x00\x00\x00\xff\x06\x00BC\x02\x00" + struct.pack("<H", 26 + len(p) - 1)
                + p + struct.pack("<II", zlib.crc32(chunk), len(chunk)))

    cut = member(data[:-10])
    with pytest.raises(ValueError, match="truncated BAM file"):
        list(O.read_bam(cut, 1 << 20))


def _fake_headers(count: int) -> bytes:
    """A chunk of BGZF member headers every 18 bytes, each claiming a 26-byte member: far more header
    matches than a real chunk holds (at least 28 bytes per member)."""
    import struct

    return (bytes.fromhex("1f8b08040000000000ff060042430200") + struct.pack("<H", 25)) * count


def test_too_many_member_candidates():
    """The reference raises "Too many candidates" when a chunk holds more than n/28 + 1024 member
    header matches (src/cubam/bgzf.py:554, src/cubam/_kernels.py:671); the oracle does the same."""
    with pytest.raises(ValueError, match="Too many candidates: the data is corrupt"):
        O.scan_members(_fake_headers(8000), True)
    few = _fake_headers(1000)  # 18,000 bytes: 1,000 matches, under 18,000 / 28 + 1024
    with pytest.raises(ValueError) as e:
        O.scan_members(few, True)
    assert "Too many" not in str(e.value)
