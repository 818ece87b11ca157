"""The BGZF writer's oracle and host side, without a GPU."""

import gzip
import zlib

import numpy as np

from oracle import bgzf_writer_oracle as W


def test_oracle_framing_matches_the_reference_rules():
    # the reference's writer test data (tests/test_bgzf.py:97-101): repetitive, then random bytes
    rng = np.random.default_rng(1)
    raw = (b"ACGT" * 50_000) + rng.integers(0, 256, 200_000, dtype=np.uint8).tobytes()
    blob, offs = W.bgzf_compress(raw)
    assert gzip.decompress(blob + W.EOF_BLOCK) == raw
    ms = W.members(blob)
    assert [m["offset"] for m in ms] == offs
    assert [m["isize"] for m in ms] == [W.BLOCK_DATA] * (len(raw) // W.BLOCK_DATA) + [len(raw) % W.BLOCK_DATA]
    pos = 0
    for m in ms:
        got = W.inflate_payload(m["payload"])
        assert got == raw[pos : pos + m["isize"]] and zlib.crc32(got) == m["crc"]
        pos += m["isize"]
    # random blocks do not shrink: stored blocks, 5 bytes over their data
    assert any(len(m["payload"]) == m["isize"] + 5 and m["payload"][0] == 1 for m in ms)


def test_empty_member_is_the_eof_block():
    assert W.member(b"") == W.EOF_BLOCK
    assert W.members(W.EOF_BLOCK)[0]["isize"] == 0


def test_writer_cuts_whole_blocks_at_flush_bytes():
    # writes of 77,777 bytes with flush_bytes=100,000 (tests/test_bgzf.py:103-106)
    raw_len = 400_000
    writes = [b"x" * min(77_777, raw_len - k) for k in range(0, raw_len, 77_777)] + [b"end"]
    sizes = W.writer_blocks(writes, flush_bytes=100_000)
    assert sum(sizes) == raw_len + 3
    assert all(s == W.BLOCK_DATA for s in sizes[:-1])
    assert W.writer_blocks([], flush_bytes=100_000) == []
    # flush() ends a block early
    assert W.writer_blocks([b"a" * 10, b"b" * 10], flushes=(0,)) == [10, 10]


def test_writer_api_is_exported_and_sizes_need_no_gpu():
    from cubam_b200 import _lib, bgzf

    for name in ("BgzfWriter", "_bgzf_compress", "_deflate_spans", "_crc32_spans", "_adler32_spans"):
        assert hasattr(bgzf, name), name
    assert bgzf.EOF_BLOCK == W.EOF_BLOCK and bgzf.BLOCK_DATA == W.BLOCK_DATA
    assert _lib.lib.cb_deflate_workspace_bytes(1) >= (1 << 16) * 5
    assert _lib.lib.cb_deflate_workspace_bytes(-1) == 0
    assert _lib.lib.cb_deflate_spans(None, None, None, -1, 1, 0, None, 0, None, None, None, None, None, 0, None) == _lib.ARG
    assert _lib.lib.cb_crc32_spans(None, None, None, 3, None, None) == _lib.ARG
    assert _lib.lib.cb_adler32_spans(None, None, None, -1, None, None) == _lib.ARG
