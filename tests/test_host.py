"""Host-side logic of the package that needs no GPU: header, FNV, strings, chunk reader."""

import numpy as np
import torch

from golden_io import GOLDEN, meta


def test_header_matches_reference():
    from cubam_b200 import BamHeader

    for name, g in meta()["header"].items():
        h = BamHeader.read(GOLDEN / name)
        assert (h.text, h.names, h.lengths, h.size) == (g["text"], g["names"], g["lengths"], g["size"])
        assert h.sort_order == g["sort_order"]
        assert h.lines("@PG") == g["pg"]


def test_fnv1a_matches_reference():
    from cubam_b200.bam import _fnv1a

    m = meta()["fnv1a"]
    keys = list(m)
    assert _fnv1a(keys).tolist() == [m[k] for k in keys]


def test_string_column_to_arrow():
    from cubam_b200.strings import StringColumn

    words = [b"ACGT-1", b"", b"read:7", b"x" * 40]
    off = np.zeros(len(words) + 1, np.int32)
    off[1:] = np.cumsum([len(w) for w in words])
    col = StringColumn(torch.frombuffer(bytearray(b"".join(words)), dtype=torch.uint8), torch.from_numpy(off))
    assert col.to_pylist() == [w.decode() for w in words]
    assert col.to_bytes_list() == words
    assert len(col) == 4


def test_chunk_reader_reads_the_file_in_slots(tmp_path):
    from cubam_b200.bgzf import _ChunkReader

    raw = (GOLDEN / "text_b1000.gz").read_bytes()
    for n_buffers in (1, 2, 3):
        r = _ChunkReader(GOLDEN / "text_b1000.gz", 10_000, n_buffers=n_buffers, n_threads=3, piece=3333)
        got, flags = bytearray(), []
        for chunk, eof in r:
            got += chunk.cpu().numpy().tobytes()
            flags.append(eof)
        r.close()
        assert bytes(got) == raw
        assert flags[-1] and not any(flags[:-1])


def test_chunk_reader_empty_file(tmp_path):
    from cubam_b200.bgzf import _ChunkReader

    p = tmp_path / "empty"
    p.write_bytes(b"")
    assert [(int(c.numel()), eof) for c, eof in _ChunkReader(p, 4096)] == [(0, True)]


def test_chunk_reader_error_reaches_the_consumer(tmp_path):
    import pytest

    from cubam_b200.bgzf import _ChunkReader

    r = _ChunkReader(tmp_path / "missing.bam", 4096)
    with pytest.raises(FileNotFoundError):
        list(r)


def test_chunk_reader_fault_in_the_thread_reaches_the_consumer(tmp_path, monkeypatch):
    """A read that fails in the reader thread after some chunks (injected on the host): the consumer
    gets every chunk read before it, then the exception itself."""
    import pytest

    from cubam_b200.bgzf import _ChunkReader

    p = tmp_path / "data"
    p.write_bytes(bytes(range(256)) * 100)  # 25,600 bytes: chunks of 4096
    real = _ChunkReader._read_piece

    def flaky(fd, dst, offset):
        if offset >= 3 * 4096:
            raise OSError(5, "injected read failure")
        real(fd, dst, offset)

    monkeypatch.setattr(_ChunkReader, "_read_piece", staticmethod(flaky))
    got = []
    with pytest.raises(OSError, match="injected read failure"):
        for chunk, _ in _ChunkReader(p, 4096, n_buffers=2, n_threads=2, piece=1000):
            got.append(chunk.cpu().numpy().tobytes())
    assert b"".join(got) == p.read_bytes()[: 3 * 4096]


def test_chunk_reader_short_file_message(tmp_path, monkeypatch):
    """The file shrinking under the reader gives the reference's message."""
    import os

    import pytest

    from cubam_b200.bgzf import _ChunkReader

    p = tmp_path / "data"
    p.write_bytes(b"x" * 10_000)
    monkeypatch.setattr(os, "fstat", lambda fd: os.stat_result((0, 0, 0, 0, 0, 0, 20_000, 0, 0, 0)))
    with pytest.raises(ValueError, match="The file is shorter than its size"):
        list(_ChunkReader(p, 4096))


def test_header_errors_and_round_trip(tmp_path):
    import gzip
    import struct

    import pytest

    from cubam_b200 import BamHeader
    from cubam_b200.bgzf import EOF_BLOCK

    h = BamHeader.read(GOLDEN / "mixed_b700.bam")
    # the header bytes written back as gzip members of one byte each: the header spans many members
    blob = h.to_bytes()
    members = b"".join(gzip.compress(blob[i : i + 1]) for i in range(len(blob)))
    p = tmp_path / "split.bam"
    p.write_bytes(members + EOF_BLOCK)
    h2 = BamHeader.read(p)
    assert h2 == h and h2.size == len(blob)
    t = h.to_bytes("@HD\tVN:1.6\tSO:queryname\n@PG\tID:x\n")
    p.write_bytes(gzip.compress(t))
    h3 = BamHeader.read(p)
    assert h3.sort_order == "queryname" and h3.lines("@PG") == ["@PG\tID:x"]
    with pytest.raises(ValueError, match="not coordinate-sorted"):
        h3.require_coordinate_sorted(p)
    p.write_bytes(gzip.compress(b"BAM\2" + blob[4:]))
    with pytest.raises(ValueError, match="not a BAM file"):
        BamHeader.read(p)
    p.write_bytes(gzip.compress(blob[:-3]))
    with pytest.raises(ValueError, match="truncated BAM header"):
        BamHeader.read(p)
    p.write_bytes(gzip.compress(b"BAM\1" + struct.pack("<i", -5)))
    with pytest.raises(ValueError, match="truncated BAM header"):
        BamHeader.read(p)
    p.write_bytes(b"plain text, not gzip")
    with pytest.raises(gzip.BadGzipFile):
        BamHeader.read(p)
    assert BamHeader("", [], [], 0).sort_order == "unknown"


def test_auto_chunk_bytes_follows_the_reference_policy(monkeypatch):
    """cubam's rule (src/cubam/_memory.py:11-23): halve while 64 chunks do not fit the free GPU memory,
    never below 32 MB; the same sizes as cubam below 32 GB free, up to 1 GB on a B200."""
    import torch

    from cubam_b200 import auto_chunk_bytes, memory_pool

    GB, MB = 1 << 30, 1 << 20
    # free memory of an 8, 12, 16 and 24 GB GPU (cubam's docstring: about 64, 128, 128 and 256 MB)
    for free, want in ((7.5 * GB, 64 * MB), (11.5 * GB, 128 * MB), (15.5 * GB, 128 * MB), (23 * GB, 256 * MB),
                       (1 * GB, 32 * MB), (60 * GB, 512 * MB), (178 * GB, 1 * GB)):
        monkeypatch.setattr(torch.cuda, "mem_get_info", lambda free=free: (free, 2 * free))
        assert auto_chunk_bytes() == want, free
    with memory_pool():
        pass
