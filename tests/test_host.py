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
    r = _ChunkReader(GOLDEN / "text_b1000.gz", 10_000, n_buffers=2, n_threads=3, piece=3333)
    got = bytearray()
    for slot, n, eof in r:
        got += r.host(slot)[:n].numpy().tobytes()
        r.release(slot)
    r.close()
    assert bytes(got) == raw


def test_chunk_reader_error_reaches_the_consumer(tmp_path):
    import pytest

    from cubam_b200.bgzf import _ChunkReader

    r = _ChunkReader(tmp_path / "missing.bam", 4096)
    with pytest.raises(FileNotFoundError):
        list(r)
