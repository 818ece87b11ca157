"""The BGZF writer on the GPU: DEFLATE streams that zlib inflates to their spans, checksums equal to
zlib's, framing equal to the reference's rules (the CPU oracle's), files our reader and gzip read."""

import gzip
import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA GPU", allow_module_level=True)

from oracle import bgzf_writer_oracle as W  # noqa: E402


def dev(b: bytes) -> torch.Tensor:
    return torch.frombuffer(bytearray(b), dtype=torch.uint8).cuda() if b else torch.empty(0, dtype=torch.uint8, device="cuda")


def bam_like(n: int, seed: int) -> bytes:
    rng = np.random.default_rng(seed)
    words = [b"chr1\t", b"12345\t", b"ACGTACGT", b"CB:Z:AAACCTGAGAAGG-1\x00", b"UB:Z:", b"GN:Z:Gene", b"\x01\x02", b"FFF:F,F"]
    out = bytearray()
    while len(out) < n:
        out += words[rng.integers(0, len(words))]
        if rng.integers(0, 5) == 0:
            out.append(int(rng.integers(0, 256)))
    return bytes(out[:n])


def spans(n, step):
    off = np.arange(0, n, step)
    return off, np.minimum(off + step, n) - off


@pytest.mark.parametrize("level", [0, 1, 2, 5])
def test_deflate_crc_adler_match_zlib(level):
    from cubam_b200.bgzf import _adler32_spans, _crc32_spans, _deflate_spans

    rng = np.random.default_rng(level)
    text = (b"chr1\t12345\tACGTACGT\tCB:Z:AAAC\n" * 20000)[:400_000]
    raw = text + rng.integers(0, 256, 150_000, dtype=np.uint8).tobytes() + b"z"
    d = dev(raw)
    off, size = spans(len(raw), 30_001)
    out, oo, osz = _deflate_spans(d, off, size, level, max_chunks=4)  # several native calls
    o, oo, osz = out.cpu().numpy(), oo.cpu().numpy(), osz.cpu().numpy()
    assert oo[0] == 0 and np.all(oo[1:] == oo[:-1] + osz[:-1]) and oo[-1] + osz[-1] == len(o)
    for a, b, s, n in zip(oo, osz, off, size, strict=True):
        assert W.inflate_payload(o[a : a + b].tobytes()) == raw[s : s + n]
    sp = list(zip(off, size, strict=True))
    assert _crc32_spans(d, off, size).cpu().tolist() == [zlib.crc32(raw[s : s + n]) for s, n in sp]
    assert _adler32_spans(d, off, size).cpu().tolist() == [zlib.adler32(raw[s : s + n]) for s, n in sp]


def test_bgzf_compress_and_writer(tmp_path):
    from cubam_b200.bgzf import EOF_BLOCK, BgzfWriter, _bgzf_compress, inflate_chunks

    rng = np.random.default_rng(1)
    raw = (b"ACGT" * 50_000) + rng.integers(0, 256, 200_000, dtype=np.uint8).tobytes()  # random: stored blocks
    blocks = _bgzf_compress(dev(raw)).cpu().numpy().tobytes()
    assert gzip.decompress(blocks + EOF_BLOCK) == raw
    p = tmp_path / "w.gz"
    with BgzfWriter(p, flush_bytes=100_000) as w:
        for k in range(0, len(raw), 77_777):
            w.write(dev(raw[k : k + 77_777]))
        w.write(b"end")
    assert gzip.decompress(p.read_bytes()) == raw + b"end"
    assert torch.cat(list(inflate_chunks(p, 50_000))).cpu().numpy().tobytes() == raw + b"end"
    writes = [raw[k : k + 77_777] for k in range(0, len(raw), 77_777)] + [b"end"]
    assert [m["isize"] for m in W.members(p.read_bytes()[: -len(EOF_BLOCK)])] == W.writer_blocks(writes, 100_000)
    with BgzfWriter(tmp_path / "e.gz"):
        pass
    assert (tmp_path / "e.gz").read_bytes() == EOF_BLOCK


@pytest.mark.parametrize("level", [1, 2])
def test_framing_equals_the_oracle_field_by_field(level):
    from cubam_b200.bgzf import _bgzf_compress

    rnd = np.random.default_rng(4).integers(0, 256, 140_000, dtype=np.uint8).tobytes()  # holds a whole random block
    raw = bam_like(700_000, 3) + rnd + b"A" * 90_000
    got, offs = _bgzf_compress(dev(raw), level, return_offsets=True)
    got = got.cpu().numpy().tobytes()
    want, _ = W.bgzf_compress(raw)
    gm, wm = W.members(got), W.members(want)
    assert len(gm) == len(wm)
    assert offs.cpu().tolist() == [m["offset"] for m in gm]
    for g, w in zip(gm, wm, strict=True):
        assert (g["isize"], g["crc"]) == (w["isize"], w["crc"])
        assert g["bsize"] == 26 + len(g["payload"]) <= 1 << 16
        assert W.inflate_payload(g["payload"]) == W.inflate_payload(w["payload"])
    # the random block is stored; compressible blocks are not
    kinds = [len(m["payload"]) == m["isize"] + 5 for m in gm]
    assert any(kinds) and not all(kinds)


def test_edge_spans():
    from cubam_b200.bgzf import EOF_BLOCK, _bgzf_compress, _deflate_spans

    rng = np.random.default_rng(7)
    raw = rng.integers(0, 256, 65_536, dtype=np.uint8).tobytes() + b"\x00" * 65_536 + b"xyz"
    d = dev(raw)
    # empty, 1 and 3 bytes, a full 65,536 random span (two stored blocks), a run of zeros, an odd offset
    off = [0, 5, 10, 0, 65_536, 131_071]
    size = [0, 1, 3, 65_536, 65_536, 4]
    out, oo, osz = _deflate_spans(d, off, size, 2)
    o = out.cpu().numpy()
    for a, b, s, n in zip(oo.cpu().tolist(), osz.cpu().tolist(), off, size, strict=True):
        assert W.inflate_payload(o[a : a + b].tobytes()) == raw[s : s + n]
    sizes = osz.cpu().tolist()
    assert sizes[0] == 2  # the empty stream: a fixed block with only its end code
    assert sizes[3] == 65_536 + 10  # two stored blocks
    assert sizes[4] < 300  # 64 KiB of zeros
    # an empty block framed is the EOF block
    e = _bgzf_compress(d, 2, block_off=[0], block_size=[0]).cpu().numpy().tobytes()
    assert e == EOF_BLOCK
    assert _bgzf_compress(dev(b"")).numel() == 0
    with pytest.raises(ValueError, match="at most 65,536"):
        _deflate_spans(d, [0], [65_537])
    with pytest.raises(ValueError, match="at most 65,280"):
        _bgzf_compress(d, block_off=[0], block_size=[65_281])
    with pytest.raises(ValueError, match="outside"):
        _deflate_spans(d, [len(raw) - 2], [3])


def test_output_depends_only_on_input_and_level():
    from cubam_b200.bgzf import _bgzf_compress

    raw = bam_like(3_000_000, 11)
    a = _bgzf_compress(dev(raw), 2).cpu().numpy().tobytes()
    b = _bgzf_compress(dev(b"pad" + raw)[3:], 2).cpu().numpy().tobytes()  # another alignment
    assert a == b
    c = _bgzf_compress(dev(raw), 1).cpu().numpy().tobytes()
    assert gzip.decompress(a) == raw == gzip.decompress(c)


def test_round_trip_of_a_bam_through_the_reader(tmp_path):
    """The inflated bytes of a golden BAM written again by the GPU writer read back to the same records."""
    from pathlib import Path

    import cubam_b200
    from cubam_b200.bgzf import BgzfWriter

    src = Path(__file__).parent / "golden" / "mixed_b65280.bam"
    raw = gzip.decompress(src.read_bytes())
    p = tmp_path / "again.bam"
    with BgzfWriter(p, level=2, flush_bytes=3 * 65_280) as w:
        for k in range(0, len(raw), 100_000):
            w.write(dev(raw[k : k + 100_000]))
    z6 = len(W.bgzf_compress(raw)[0])
    assert len(p.read_bytes()) < 1.25 * z6  # within a quarter of zlib level 6
    a = list(cubam_b200.read_bam(src))
    b = list(cubam_b200.read_bam(p))
    assert sum(len(x) for x in a) == sum(len(x) for x in b)
    assert torch.cat([x.pos for x in a]).cpu().tolist() == torch.cat([x.pos for x in b]).cpu().tolist()


@pytest.fixture(scope="module")
def host_model(tmp_path_factory):
    """tests/deflate_model.cu built as a host program: the kernel's DEFLATE coder on one thread."""
    import subprocess
    from pathlib import Path

    from cubam_b200 import build

    exe = tmp_path_factory.mktemp("model") / "deflate_model"
    src = Path(__file__).parent / "deflate_model.cu"
    subprocess.run([build.nvcc(), "-O2", "-std=c++17", "-Wno-deprecated-gpu-targets", str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    return exe


@pytest.mark.parametrize("level", [0, 1, 2])
def test_streams_equal_the_host_model_byte_for_byte(tmp_path, host_model, level):
    """Every stream of the GPU coder is the host model's, byte for byte (the kernel's parse, codes and
    block choice are deterministic), on BAM bytes, random bytes, runs and odd span sizes."""
    import struct
    import subprocess
    from pathlib import Path

    from cubam_b200.bgzf import _deflate_spans

    golden = gzip.decompress((Path(__file__).parent / "golden" / "mixed_b65280.bam").read_bytes())
    rnd = np.random.default_rng(31).integers(0, 256, 70_000, dtype=np.uint8).tobytes()
    raw = golden + bam_like(600_000, 5) + rnd + b"A" * 70_000 + b"ACGT" * 5_000
    rng = np.random.default_rng(level)
    off, size, o = [], [], 0
    while o < len(raw):
        n = int(min(len(raw) - o, rng.choice([65_280, 65_536, 1, 3, 4, 511, 512, 513, int(rng.integers(1, 65_536))])))
        off.append(o)
        size.append(n)
        o += n
    off.append(0)  # an empty span
    size.append(0)
    (tmp_path / "in").write_bytes(raw)
    np.stack([np.array(off, np.int64), np.array(size, np.int64)], 1).tofile(tmp_path / "spans")
    subprocess.run([str(host_model), str(tmp_path / "in"), str(tmp_path / "spans"), str(level), str(tmp_path / "out")],
                   check=True)
    want, p = [], 0
    blob = (tmp_path / "out").read_bytes()
    while p < len(blob):
        n = struct.unpack_from("<I", blob, p)[0]
        want.append(blob[p + 4 : p + 4 + n])
        p += 4 + n
    out, oo, osz = _deflate_spans(dev(raw), off, size, level)
    got = out.cpu().numpy().tobytes()
    oo, osz = oo.cpu().tolist(), osz.cpu().tolist()
    assert len(want) == len(off)
    for i, (a, b) in enumerate(zip(oo, osz, strict=True)):
        assert got[a : a + b] == want[i], (i, off[i], size[i])


def test_writer_flush_ends_blocks_and_failures_are_raised(tmp_path, monkeypatch):
    """flush() ends a block early (the oracle's block sizes); a write that fails in the writer thread is
    raised by the owner's next call."""
    import os

    from cubam_b200.bgzf import EOF_BLOCK, BgzfWriter

    rng = np.random.default_rng(5)
    parts = [rng.integers(65, 70, k, dtype=np.uint8).tobytes() for k in (1000, 70_000, 5, 200_000, 65_280)]
    p = tmp_path / "f.gz"
    with BgzfWriter(p, flush_bytes=100_000) as w:
        for i, part in enumerate(parts):
            w.write(dev(part))
            if i in (0, 2):
                w.flush()
    assert gzip.decompress(p.read_bytes()) == b"".join(parts)
    sizes = [m["isize"] for m in W.members(p.read_bytes()[: -len(EOF_BLOCK)])]
    assert sizes == W.writer_blocks(parts, 100_000, flushes=(0, 2))
    real = os.pwrite
    calls = []

    def failing(fd, data, offset):
        calls.append(offset)
        if len(calls) > 1:
            raise OSError(28, "injected: no space left")
        return real(fd, data, offset)

    monkeypatch.setattr(os, "pwrite", failing)
    w = BgzfWriter(tmp_path / "g.gz", flush_bytes=65_280, n_threads=1)
    with pytest.raises(OSError, match="injected"):
        try:
            for part in parts * 3:
                w.write(dev(part))
        finally:
            w.close()
